/* The logging calls of the reference (its mlog submodule is not vendored): messages go to
   stderr when RG_REF_VERBOSE is set, errors always.  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_MLOG_H
#define RG_SHIM_MLOG_H
#include <stdbool.h>
#include "mpi.h"
#ifdef __cplusplus
extern "C" {
#endif

#define MLOG_MESG 0x1
#define MLOG_OPEN 0x2
#define MLOG_CLOSE 0x4
#define MLOG_CONT 0x8
#define MLOG_TIMERSTART 0x10
#define MLOG_TIMERSTOP 0x20
#define MLOG_FLUSH 0x40
#define MLOG_ALLRANKS 0x80

void mlog(const char* fmt, int flags, ...);
void mlog_error(const char* fmt, ...);

#ifdef __cplusplus
}
#endif
#endif
