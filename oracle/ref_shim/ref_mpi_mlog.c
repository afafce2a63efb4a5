/* One MPI rank and the logging calls, for the reference's reionization sources -- TEST
 * INFRASTRUCTURE ONLY (oracle/_ref).  With one rank every collective leaves (MPI_IN_PLACE) or
 * copies its buffer; a point-to-point call has no partner and aborts.  Log messages go to
 * stderr when RG_REF_VERBOSE is set; errors always do.
 */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mlog.h"
#include "mpi.h"

static size_t type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_BYTE:
    case MPI_CHAR:
    case MPI_C_BOOL: return 1;
    case MPI_INT:
    case MPI_UNSIGNED:
    case MPI_FLOAT: return 4;
    case MPI_LONG:
    case MPI_LONG_LONG:
    case MPI_DOUBLE: return 8;
    default: fprintf(stderr, "ref_mpi: unknown datatype %d\n", t); abort();
  }
}

static void copy_in(const void* s, void* r, int count, MPI_Datatype t) {
  if (s == MPI_IN_PLACE || s == r) return;
  memcpy(r, s, (size_t)count * type_size(t));
}

int MPI_Init(int* argc, char*** argv) {
  (void)argc;
  (void)argv;
  return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
void rg_ref_on_abort(int code); /* ref_driver.c */

int MPI_Abort(MPI_Comm comm, int code) {
  (void)comm;
  fprintf(stderr, "ref_mpi: MPI_Abort(%d)\n", code);
  rg_ref_on_abort(code);
  return code;
}
int MPI_Comm_rank(MPI_Comm comm, int* rank) {
  (void)comm;
  *rank = 0;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm comm, int* size) {
  (void)comm;
  *size = 1;
  return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm comm) {
  (void)comm;
  return MPI_SUCCESS;
}
int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm comm) {
  (void)buf;
  (void)count;
  (void)t;
  (void)root;
  (void)comm;
  return MPI_SUCCESS;
}
int MPI_Allreduce(const void* s, void* r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm) {
  (void)op;
  (void)comm;
  copy_in(s, r, count, t);
  return MPI_SUCCESS;
}
int MPI_Reduce(const void* s, void* r, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm) {
  (void)op;
  (void)root;
  (void)comm;
  copy_in(s, r, count, t);
  return MPI_SUCCESS;
}
int MPI_Allgather(const void* s, int scount, MPI_Datatype st, void* r, int rcount, MPI_Datatype rt, MPI_Comm comm) {
  (void)rcount;
  (void)rt;
  (void)comm;
  copy_in(s, r, scount, st);
  return MPI_SUCCESS;
}
int MPI_Allgatherv(const void* s, int scount, MPI_Datatype st, void* r, const int* rcounts, const int* displs,
                   MPI_Datatype rt, MPI_Comm comm) {
  (void)rcounts;
  (void)comm;
  if (s == MPI_IN_PLACE) return MPI_SUCCESS;
  memcpy((char*)r + (size_t)displs[0] * type_size(rt), s, (size_t)scount * type_size(st));
  return MPI_SUCCESS;
}
static int no_partner(const char* what) {
  fprintf(stderr, "ref_mpi: %s has no partner on one rank\n", what);
  abort();
}
int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm) {
  (void)buf, (void)count, (void)t, (void)dest, (void)tag, (void)comm;
  return no_partner("MPI_Send");
}
int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Status* st) {
  (void)buf, (void)count, (void)t, (void)src, (void)tag, (void)comm, (void)st;
  return no_partner("MPI_Recv");
}
int MPI_Sendrecv(const void* sbuf, int scount, MPI_Datatype stype, int dest, int stag, void* rbuf, int rcount,
                 MPI_Datatype rtype, int src, int rtag, MPI_Comm comm, MPI_Status* st) {
  (void)rcount, (void)rtype, (void)stag, (void)rtag, (void)comm, (void)st;
  if (dest == 0 && src == 0) {
    memcpy(rbuf, sbuf, (size_t)scount * type_size(stype));
    return MPI_SUCCESS;
  }
  return no_partner("MPI_Sendrecv");
}

void mlog(const char* fmt, int flags, ...) {
  (void)flags;
  if (!getenv("RG_REF_VERBOSE")) return;
  va_list ap;
  va_start(ap, flags);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fputc('\n', stderr);
}

void mlog_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  fputs("reference error: ", stderr);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fputc('\n', stderr);
}
