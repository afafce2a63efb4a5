/* Interpolation types and accelerators (GSL 2 API names); only the natural cubic spline is
   implemented (ref_gsl.c).  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_GSL_INTERP_H
#define RG_SHIM_GSL_INTERP_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct { size_t cache, miss_count, hit_count; } gsl_interp_accel;
typedef struct { const char* name; unsigned int min_size; } gsl_interp_type;
extern const gsl_interp_type* gsl_interp_cspline;
extern const gsl_interp_type* gsl_interp_linear;
gsl_interp_accel* gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel* a);
#ifdef __cplusplus
}
#endif
#endif
