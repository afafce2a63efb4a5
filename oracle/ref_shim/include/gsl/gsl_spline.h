/* gsl_spline (GSL 2 API names) over the natural cubic spline of ref_gsl.c.  Test
   infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_GSL_SPLINE_H
#define RG_SHIM_GSL_SPLINE_H
#include <stddef.h>
#include "gsl_interp.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct {
  const gsl_interp_type* type;
  size_t size;
  double *x, *y, *c2;   /* knots, values, second derivatives */
} gsl_spline;
gsl_spline* gsl_spline_alloc(const gsl_interp_type* T, size_t size);
int gsl_spline_init(gsl_spline* spline, const double xa[], const double ya[], size_t size);
double gsl_spline_eval(const gsl_spline* spline, double x, gsl_interp_accel* a);
void gsl_spline_free(gsl_spline* spline);
#ifdef __cplusplus
}
#endif
#endif
