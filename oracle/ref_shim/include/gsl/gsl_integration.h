/* QAG with the Gauss-Kronrod rules (GSL 2 API names); only GSL_INTEG_GAUSS61 is implemented
   (ref_gsl.c).  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_GSL_INTEGRATION_H
#define RG_SHIM_GSL_INTEGRATION_H
#include <stddef.h>
#include "gsl_math.h"
#ifdef __cplusplus
extern "C" {
#endif
enum { GSL_INTEG_GAUSS15 = 1, GSL_INTEG_GAUSS21 = 2, GSL_INTEG_GAUSS31 = 3, GSL_INTEG_GAUSS41 = 4,
       GSL_INTEG_GAUSS51 = 5, GSL_INTEG_GAUSS61 = 6 };
typedef struct {
  size_t limit, size, nrmax, i, maximum_level;
  double *alist, *blist, *rlist, *elist;
  size_t *order, *level;
} gsl_integration_workspace;
gsl_integration_workspace* gsl_integration_workspace_alloc(const size_t n);
void gsl_integration_workspace_free(gsl_integration_workspace* w);
int gsl_integration_qag(const gsl_function* f, double a, double b, double epsabs, double epsrel, size_t limit,
                        int key, gsl_integration_workspace* workspace, double* result, double* abserr);
#ifdef __cplusplus
}
#endif
#endif
