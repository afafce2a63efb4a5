/* Random distributions (GSL 2 API names): declarations only, see gsl_rng.h. */
#ifndef RG_SHIM_GSL_RANDIST_H
#define RG_SHIM_GSL_RANDIST_H
#include "gsl_rng.h"
#ifdef __cplusplus
extern "C" {
#endif
double gsl_ran_gaussian(const gsl_rng* r, double sigma);
double gsl_ran_lognormal(const gsl_rng* r, double zeta, double sigma);
unsigned int gsl_ran_poisson(const gsl_rng* r, double mu);
#ifdef __cplusplus
}
#endif
#endif
