/* The random-number generator type of GSL (GSL 2 API names).  The reionization step draws no
   random numbers; ref_stubs.c makes these calls abort.  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_GSL_RNG_H
#define RG_SHIM_GSL_RNG_H
#ifdef __cplusplus
extern "C" {
#endif
typedef struct { const char* name; } gsl_rng_type;
typedef struct { const gsl_rng_type* type; void* state; } gsl_rng;
extern const gsl_rng_type* gsl_rng_ranlxd1;
extern const gsl_rng_type* gsl_rng_default;
gsl_rng* gsl_rng_alloc(const gsl_rng_type* T);
void gsl_rng_set(const gsl_rng* r, unsigned long int s);
void gsl_rng_free(gsl_rng* r);
double gsl_rng_uniform(const gsl_rng* r);
#ifdef __cplusplus
}
#endif
#endif
