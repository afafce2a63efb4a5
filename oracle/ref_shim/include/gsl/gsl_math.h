/* gsl_function, as GSL declares it.  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_GSL_MATH_H
#define RG_SHIM_GSL_MATH_H
#include <math.h>
typedef struct gsl_function_struct {
  double (*function)(double x, void* params);
  void* params;
} gsl_function;
#define GSL_FN_EVAL(F, x) (*((F)->function))(x, (F)->params)
#endif
