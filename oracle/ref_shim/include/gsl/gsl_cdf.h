/* Cumulative distributions (GSL 2 API names): declarations only; the reionization step calls
   none of them (ref_stubs.c makes them abort). */
#ifndef RG_SHIM_GSL_CDF_H
#define RG_SHIM_GSL_CDF_H
#ifdef __cplusplus
extern "C" {
#endif
double gsl_cdf_ugaussian_Pinv(double P);
double gsl_cdf_ugaussian_P(double x);
double gsl_cdf_gaussian_Pinv(double P, double sigma);
double gsl_cdf_gaussian_P(double x, double sigma);
double gsl_cdf_gaussian_Qinv(double Q, double sigma);
#ifdef __cplusplus
}
#endif
#endif
