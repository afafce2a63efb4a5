/* GSL error codes and calls used by the reference (GSL 2 API names).  Implemented in
   ref_gsl.c.  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_GSL_ERRNO_H
#define RG_SHIM_GSL_ERRNO_H
#ifdef __cplusplus
extern "C" {
#endif
enum { GSL_SUCCESS = 0, GSL_FAILURE = -1, GSL_CONTINUE = -2, GSL_EDOM = 1, GSL_EINVAL = 4, GSL_EMAXITER = 11,
       GSL_EROUND = 18, GSL_ESING = 21, GSL_EBADTOL = 13, GSL_ETOL = 14, GSL_EBADFUNC = 9, GSL_ENOMEM = 8 };
typedef void gsl_error_handler_t(const char* reason, const char* file, int line, int gsl_errno);
const char* gsl_strerror(const int gsl_errno);
gsl_error_handler_t* gsl_set_error_handler(gsl_error_handler_t* h);
gsl_error_handler_t* gsl_set_error_handler_off(void);
void gsl_error(const char* reason, const char* file, int line, int gsl_errno);
#ifdef __cplusplus
}
#endif
#endif
