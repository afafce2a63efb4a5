/* Declarations of the single-precision FFTW 3 calls the reference's reionization step makes
   (fftw3.h of FFTW 3.3 API, names and signatures only).  Implemented by ref_fft.c over an
   in-tree double-precision FFT.  Test infrastructure for oracle/_ref only. */
#ifndef RG_SHIM_FFTW3_H
#define RG_SHIM_FFTW3_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* <complex.h> precedes this header in the reference, so FFTW uses the C99 complex type */
typedef float _Complex fftwf_complex;
typedef struct rg_shim_fftwf_plan_s* fftwf_plan;

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

float* fftwf_alloc_real(size_t n);
fftwf_complex* fftwf_alloc_complex(size_t n);
void* fftwf_malloc(size_t n);
void fftwf_free(void* p);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float* in, fftwf_complex* out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex* in, float* out, unsigned flags);
int fftwf_import_wisdom_from_filename(const char* filename);
int fftwf_export_wisdom_to_filename(const char* filename);
void fftwf_cleanup(void);

#ifdef __cplusplus
}
#endif
#endif
