/* The single-precision FFTW plans the reference's reionization step makes, over an in-tree
 * double-precision FFT -- TEST INFRASTRUCTURE ONLY (oracle/_ref).
 *
 * FFTW semantics kept: r2c is unnormalised (sign -1) from a real array whose last dimension is
 * padded to 2 (n2/2 + 1) floats (the layout fftwf_mpi plans use, in place or not) into
 * n0 x n1 x (n2/2 + 1) complex values; c2r is the unnormalised inverse (sign +1) of a Hermitian
 * half spectrum into the padded real layout, and may run in place.  Each transform is computed
 * in double (mixed-radix Cooley-Tukey over the smallest prime factors, twiddles from libm's
 * cos/sin) and rounded to float once, so it is at least as accurate as FFTW's float plans; the
 * rounding of single values differs from FFTW's.  One MPI rank holds the whole grid.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3-mpi.h"

typedef struct {
  double re, im;
} cd;

enum { KIND_R2C = 1, KIND_C2R = 2 };

struct rg_shim_fftwf_plan_s {
  int kind;
  int n0, n1, n2;
  float* real;
  fftwf_complex* cplx;
};

static void* xmalloc(size_t n) {
  void* p = NULL;
  if (posix_memalign(&p, 64, n ? n : 1) != 0) {
    fprintf(stderr, "ref_fft: out of memory (%zu bytes)\n", n);
    abort();
  }
  return p;
}

/* ---- 1-D complex FFT of length n (any n), sign -1 (forward) or +1 (backward) ---- */

typedef struct {
  int n, sign;
  cd* w; /* w[j] = exp(sign 2 pi i j / n) */
} fft1d;

static void fft1d_init(fft1d* f, int n, int sign) {
  f->n = n;
  f->sign = sign;
  f->w = (cd*)xmalloc(sizeof(cd) * (size_t)n);
  for (int j = 0; j < n; ++j) {
    const double a = 2.0 * M_PI * (double)j / (double)n;
    f->w[j].re = cos(a);
    f->w[j].im = sign * sin(a);
  }
}

static int smallest_factor(int n) {
  if (n % 4 == 0) return 4;
  for (int p = 2; p * p <= n; ++p)
    if (n % p == 0) return p;
  return n;
}

/* y[0..n) = DFT of x[0], x[xs], ..., x[(n-1) xs] with twiddles W^(wstep k) of the top-level table */
static void fft_rec(const fft1d* f, const cd* x, size_t xs, cd* y, int n, int wstep) {
  if (n == 1) {
    y[0] = x[0];
    return;
  }
  const int N = f->n;
  const int p = smallest_factor(n);
  const int m = n / p;
  for (int r = 0; r < p; ++r) fft_rec(f, x + (size_t)r * xs, xs * (size_t)p, y + (size_t)r * m, m, wstep * p);
  cd t[64];
  cd* tt = p <= 64 ? t : (cd*)xmalloc(sizeof(cd) * (size_t)p);
  for (int k = 0; k < m; ++k) {
    for (int r = 0; r < p; ++r) {
      const cd v = y[(size_t)r * m + k];
      const cd w = f->w[((long long)wstep * r * k) % N];
      tt[r].re = v.re * w.re - v.im * w.im;
      tt[r].im = v.re * w.im + v.im * w.re;
    }
    for (int q = 0; q < p; ++q) {
      double sr = 0.0, si = 0.0;
      for (int r = 0; r < p; ++r) {
        const cd w = f->w[((long long)wstep * m * r * q) % N];
        sr += tt[r].re * w.re - tt[r].im * w.im;
        si += tt[r].re * w.im + tt[r].im * w.re;
      }
      y[(size_t)q * m + k].re = sr;
      y[(size_t)q * m + k].im = si;
    }
  }
  if (tt != t) free(tt);
}

/* in-place transform of `line` (length f->n) using `tmp` (same length) */
static void fft1d_run(const fft1d* f, cd* line, cd* tmp) {
  fft_rec(f, line, 1, tmp, f->n, 1);
  memcpy(line, tmp, sizeof(cd) * (size_t)f->n);
}

/* ---- 3-D transforms ---- */

static void transform_axes01(cd* a, int n0, int n1, int nh, int sign) {
  /* along axis 1 (stride nh), then axis 0 (stride n1 nh), for every kz */
  fft1d f1, f0;
  fft1d_init(&f1, n1, sign);
  fft1d_init(&f0, n0, sign);
  const int nl = n0 > n1 ? n0 : n1;
  cd* line = (cd*)xmalloc(sizeof(cd) * (size_t)nl);
  cd* tmp = (cd*)xmalloc(sizeof(cd) * (size_t)nl);
  for (int i = 0; i < n0; ++i)
    for (int k = 0; k < nh; ++k) {
      cd* base = a + (size_t)i * n1 * nh + k;
      for (int j = 0; j < n1; ++j) line[j] = base[(size_t)j * nh];
      fft1d_run(&f1, line, tmp);
      for (int j = 0; j < n1; ++j) base[(size_t)j * nh] = line[j];
    }
  for (int j = 0; j < n1; ++j)
    for (int k = 0; k < nh; ++k) {
      cd* base = a + (size_t)j * nh + k;
      for (int i = 0; i < n0; ++i) line[i] = base[(size_t)i * n1 * nh];
      fft1d_run(&f0, line, tmp);
      for (int i = 0; i < n0; ++i) base[(size_t)i * n1 * nh] = line[i];
    }
  free(line);
  free(tmp);
  free(f1.w);
  free(f0.w);
}

static void exec_r2c(const struct rg_shim_fftwf_plan_s* p) {
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2, nh = n2 / 2 + 1, pad = 2 * nh;
  cd* a = (cd*)xmalloc(sizeof(cd) * (size_t)n0 * n1 * nh);
  fft1d f2;
  fft1d_init(&f2, n2, -1);
  cd* line = (cd*)xmalloc(sizeof(cd) * (size_t)n2);
  cd* tmp = (cd*)xmalloc(sizeof(cd) * (size_t)n2);
  for (int i = 0; i < n0; ++i)
    for (int j = 0; j < n1; ++j) {
      const float* row = p->real + ((size_t)i * n1 + j) * pad;
      for (int k = 0; k < n2; ++k) {
        line[k].re = row[k];
        line[k].im = 0.0;
      }
      fft1d_run(&f2, line, tmp);
      memcpy(a + ((size_t)i * n1 + j) * nh, line, sizeof(cd) * (size_t)nh);
    }
  free(line);
  free(tmp);
  free(f2.w);
  transform_axes01(a, n0, n1, nh, -1);
  float* out = (float*)p->cplx;
  for (size_t e = 0; e < (size_t)n0 * n1 * nh; ++e) {
    out[2 * e] = (float)a[e].re;
    out[2 * e + 1] = (float)a[e].im;
  }
  free(a);
}

static void exec_c2r(const struct rg_shim_fftwf_plan_s* p) {
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2, nh = n2 / 2 + 1, pad = 2 * nh;
  cd* a = (cd*)xmalloc(sizeof(cd) * (size_t)n0 * n1 * nh);
  const float* in = (const float*)p->cplx;
  for (size_t e = 0; e < (size_t)n0 * n1 * nh; ++e) {
    a[e].re = in[2 * e];
    a[e].im = in[2 * e + 1];
  }
  transform_axes01(a, n0, n1, nh, +1);
  /* last axis: Hermitian half line -> real line (the imaginary parts of the k = 0 and, for even
     n2, k = n2/2 terms do not enter a real result) */
  fft1d f2;
  fft1d_init(&f2, n2, +1);
  cd* line = (cd*)xmalloc(sizeof(cd) * (size_t)n2);
  cd* tmp = (cd*)xmalloc(sizeof(cd) * (size_t)n2);
  for (int i = 0; i < n0; ++i)
    for (int j = 0; j < n1; ++j) {
      const cd* h = a + ((size_t)i * n1 + j) * nh;
      for (int k = 0; k < nh; ++k) line[k] = h[k];
      line[0].im = 0.0;
      if (n2 % 2 == 0) line[n2 / 2].im = 0.0;
      for (int k = nh; k < n2; ++k) {
        line[k].re = h[n2 - k].re;
        line[k].im = -h[n2 - k].im;
      }
      fft1d_run(&f2, line, tmp);
      float* row = p->real + ((size_t)i * n1 + j) * pad;
      for (int k = 0; k < n2; ++k) row[k] = (float)line[k].re;
      for (int k = n2; k < pad; ++k) row[k] = 0.0f;
    }
  free(line);
  free(tmp);
  free(f2.w);
  free(a);
}

/* ---- the FFTW API ---- */

float* fftwf_alloc_real(size_t n) { return (float*)xmalloc(sizeof(float) * n); }
fftwf_complex* fftwf_alloc_complex(size_t n) { return (fftwf_complex*)xmalloc(sizeof(fftwf_complex) * n); }
void* fftwf_malloc(size_t n) { return xmalloc(n); }
void fftwf_free(void* p) { free(p); }

static fftwf_plan make_plan(int kind, ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, float* real, fftwf_complex* c) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0 || n0 > (1 << 16) || n1 > (1 << 16) || n2 > (1 << 16)) {
    fprintf(stderr, "ref_fft: invalid plan size %td x %td x %td\n", n0, n1, n2);
    abort();
  }
  struct rg_shim_fftwf_plan_s* p = (struct rg_shim_fftwf_plan_s*)calloc(1, sizeof(*p));
  p->kind = kind;
  p->n0 = (int)n0;
  p->n1 = (int)n1;
  p->n2 = (int)n2;
  p->real = real;
  p->cplx = c;
  return p;
}

fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float* in, fftwf_complex* out, unsigned flags) {
  (void)flags;
  return make_plan(KIND_R2C, n0, n1, n2, in, out);
}
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex* in, float* out, unsigned flags) {
  (void)flags;
  return make_plan(KIND_C2R, n0, n1, n2, out, in);
}
fftwf_plan fftwf_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, float* in, fftwf_complex* out,
                                     MPI_Comm comm, unsigned flags) {
  (void)comm;
  (void)flags;
  return make_plan(KIND_R2C, n0, n1, n2, in, out);
}
fftwf_plan fftwf_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftwf_complex* in, float* out,
                                     MPI_Comm comm, unsigned flags) {
  (void)comm;
  (void)flags;
  return make_plan(KIND_C2R, n0, n1, n2, out, in);
}

void fftwf_execute(const fftwf_plan p) {
  if (!p) {
    fprintf(stderr, "ref_fft: fftwf_execute on a NULL plan\n");
    abort();
  }
  if (p->kind == KIND_R2C)
    exec_r2c(p);
  else
    exec_c2r(p);
}

void fftwf_destroy_plan(fftwf_plan p) { free(p); }

ptrdiff_t fftwf_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm comm, ptrdiff_t* local_n0,
                                  ptrdiff_t* local_0_start) {
  (void)comm;
  *local_n0 = n0;
  *local_0_start = 0;
  return n0 * n1 * n2;
}

void fftwf_mpi_init(void) {}
void fftwf_mpi_cleanup(void) {}
void fftwf_cleanup(void) {}
void fftwf_mpi_gather_wisdom(MPI_Comm comm) { (void)comm; }
void fftwf_mpi_broadcast_wisdom(MPI_Comm comm) { (void)comm; }
int fftwf_import_wisdom_from_filename(const char* filename) {
  (void)filename;
  return 0;
}
int fftwf_export_wisdom_to_filename(const char* filename) {
  (void)filename;
  return 1;
}
