/* The GSL routines the reference's reionization step calls, restated from GSL's published
 * algorithms -- TEST INFRASTRUCTURE ONLY (oracle/_ref).
 *
 * - gsl_spline with gsl_interp_cspline: the natural cubic spline (second derivatives zero at
 *   both ends), coefficients from the symmetric tridiagonal system of the knots, the interval by
 *   binary search (x equal to the last knot uses the last interval), evaluation in the form
 *   y_i + dx (b_i + dx (c_i + dx d_i)); x outside the knots is a domain error.
 * - gsl_integration_qag with GSL_INTEG_GAUSS61: QUADPACK's QAGE (bisect the interval of largest
 *   error estimate; roundoff and subinterval-size tests) with the 61-point Gauss-Kronrod rule of
 *   ref_gk61.h, which the build generates from oracle/gk61.py.
 * - gsl_root_fsolver_brent and gsl_root_test_interval: Brent's method (Brent 1973, the GSL
 *   iteration) and GSL's interval test.
 * - errors: GSL's handler convention; the reference switches the handler off at start-up
 *   (src/core/init.c:257), and rg_ref_init does the same.
 */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/gsl_errno.h"
#include "gsl/gsl_integration.h"
#include "gsl/gsl_interp.h"
#include "gsl/gsl_roots.h"
#include "gsl/gsl_spline.h"
#include "ref_gk61.h"

/* ---- errors ---- */

static void default_handler(const char* reason, const char* file, int line, int gsl_errno) {
  fprintf(stderr, "gsl: %s:%d: ERROR: %s (%d)\n", file, line, reason, gsl_errno);
  abort();
}
static gsl_error_handler_t* g_handler = default_handler;

void gsl_error(const char* reason, const char* file, int line, int gsl_errno) {
  if (g_handler) g_handler(reason, file, line, gsl_errno);
}
gsl_error_handler_t* gsl_set_error_handler(gsl_error_handler_t* h) {
  gsl_error_handler_t* old = g_handler;
  g_handler = h;
  return old;
}
static void no_handler(const char* reason, const char* file, int line, int gsl_errno) {
  (void)reason;
  (void)file;
  (void)line;
  (void)gsl_errno;
}
gsl_error_handler_t* gsl_set_error_handler_off(void) { return gsl_set_error_handler(no_handler); }

const char* gsl_strerror(const int e) {
  switch (e) {
    case GSL_SUCCESS: return "success";
    case GSL_FAILURE: return "failure";
    case GSL_CONTINUE: return "the iteration has not converged yet";
    case GSL_EDOM: return "input domain error";
    case GSL_EINVAL: return "invalid argument supplied by user";
    case GSL_EMAXITER: return "exceeded max number of iterations";
    case GSL_EROUND: return "failed because of roundoff error";
    case GSL_ESING: return "apparent singularity detected";
    case GSL_EBADFUNC: return "problem with user-supplied function";
    default: return "unknown error code";
  }
}
#define SHIM_ERROR(reason, code)              \
  do {                                        \
    gsl_error(reason, __FILE__, __LINE__, code); \
    return code;                              \
  } while (0)

/* ---- interpolation ---- */

static const gsl_interp_type cspline_type = {"cspline", 3};
static const gsl_interp_type linear_type = {"linear", 2};
const gsl_interp_type* gsl_interp_cspline = &cspline_type;
const gsl_interp_type* gsl_interp_linear = &linear_type;

gsl_interp_accel* gsl_interp_accel_alloc(void) { return (gsl_interp_accel*)calloc(1, sizeof(gsl_interp_accel)); }
void gsl_interp_accel_free(gsl_interp_accel* a) { free(a); }

gsl_spline* gsl_spline_alloc(const gsl_interp_type* T, size_t size) {
  if (T != gsl_interp_cspline || size < 3) {
    fprintf(stderr, "ref_gsl: only natural cubic splines of 3 or more knots are provided\n");
    abort();
  }
  gsl_spline* s = (gsl_spline*)calloc(1, sizeof(gsl_spline));
  s->type = T;
  s->size = size;
  s->x = (double*)malloc(sizeof(double) * size);
  s->y = (double*)malloc(sizeof(double) * size);
  s->c2 = (double*)malloc(sizeof(double) * size);
  return s;
}

void gsl_spline_free(gsl_spline* s) {
  if (!s) return;
  free(s->x);
  free(s->y);
  free(s->c2);
  free(s);
}

int gsl_spline_init(gsl_spline* s, const double xa[], const double ya[], size_t n) {
  if (n != s->size) SHIM_ERROR("data must match size of spline object", GSL_EINVAL);
  for (size_t i = 1; i < n; ++i)
    if (!(xa[i] > xa[i - 1])) SHIM_ERROR("x values must be strictly increasing", GSL_EINVAL);
  memcpy(s->x, xa, sizeof(double) * n);
  memcpy(s->y, ya, sizeof(double) * n);
  /* c_i (half the second derivative) at the interior knots from
       h_{i-1} c_{i-1} + 2 (h_{i-1} + h_i) c_i + h_i c_{i+1} = 3 (dy_i / h_i - dy_{i-1} / h_{i-1}),
     c_0 = c_{n-1} = 0, solved by symmetric tridiagonal elimination */
  const size_t m = n - 2;
  double* diag = (double*)malloc(sizeof(double) * (m ? m : 1));
  double* off = (double*)malloc(sizeof(double) * (m ? m : 1));
  double* rhs = (double*)malloc(sizeof(double) * (m ? m : 1));
  for (size_t i = 0; i < m; ++i) {
    const double h0 = xa[i + 1] - xa[i], h1 = xa[i + 2] - xa[i + 1];
    diag[i] = 2.0 * (h0 + h1);
    off[i] = h1;
    rhs[i] = 3.0 * ((ya[i + 2] - ya[i + 1]) / h1 - (ya[i + 1] - ya[i]) / h0);
  }
  for (size_t i = 1; i < m; ++i) {
    const double w = off[i - 1] / diag[i - 1];
    diag[i] -= w * off[i - 1];
    rhs[i] -= w * rhs[i - 1];
  }
  s->c2[0] = 0.0;
  s->c2[n - 1] = 0.0;
  for (size_t k = m; k-- > 0;) {
    const double nxt = (k + 1 < m) ? s->c2[k + 2] : 0.0;
    s->c2[k + 1] = (rhs[k] - off[k] * nxt) / diag[k];
  }
  free(diag);
  free(off);
  free(rhs);
  return GSL_SUCCESS;
}

static size_t bsearch_interval(const double* xa, double x, size_t lo, size_t hi) {
  while (hi > lo + 1) {
    const size_t mid = (hi + lo) / 2;
    if (xa[mid] > x)
      hi = mid;
    else
      lo = mid;
  }
  return lo;
}

double gsl_spline_eval(const gsl_spline* s, double x, gsl_interp_accel* a) {
  const size_t n = s->size;
  if (x < s->x[0] || x > s->x[n - 1]) {
    gsl_error("interpolation error", __FILE__, __LINE__, GSL_EDOM);
    return NAN;
  }
  size_t i;
  if (a && a->cache < n - 1 && s->x[a->cache] <= x && x < s->x[a->cache + 1]) {
    i = a->cache;
    a->hit_count++;
  } else {
    i = bsearch_interval(s->x, x, 0, n - 1);
    if (a) {
      a->cache = i;
      a->miss_count++;
    }
  }
  const double xl = s->x[i], xh = s->x[i + 1];
  const double dx = xh - xl, dy = s->y[i + 1] - s->y[i];
  const double ci = s->c2[i], cn = s->c2[i + 1];
  const double b = dy / dx - dx * (cn + 2.0 * ci) / 3.0;
  const double d = (cn - ci) / (3.0 * dx);
  const double t = x - xl;
  return s->y[i] + t * (b + t * (ci + t * d));
}

/* ---- QAG with the 61-point Gauss-Kronrod rule ---- */

gsl_integration_workspace* gsl_integration_workspace_alloc(const size_t n) {
  gsl_integration_workspace* w = (gsl_integration_workspace*)calloc(1, sizeof(*w));
  w->limit = n;
  w->alist = (double*)malloc(sizeof(double) * n);
  w->blist = (double*)malloc(sizeof(double) * n);
  w->rlist = (double*)malloc(sizeof(double) * n);
  w->elist = (double*)malloc(sizeof(double) * n);
  w->order = (size_t*)malloc(sizeof(size_t) * n);
  w->level = (size_t*)malloc(sizeof(size_t) * n);
  return w;
}

void gsl_integration_workspace_free(gsl_integration_workspace* w) {
  if (!w) return;
  free(w->alist);
  free(w->blist);
  free(w->rlist);
  free(w->elist);
  free(w->order);
  free(w->level);
  free(w);
}

static double rescale_error(double err, double result_abs, double result_asc) {
  err = fabs(err);
  if (result_asc != 0 && err != 0) {
    const double scale = pow(200 * err / result_asc, 1.5);
    err = scale < 1 ? result_asc * scale : result_asc;
  }
  if (result_abs > DBL_MIN / (50 * DBL_EPSILON)) {
    const double min_err = 50 * DBL_EPSILON * result_abs;
    if (min_err > err) err = min_err;
  }
  return err;
}

/* the rule: xgk[31] (descending, xgk[30] = 0), wgk[31], wg_full[30] (Gauss weights at the odd
   positions of xgk, zero at the Kronrod-only ones) */
static void qk61(const gsl_function* f, double a, double b, double* result, double* abserr, double* resabs,
                 double* resasc) {
  const int n = 31;
  double fv1[31], fv2[31];
  const double center = 0.5 * (a + b);
  const double half = 0.5 * (b - a);
  const double abs_half = fabs(half);
  const double fc = GSL_FN_EVAL(f, center);
  double rg = 0.0, rk = fc * RG_REF_WGK[n - 1];
  double rabs = fabs(rk), rasc;
  for (int j = 0; j < (n - 1) / 2; ++j) {
    const int jtw = 2 * j + 1;
    const double x = half * RG_REF_XGK[jtw];
    const double f1 = GSL_FN_EVAL(f, center - x), f2 = GSL_FN_EVAL(f, center + x);
    fv1[jtw] = f1;
    fv2[jtw] = f2;
    rg += RG_REF_WG[jtw] * (f1 + f2);
    rk += RG_REF_WGK[jtw] * (f1 + f2);
    rabs += RG_REF_WGK[jtw] * (fabs(f1) + fabs(f2));
  }
  for (int j = 0; j < n / 2; ++j) {
    const int jtwm1 = 2 * j;
    const double x = half * RG_REF_XGK[jtwm1];
    const double f1 = GSL_FN_EVAL(f, center - x), f2 = GSL_FN_EVAL(f, center + x);
    fv1[jtwm1] = f1;
    fv2[jtwm1] = f2;
    rk += RG_REF_WGK[jtwm1] * (f1 + f2);
    rabs += RG_REF_WGK[jtwm1] * (fabs(f1) + fabs(f2));
  }
  const double mean = rk * 0.5;
  rasc = RG_REF_WGK[n - 1] * fabs(fc - mean);
  for (int j = 0; j < n - 1; ++j) rasc += RG_REF_WGK[j] * (fabs(fv1[j] - mean) + fabs(fv2[j] - mean));
  const double err = (rk - rg) * half;
  *result = rk * half;
  *resabs = rabs * abs_half;
  *resasc = rasc * abs_half;
  *abserr = rescale_error(err, *resabs, *resasc);
}

static size_t largest_error(const gsl_integration_workspace* w) {
  size_t im = 0;
  for (size_t i = 1; i < w->size; ++i)
    if (w->elist[i] > w->elist[im]) im = i;
  return im;
}

int gsl_integration_qag(const gsl_function* f, double a, double b, double epsabs, double epsrel, size_t limit,
                        int key, gsl_integration_workspace* w, double* result, double* abserr) {
  *result = 0;
  *abserr = 0;
  if (key != GSL_INTEG_GAUSS61) {
    fprintf(stderr, "ref_gsl: only GSL_INTEG_GAUSS61 is provided\n");
    abort();
  }
  if (limit > w->limit) SHIM_ERROR("iteration limit exceeds available workspace", GSL_EINVAL);
  if (epsabs <= 0 && (epsrel < 50 * DBL_EPSILON || epsrel < 0.5e-28))
    SHIM_ERROR("tolerance cannot be achieved with given epsabs and epsrel", GSL_EINVAL);
  double r0, e0, ra0, rc0;
  qk61(f, a, b, &r0, &e0, &ra0, &rc0);
  w->size = 1;
  w->alist[0] = a;
  w->blist[0] = b;
  w->rlist[0] = r0;
  w->elist[0] = e0;
  w->level[0] = 0;
  double tolerance = fmax(epsabs, epsrel * fabs(r0));
  const double round_off = 50 * DBL_EPSILON * ra0;
  if (e0 <= round_off && e0 > tolerance) {
    *result = r0;
    *abserr = e0;
    SHIM_ERROR("cannot reach tolerance because of roundoff error on first attempt", GSL_EROUND);
  } else if ((e0 <= tolerance && e0 != rc0) || e0 == 0.0) {
    *result = r0;
    *abserr = e0;
    return GSL_SUCCESS;
  } else if (limit == 1) {
    *result = r0;
    *abserr = e0;
    SHIM_ERROR("a maximum of one iteration was insufficient", GSL_EMAXITER);
  }
  double area = r0, errsum = e0;
  size_t iteration = 1;
  int rt1 = 0, rt2 = 0, error_type = 0;
  do {
    const size_t im = largest_error(w);
    const double a_i = w->alist[im], b_i = w->blist[im], r_i = w->rlist[im], e_i = w->elist[im];
    const double a1 = a_i, b1 = 0.5 * (a_i + b_i), a2 = b1, b2 = b_i;
    double area1, error1, resabs1, resasc1, area2, error2, resabs2, resasc2;
    qk61(f, a1, b1, &area1, &error1, &resabs1, &resasc1);
    qk61(f, a2, b2, &area2, &error2, &resabs2, &resasc2);
    const double area12 = area1 + area2, error12 = error1 + error2;
    errsum += (error12 - e_i);
    area += area12 - r_i;
    if (resasc1 != error1 && resasc2 != error2) {
      const double delta = r_i - area12;
      if (fabs(delta) <= 1.0e-5 * fabs(area12) && error12 >= 0.99 * e_i) rt1++;
      if (iteration >= 10 && error12 > e_i) rt2++;
    }
    tolerance = fmax(epsabs, epsrel * fabs(area));
    if (errsum > tolerance) {
      if (rt1 >= 6 || rt2 >= 20) error_type = 2;
      const double tmp = (1 + 100 * DBL_EPSILON) * (fabs(a2) + 1000 * DBL_MIN);
      if (fabs(a1) <= tmp && fabs(b2) <= tmp) error_type = 3;
    }
    /* the half with the larger error keeps the bisected interval's slot */
    const size_t in = w->size;
    const size_t lev = w->level[im] + 1;
    if (error2 > error1) {
      w->alist[im] = a2;
      w->rlist[im] = area2;
      w->elist[im] = error2;
      w->level[im] = lev;
      w->alist[in] = a1;
      w->blist[in] = b1;
      w->rlist[in] = area1;
      w->elist[in] = error1;
      w->level[in] = lev;
    } else {
      w->blist[im] = b1;
      w->rlist[im] = area1;
      w->elist[im] = error1;
      w->level[im] = lev;
      w->alist[in] = a2;
      w->blist[in] = b2;
      w->rlist[in] = area2;
      w->elist[in] = error2;
      w->level[in] = lev;
    }
    w->size++;
    iteration++;
  } while (iteration < limit && !error_type && errsum > tolerance);
  double sum = 0.0;
  for (size_t k = 0; k < w->size; ++k) sum += w->rlist[k];
  *result = sum;
  *abserr = errsum;
  if (errsum <= tolerance) return GSL_SUCCESS;
  if (error_type == 2) SHIM_ERROR("roundoff error prevents tolerance from being achieved", GSL_EROUND);
  if (error_type == 3) SHIM_ERROR("bad integrand behavior found in the integration interval", GSL_ESING);
  if (iteration == limit) SHIM_ERROR("maximum number of subdivisions reached", GSL_EMAXITER);
  SHIM_ERROR("could not integrate function", GSL_FAILURE);
}

/* ---- Brent's root finder ---- */

static const gsl_root_fsolver_type brent_type = {"brent"};
const gsl_root_fsolver_type* gsl_root_fsolver_brent = &brent_type;

gsl_root_fsolver* gsl_root_fsolver_alloc(const gsl_root_fsolver_type* T) {
  gsl_root_fsolver* s = (gsl_root_fsolver*)calloc(1, sizeof(*s));
  s->type = T;
  return s;
}
void gsl_root_fsolver_free(gsl_root_fsolver* s) { free(s); }

int gsl_root_fsolver_set(gsl_root_fsolver* s, gsl_function* f, double x_lower, double x_upper) {
  if (x_lower > x_upper) SHIM_ERROR("invalid interval (lower > upper)", GSL_EINVAL);
  s->function = f;
  s->root = 0.5 * (x_lower + x_upper);
  s->x_lower = x_lower;
  s->x_upper = x_upper;
  const double fl = GSL_FN_EVAL(f, x_lower), fu = GSL_FN_EVAL(f, x_upper);
  s->a = x_lower;
  s->fa = fl;
  s->b = x_upper;
  s->fb = fu;
  s->c = x_upper;
  s->fc = fu;
  s->d = x_upper - x_lower;
  s->e = x_upper - x_lower;
  if ((fl < 0.0 && fu < 0.0) || (fl > 0.0 && fu > 0.0)) SHIM_ERROR("endpoints do not straddle y=0", GSL_EINVAL);
  return GSL_SUCCESS;
}

int gsl_root_fsolver_iterate(gsl_root_fsolver* s) {
  double a = s->a, b = s->b, c = s->c, d = s->d, e = s->e, fa = s->fa, fb = s->fb, fc = s->fc;
  int ac_equal = 0;
  if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) {
    ac_equal = 1;
    c = a;
    fc = fa;
    d = b - a;
    e = b - a;
  }
  if (fabs(fc) < fabs(fb)) {
    ac_equal = 1;
    a = b;
    b = c;
    c = a;
    fa = fb;
    fb = fc;
    fc = fa;
  }
  const double tol = 0.5 * DBL_EPSILON * fabs(b);
  const double m = 0.5 * (c - b);
  if (fb == 0) {
    s->root = b;
    s->x_lower = b;
    s->x_upper = b;
    return GSL_SUCCESS;
  }
  if (fabs(m) <= tol) {
    s->root = b;
    if (b < c) {
      s->x_lower = b;
      s->x_upper = c;
    } else {
      s->x_lower = c;
      s->x_upper = b;
    }
    return GSL_SUCCESS;
  }
  if (fabs(e) < tol || fabs(fa) <= fabs(fb)) {
    d = m;
    e = m;
  } else {
    double p, q, r;
    const double sr = fb / fa;
    if (ac_equal) {
      p = 2 * m * sr;
      q = 1 - sr;
    } else {
      q = fa / fc;
      r = fb / fc;
      p = sr * (2 * m * q * (q - r) - (b - a) * (r - 1));
      q = (q - 1) * (r - 1) * (sr - 1);
    }
    if (p > 0)
      q = -q;
    else
      p = -p;
    if (2 * p < fmin(3 * m * q - fabs(tol * q), fabs(e * q))) {
      e = d;
      d = p / q;
    } else {
      d = m;
      e = m;
    }
  }
  a = b;
  fa = fb;
  if (fabs(d) > tol)
    b += d;
  else
    b += (m > 0 ? +tol : -tol);
  fb = GSL_FN_EVAL(s->function, b);
  if (!isfinite(fb)) SHIM_ERROR("function value is not finite", GSL_EBADFUNC);
  s->a = a;
  s->b = b;
  s->c = c;
  s->d = d;
  s->e = e;
  s->fa = fa;
  s->fb = fb;
  s->fc = fc;
  s->root = b;
  if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) c = a;
  if (b < c) {
    s->x_lower = b;
    s->x_upper = c;
  } else {
    s->x_lower = c;
    s->x_upper = b;
  }
  return GSL_SUCCESS;
}

double gsl_root_fsolver_root(const gsl_root_fsolver* s) { return s->root; }
double gsl_root_fsolver_x_lower(const gsl_root_fsolver* s) { return s->x_lower; }
double gsl_root_fsolver_x_upper(const gsl_root_fsolver* s) { return s->x_upper; }

int gsl_root_test_interval(double x_lower, double x_upper, double epsabs, double epsrel) {
  if (epsrel < 0.0) SHIM_ERROR("relative tolerance is negative", GSL_EBADTOL);
  if (epsabs < 0.0) SHIM_ERROR("absolute tolerance is negative", GSL_EBADTOL);
  if (x_lower > x_upper) SHIM_ERROR("lower bound larger than upper bound", GSL_EINVAL);
  const double abs_lower = fabs(x_lower), abs_upper = fabs(x_upper);
  double min_abs;
  if ((x_lower > 0.0 && x_upper > 0.0) || (x_lower < 0.0 && x_upper < 0.0))
    min_abs = fmin(abs_lower, abs_upper);
  else
    min_abs = 0;
  const double tolerance = epsabs + epsrel * min_abs;
  if (fabs(x_upper - x_lower) < tolerance) return GSL_SUCCESS;
  return GSL_CONTINUE;
}
