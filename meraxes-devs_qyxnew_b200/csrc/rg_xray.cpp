// Host FP64 coefficient engine of the spin-temperature step.  See rg_xray.h.
#include "rg_xray.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>

#include "rg_gk61.h"
#include "rg_internal.h"

namespace rg {

// ---------------------------------------------------------------------------
// QAG with the 61-point Gauss-Kronrod rule (QUADPACK's QAGE, Piessens et al. 1983)

static double rescale_error(double err, double result_abs, double result_asc) {
  err = std::fabs(err);
  if (result_asc != 0 && err != 0) {
    const double scale = std::pow((200 * err / result_asc), 1.5);
    err = scale < 1 ? result_asc * scale : result_asc;
  }
  if (result_abs > DBL_MIN / (50 * DBL_EPSILON)) {
    const double min_err = 50 * DBL_EPSILON * result_abs;
    if (min_err > err) err = min_err;
  }
  return err;
}

static void qk61(const std::function<double(double)>& f, double a, double b, double* result, double* abserr,
                 double* resabs, double* resasc) {
  const double center = 0.5 * (a + b);
  const double half_length = 0.5 * (b - a);
  const double abs_half_length = std::fabs(half_length);
  const double f_center = f(center);
  double result_gauss = 0;  // the 30-point Gauss rule has no centre node
  double result_kronrod = f_center * GK61_WK[30];
  double result_abs = std::fabs(result_kronrod);
  double fv1[30], fv2[30];
  for (int k = 0; k < 30; ++k) {
    const double abscissa = half_length * GK61_X[k];
    const double f1 = f(center - abscissa);
    const double f2 = f(center + abscissa);
    const double fsum = f1 + f2;
    fv1[k] = f1;
    fv2[k] = f2;
    result_gauss += GK61_WG[k] * fsum;
    result_kronrod += GK61_WK[k] * fsum;
    result_abs += GK61_WK[k] * (std::fabs(f1) + std::fabs(f2));
  }
  const double mean = result_kronrod * 0.5;
  double result_asc = GK61_WK[30] * std::fabs(f_center - mean);
  for (int k = 0; k < 30; ++k) result_asc += GK61_WK[k] * (std::fabs(fv1[k] - mean) + std::fabs(fv2[k] - mean));
  const double err = (result_kronrod - result_gauss) * half_length;
  result_kronrod *= half_length;
  result_abs *= abs_half_length;
  result_asc *= abs_half_length;
  *result = result_kronrod;
  *resabs = result_abs;
  *resasc = result_asc;
  *abserr = rescale_error(err, result_abs, result_asc);
}

int qag61(const std::function<double(double)>& f, double a, double b, double epsabs, double epsrel, int limit,
          double* result, double* abserr) {
  struct Iv {
    double a, b, r, e;
  };
  double r0, e0, ra0, rc0;
  qk61(f, a, b, &r0, &e0, &ra0, &rc0);
  double tolerance = std::fmax(epsabs, epsrel * std::fabs(r0));
  const double round_off = 50 * DBL_EPSILON * ra0;
  *result = r0;
  *abserr = e0;
  if (e0 <= round_off && e0 > tolerance) return 2;                 // roundoff
  if ((e0 <= tolerance && e0 != rc0) || e0 == 0.0) return 0;
  if (limit == 1) return 3;
  std::vector<Iv> iv;
  iv.reserve(limit);
  iv.push_back({a, b, r0, e0});
  double area = r0, errsum = e0;
  int iteration = 1, roundoff_type1 = 0, roundoff_type2 = 0, error_type = 0;
  do {
    // the interval with the largest error
    size_t im = 0;
    for (size_t i = 1; i < iv.size(); ++i)
      if (iv[i].e > iv[im].e) im = i;
    const Iv cur = iv[im];
    const double a1 = cur.a, b1 = 0.5 * (cur.a + cur.b), a2 = b1, b2 = cur.b;
    double area1, error1, resabs1, resasc1, area2, error2, resabs2, resasc2;
    qk61(f, a1, b1, &area1, &error1, &resabs1, &resasc1);
    qk61(f, a2, b2, &area2, &error2, &resabs2, &resasc2);
    const double area12 = area1 + area2, error12 = error1 + error2;
    errsum += (error12 - cur.e);
    area += area12 - cur.r;
    if (resasc1 != error1 && resasc2 != error2) {
      const double delta = cur.r - area12;
      if (std::fabs(delta) <= 1.0e-5 * std::fabs(area12) && error12 >= 0.99 * cur.e) roundoff_type1++;
      if (iteration >= 10 && error12 > cur.e) roundoff_type2++;
    }
    tolerance = std::fmax(epsabs, epsrel * std::fabs(area));
    if (errsum > tolerance) {
      if (roundoff_type1 >= 6 || roundoff_type2 >= 20) error_type = 2;
      const double tmp = (1 + 100 * DBL_EPSILON) * (std::fabs(a2) + 1000 * DBL_MIN);
      if (std::fabs(a1) <= tmp && std::fabs(b2) <= tmp) error_type = 3;
    }
    iv[im] = {a1, b1, area1, error1};
    iv.push_back({a2, b2, area2, error2});
    iteration++;
  } while (iteration < limit && !error_type && errsum > tolerance);
  double sum = 0;
  for (const auto& x : iv) sum += x.r;
  *result = sum;
  *abserr = errsum;
  if (errsum <= tolerance) return 0;
  if (error_type) return error_type;
  return 1;  // iteration limit
}

// ---------------------------------------------------------------------------
// Brent's method (Brent 1973), the iteration GSL's brent solver performs

double brent_root(const std::function<double(double)>& fn, double x_lower, double x_upper, double epsabs,
                  double epsrel, int max_iter, int* status) {
  double a = x_lower, b = x_upper;
  double fa = fn(a), fb = fn(b);
  *status = 0;
  if ((fa < 0.0 && fb < 0.0) || (fa > 0.0 && fb > 0.0)) {
    *status = 1;  // endpoints do not straddle zero
    return b;
  }
  double c = b, fc = fb, d = b - a, e = b - a;
  double root = b, lo = x_lower, hi = x_upper;
  for (int iter = 1; iter <= max_iter; ++iter) {
    bool ac_equal = false;
    if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) {
      ac_equal = true;
      c = a;
      fc = fa;
      d = b - a;
      e = b - a;
    }
    if (std::fabs(fc) < std::fabs(fb)) {
      ac_equal = true;
      a = b;
      b = c;
      c = a;
      fa = fb;
      fb = fc;
      fc = fa;
    }
    const double tol = 0.5 * DBL_EPSILON * std::fabs(b);
    const double m = 0.5 * (c - b);
    if (fb == 0) {
      root = b;
      lo = hi = b;
    } else if (std::fabs(m) <= tol) {
      root = b;
      lo = b < c ? b : c;
      hi = b < c ? c : b;
    } else {
      if (std::fabs(e) < tol || std::fabs(fa) <= std::fabs(fb)) {
        d = m;  // bisection
        e = m;
      } else {
        double p, q, r;
        const double s = fb / fa;
        if (ac_equal) {
          p = 2 * m * s;
          q = 1 - s;
        } else {
          q = fa / fc;
          r = fb / fc;
          p = s * (2 * m * q * (q - r) - (b - a) * (r - 1));
          q = (q - 1) * (r - 1) * (s - 1);
        }
        if (p > 0)
          q = -q;
        else
          p = -p;
        if (2 * p < std::fmin(3 * m * q - std::fabs(tol * q), std::fabs(e * q))) {
          e = d;
          d = p / q;
        } else {
          d = m;  // interpolation failed, bisect
          e = m;
        }
      }
      a = b;
      fa = fb;
      if (std::fabs(d) > tol)
        b += d;
      else
        b += (m > 0 ? +tol : -tol);
      fb = fn(b);
      root = b;
      if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) c = a;
      lo = b < c ? b : c;
      hi = b < c ? c : b;
    }
    // gsl_root_test_interval(lo, hi, epsabs, epsrel)
    const double abs_lo = std::fabs(lo), abs_hi = std::fabs(hi);
    const double min_abs = ((lo > 0 && hi > 0) || (lo < 0 && hi < 0)) ? std::fmin(abs_lo, abs_hi) : 0;
    if (std::fabs(hi - lo) < epsabs + epsrel * min_abs) return root;
  }
  *status = 2;
  return root;
}

// ---------------------------------------------------------------------------
// cosmology (XRayHeatingFunctions.c:426-552, 1595-1637; reionization.h:15-32)

Cosmo::Cosmo(const rg_params* prm) : p(prm) {
  const double h = p->Hubble_h;
  const double RHOcrit_cgs = 3.0 * HUBBLE * HUBBLE * h * h / (8.0 * M_PI * GRAVITY);
  const double OMb = p->BaryonFrac * p->OmegaM;
  No = RHOcrit_cgs * OMb * (1 - p->Y_He) / PROTONMASS;
  He_No = RHOcrit_cgs * OMb * p->Y_He / (4.0 * PROTONMASS);
  N_b0 = No + He_No;
  f_H = No / (No + He_No);
  f_He = He_No / (No + He_No);
}

double Cosmo::dtdz(float z) const {
  const double OMl = p->OmegaLambda, OMm = p->OmegaM;
  const double opz = (double)(1.0f + z);  // 1 + z is a float sum in the C
  const double x = std::sqrt(OMl / OMm) * std::pow(opz, -3.0 / 2.0);
  const double dxdz = std::sqrt(OMl / OMm) * std::pow(opz, -5.0 / 2.0) * (-3.0 / 2.0);
  const double const1 = 2 * std::sqrt(1 + OMm / OMl) / (3.0 * HUBBLE * p->Hubble_h);
  const double numer = dxdz * (1 + x * std::pow(std::pow(x, 2) + 1, -0.5));
  const double denom = x + std::sqrt(std::pow(x, 2) + 1);
  return const1 * numer / denom;
}

double Cosmo::drdz(float z) const { return (1.0 + (double)z) * SPEED_OF_LIGHT * dtdz(z); }

double Cosmo::hubble(float z) const {
  const double opz = (double)(1.0f + z);
  return HUBBLE * p->Hubble_h *
         std::sqrt(p->OmegaM * std::pow(opz, 3) + p->OmegaR * std::pow(opz, 4) + p->OmegaLambda);
}

double Cosmo::dicke(double z) const {
  const double tiny = 1e-4;
  const double OMm = p->OmegaM, OMl = p->OmegaLambda, OMr = p->OmegaR, OMk = p->OmegaK, wl = p->wLambda;
  const double OMtot = OMm + OMl + OMr + OMk;
  if (std::fabs(OMm - 1.0) < tiny) return 1.0 / (1.0 + z);
  if ((OMl > (-tiny)) && (std::fabs(OMl + OMm + OMr - 1.0) < 0.01) && (std::fabs(wl + 1.0) < tiny)) {
    const double omegaM_z = OMm * std::pow(1 + z, 3) / (OMl + OMm * std::pow(1 + z, 3) + OMr * std::pow(1 + z, 4));
    const double dick_z =
        2.5 * omegaM_z / (1.0 / 70.0 + omegaM_z * (209 - omegaM_z) / 140.0 + std::pow(omegaM_z, 4.0 / 7.0));
    const double dick_0 = 2.5 * OMm / (1.0 / 70.0 + OMm * (209 - OMm) / 140.0 + std::pow(OMm, 4.0 / 7.0));
    return dick_z / (dick_0 * (1.0 + z));
  }
  if ((OMtot < (1 + tiny)) && (std::fabs(OMl) < tiny)) {
    const double x_0 = 1.0 / (OMm + 0.0) - 1.0;
    const double dick_0 = 1 + 3.0 / x_0 + 3 * std::log(std::sqrt(1 + x_0) - std::sqrt(x_0)) * std::sqrt(1 + x_0) /
                                             std::pow(x_0, 1.5);
    const double x = std::fabs(1.0 / (OMm + 0.0) - 1.0) / (1 + z);
    const double dick_z =
        1 + 3.0 / x + 3 * std::log(std::sqrt(1 + x) - std::sqrt(x)) * std::sqrt(1 + x) / std::pow(x, 1.5);
    return dick_z / dick_0;
  }
  return -1;
}

double Cosmo::ddicke_dz(double z) const {
  const float dz = 1e-10f;
  return (dicke(z + dz) - dicke(z)) / dz;
}

// cross sections (XRayHeatingFunctions.c:471-516)
double HeI_ion_crosssec(double nu) {
  if (nu < HeI_NUIONIZATION) return 0;
  const double x = nu / NU_over_EV / 13.61 - 0.4434;
  const double y = std::sqrt(x * x + std::pow(2.136, 2));
  return 9.492e-16 * ((x - 1) * (x - 1) + 2.039 * 2.039) * std::pow(y, (0.5 * 3.188 - 5.5)) *
         std::pow(1.0 + std::sqrt(y / 1.469), -3.188);
}

double HeII_ion_crosssec(double nu) {
  const double Z = 2;
  if (nu < HeII_NUIONIZATION) return 0;
  if (nu == HeII_NUIONIZATION) nu += TINY;
  const double epsilon = std::sqrt(nu / HeII_NUIONIZATION - 1);
  return (6.3e-18) / Z / Z * std::pow(HeII_NUIONIZATION / nu, 4) * std::exp(4 - (4 * std::atan(epsilon) / epsilon)) /
         (1 - std::exp(-2 * M_PI / epsilon));
}

double HI_ion_crosssec(double nu) {
  const double Z = 1;
  if (nu < NUIONIZATION) return 0;
  if (nu == NUIONIZATION) nu += TINY;
  const double epsilon = std::sqrt(nu / NUIONIZATION - 1);
  return SIGMA_HI / Z / Z * std::pow(NUIONIZATION / nu, 4) * std::exp(4 - (4 * std::atan(epsilon) / epsilon)) /
         (1 - std::exp(-2 * M_PI / epsilon));
}

// electron interpolation tables (XRayHeatingFunctions.c:970-1276), float arithmetic as in the C
static int locate_energy_index(float En) {
  if (En < 1008.88f) return (int)(std::log((double)En / 10.0) / 1.98026273e-2);
  return 232 + (int)(std::log((double)En / 1008.88) / 9.53101798e-2);
}

int locate_xHII_index(const Tables& t, float xHII_call) {
  int m = x_int_NXHII - 1;
  while (xHII_call < t.x_int_XHII[m]) m--;
  return m;
}

float interp_x_int(const Tables& t, const std::vector<float>& tab, float En, float xHII_call, float below) {
  const float* E = t.x_int_Energy.data();
  const float* X = t.x_int_XHII.data();
  if ((double)En > 0.999 * (double)E[x_int_NENERGY - 1]) {
    En = (float)((double)E[x_int_NENERGY - 1] * 0.999);
  } else if (En < E[0]) {
    return below;
  }
  if ((double)xHII_call > (double)X[x_int_NXHII - 1] * 0.999) {
    xHII_call = (float)((double)X[x_int_NXHII - 1] * 0.999);
  } else if (xHII_call < X[0]) {
    xHII_call = (float)(1.001 * (double)X[0]);
  }
  const int n_low = locate_energy_index(En), n_high = n_low + 1;
  const int m_low = locate_xHII_index(t, xHII_call), m_high = m_low + 1;
  const float* lo = tab.data() + (size_t)m_low * x_int_NENERGY;
  const float* hi = tab.data() + (size_t)m_high * x_int_NENERGY;
  float elow = ((lo[n_high] - lo[n_low]) / (E[n_high] - E[n_low]));
  elow *= (En - E[n_low]);
  elow += lo[n_low];
  float ehigh = ((hi[n_high] - hi[n_low]) / (E[n_high] - E[n_low]));
  ehigh *= (En - E[n_low]);
  ehigh += hi[n_low];
  float r = (ehigh - elow) / (X[m_high] - X[m_low]);
  r *= (xHII_call - X[m_low]);
  r += elow;
  return r;
}

float zmax(float z, int n) {
  const double num = 1 - std::pow(n + 1, -2);
  const double denom = 1 - std::pow(n, -2);
  return (float)((double)(1.0f + z) * num / denom - 1);
}

double nu_n(int n) {
  double ans = 1.0 - std::pow(n, -2.0);
  ans /= 0.75;
  return ans;
}

double frecycle(int n) {
  static const double f[31] = {1,      1,      1,      0,      0.2609, 0.3078, 0.3259, 0.3353, 0.3410, 0.3448, 0.3476,
                               0.3496, 0.3512, 0.3524, 0.3535, 0.3543, 0.3550, 0.3556, 0.3561, 0.3565, 0.3569, 0.3572,
                               0.3575, 0.3578, 0.3580, 0.3582, 0.3584, 0.3586, 0.3587, 0.3589, 0.3590};
  return (n >= 0 && n <= 30) ? f[n] : 0;
}

double spectral_emissivity(const Tables& t, double nu_norm) {
  // flag 0, Pop II (XRayHeatingFunctions.c:709-727)
  for (int i = 1; i < (NSPEC_MAX - 1); i++) {
    if ((nu_norm >= t.spec_nu[i]) && (nu_norm < t.spec_nu[i + 1])) {
      const double ans = t.spec_N0_2[i] * std::pow(nu_norm, (double)t.spec_alpha2[i]);
      return ans / NU_LA;
    }
  }
  const int i = NSPEC_MAX - 1;
  return t.spec_N0_2[i] * std::pow(nu_norm, (double)t.spec_alpha2[i]) / NU_LA;
}

// ---------------------------------------------------------------------------
// shells and the SFR-history combination (ComputeTs.c:339-478)

TsShells ts_shells(const rg_params* p, const double* ZZ, int n_snap, int snapshot, int n_hist) {
  TsShells sh;
  const Cosmo cm(p);
  const int nS = p->TsNumFilterSteps;
  sh.nS = nS;
  sh.nsrc = 1 + n_hist;
  const double box_size = p->BoxSize / p->Hubble_h;  // Mpc
  const int N = p->ReionGridDim;
  const double zp = ZZ[snapshot];
  const double prev_redshift = snapshot == 0 ? ZZ[snapshot] : ZZ[snapshot - 1];
  const double dzp = zp - prev_redshift;
  const double dt_dzp = cm.dtdz((float)zp);
  double R = L_FACTOR * box_size / (float)N;
  const double R_factor = std::pow(R_XLy_MAX / R, 1 / (float)nS);
  sh.R.assign(nS, 0);
  sh.zpp_edge.assign(nS, 0);
  sh.zpp.assign(nS, 0);
  sh.dzpp.assign(nS, 0);
  sh.dt_dzpp.assign(nS, 0);
  sh.coef.assign((size_t)nS * sh.nsrc, 0.f);
  std::vector<int> scb(nS, 0);   // snapshot_counter_backwards
  std::vector<float> cur(sh.nsrc, 0.f);
  cur[0] = 1.f;                  // grids->sfr starts as this snapshot's grid
  auto hist = [&](int idx) -> int {  // source index of sfr_histories[idx]
    if (idx < 0 || idx >= n_hist) {
      sh.error = true;
      sh.msg = "the SFR history needs more snapshots than n_hist provides";
      return -1;
    }
    return 1 + idx;
  };
  auto load = [&](int idx, double weight, int new_load) {  // load_reion_sfr_grids (float weight)
    const int k = hist(idx);
    if (k < 0) return;
    const float w = (float)weight;
    if (new_load) std::fill(cur.begin(), cur.end(), 0.f);
    cur[k] += w;
  };
  double weight = 1;
  scb[0] = 1;
  for (int R_ct = 0; R_ct < nS; R_ct++) {
    sh.R[R_ct] = R;
    double prev_zpp, prev_R;
    if (R_ct == 0) {
      prev_zpp = zp;
      prev_R = 0;
    } else {
      prev_zpp = sh.zpp_edge[R_ct - 1];
      prev_R = sh.R[R_ct - 1];
      scb[R_ct] = scb[R_ct - 1];
    }
    sh.zpp_edge[R_ct] = prev_zpp - (R - prev_R) * MPC / (cm.drdz((float)prev_zpp));
    const double zpp = (sh.zpp_edge[R_ct] + prev_zpp) * 0.5;
    const double total_weight = (prev_zpp - sh.zpp_edge[R_ct]) * cm.dtdz((float)zpp);
    if (snapshot - scb[R_ct] >= 0) {
      if (snapshot - scb[R_ct] == 0 && weight < 0) {
        std::fill(cur.begin(), cur.end(), 0.f);
        scb[R_ct] += 1;
      } else if (sh.zpp_edge[R_ct] > ZZ[snapshot - scb[R_ct]]) {
        if (R_ct == 0) {
          weight = dt_dzp * dzp / total_weight;
          for (auto& v : cur) v = (float)((double)v * weight);
        } else {
          if (ZZ[snapshot - scb[R_ct]] > sh.zpp_edge[R_ct - 1]) {
            weight = -cm.dtdz((float)(0.5 * (ZZ[snapshot - scb[R_ct]] + sh.zpp_edge[R_ct - 1])));
            weight *= (ZZ[snapshot - scb[R_ct]] - sh.zpp_edge[R_ct - 1]);
            weight /= total_weight;
            load(scb[R_ct] - 1, weight, 1);
          } else {
            std::fill(cur.begin(), cur.end(), 0.f);
          }
        }
        while (sh.zpp_edge[R_ct] > ZZ[snapshot - scb[R_ct]]) {
          if (snapshot - scb[R_ct] == 0) {
            weight = -1;
            break;
          }
          if (sh.zpp_edge[R_ct] < ZZ[snapshot - scb[R_ct] - 1]) {
            const double zedge = prev_zpp > ZZ[snapshot - scb[R_ct]] ? prev_zpp : ZZ[snapshot - scb[R_ct]];
            weight = sh.zpp_edge[R_ct] - zedge;
            weight *= -cm.dtdz((float)(0.5 * (sh.zpp_edge[R_ct] + zedge)));
          } else {
            weight = ZZ[snapshot - scb[R_ct] - 1] - ZZ[snapshot - scb[R_ct]];
            weight *= -cm.dtdz((float)(0.5 * (ZZ[snapshot - scb[R_ct] - 1] + ZZ[snapshot - scb[R_ct]])));
          }
          weight /= total_weight;
          load(scb[R_ct], weight, 0);
          scb[R_ct] += 1;
        }
      } else {
        if (R_ct > 0) {
          if (weight != 1) {
            weight = 1;
            load(scb[R_ct] - 1, weight, 1);
          }
        }
      }
    }
    for (int k = 0; k < sh.nsrc; ++k) sh.coef[(size_t)R_ct * sh.nsrc + k] = cur[k];
    R *= R_factor;
    if (sh.error) return sh;
  }
  (void)n_snap;
  sh.final_weight = weight;
  // shell redshifts and widths of the evolveInt sums (XRayHeatingFunctions.c:1379-1389)
  for (int ct = 0; ct < nS; ++ct) {
    if (ct == 0) {
      sh.zpp[ct] = (sh.zpp_edge[0] + zp) * 0.5;
      sh.dzpp[ct] = zp - sh.zpp_edge[0];
    } else {
      sh.zpp[ct] = (sh.zpp_edge[ct] + sh.zpp_edge[ct - 1]) * 0.5;
      sh.dzpp[ct] = sh.zpp_edge[ct - 1] - sh.zpp_edge[ct];
    }
    sh.dt_dzpp[ct] = cm.dtdz((float)sh.zpp[ct]);
  }
  return sh;
}

// ---------------------------------------------------------------------------
// frequency tables (ComputeTs.c:761-1011)

int ts_tables(const rg_params* p, const Tables& t, const TsShells& sh, double zp, double x_e_ave,
              double collapse_fraction, const double* ZZ, const double* stored_fcoll, int snapshot, TsTables* out,
              std::string* msg) {
  const Cosmo cm(p);
  const int nS = sh.nS;
  out->heat.assign((size_t)x_int_NXHII * nS, 0);
  out->ion.assign((size_t)x_int_NXHII * nS, 0);
  out->lya.assign((size_t)x_int_NXHII * nS, 0);
  out->sum_lyn.assign(nS, 0);
  const double ion_eff = p->ReionEfficiency;
  // interpolate_fcoll (XRayHeatingFunctions.c:2010-2026); stored_fcoll[snapshot] is this step's
  auto fcoll_at = [&](double redshift) {
    double v;
    if (snapshot == 0)
      v = collapse_fraction;
    else
      v = stored_fcoll[snapshot - 1] +
          (redshift - ZZ[snapshot - 1]) * (collapse_fraction - stored_fcoll[snapshot - 1]) / (ZZ[snapshot] - ZZ[snapshot - 1]);
    return v < 0.0 ? 0.0 : v;
  };
  auto sigma_tilde = [&](double nu, double x_e) {
    return cm.f_H * (1 - x_e) * HI_ion_crosssec(nu) + cm.f_He * (1 - x_e) * HeI_ion_crosssec(nu) +
           cm.f_He * x_e * HeII_ion_crosssec(nu);
  };
  // tauX (XRayHeatingFunctions.c:339-424)
  auto tauX = [&](double nu, double x_e, double zpv, double zpp) {
    const double nu_0 = nu / (1 + zpv);
    auto integrand = [&](double zhat) {
      const double drpropdz = SPEED_OF_LIGHT * cm.dtdz((float)zhat);
      const double n = cm.N_b0 * std::pow(1 + zhat, 3);
      const double nuhat = nu_0 * (1 + zhat);
      const double fcoll = fcoll_at(zhat);
      double ff = fcoll < 1e-20 ? 1 : 1 - (ion_eff * fcoll) / (1.0 - x_e_ave);
      if (ff < 1e-4) ff = 1e-4;
      return drpropdz * n * ff * sigma_tilde(nuhat, x_e);
    };
    double result, error;
    const int status = qag61(integrand, zpp, zpv, 0, 0.005, 1000, &result, &error);
    if (status != 0) return 1e10;
    return result;
  };
  auto nu_tau_one = [&](double zpv, double zpp, double x_e) {
    if (x_e > 0.9999) return -1.0;
    if (tauX(HeI_NUIONIZATION, x_e, zpv, zpp) < 1) return HeI_NUIONIZATION;
    int st = 0;
    return brent_root([&](double nu) { return tauX(nu, x_e, zpv, zpp) - 1; }, HeI_NUIONIZATION, 1e6 * NU_over_EV, 0,
                      0.02, 100, &st);
  };
  const double thresh = p->NuXrayThreshold;
  // integrate_over_nu (XRayHeatingFunctions.c:742-856) for the spectral index alpha
  auto integrate_over_nu = [&](double local_x_e, double lo, double hi, int FLAG, double alpha) {
    if (lo >= hi) return 0.0;
    const float xf = (float)local_x_e;
    auto pw = [&](double nu) { return std::pow(nu / (thresh * NU_over_EV), -alpha - 1); };
    std::function<double(double)> f;
    if (FLAG == 0) {
      f = [&](double nu) {
        double s = interp_x_int(t, t.fheat, (float)((nu - NUIONIZATION) / NU_over_EV), xf, 1.0f) * PLANCK *
                   (nu - NUIONIZATION) * cm.f_H * (1 - local_x_e) * HI_ion_crosssec(nu);
        s += interp_x_int(t, t.fheat, (float)((nu - HeI_NUIONIZATION) / NU_over_EV), xf, 1.0f) * PLANCK *
             (nu - HeI_NUIONIZATION) * cm.f_He * (1 - local_x_e) * HeI_ion_crosssec(nu);
        s += interp_x_int(t, t.fheat, (float)((nu - HeII_NUIONIZATION) / NU_over_EV), xf, 1.0f) * PLANCK *
             (nu - HeII_NUIONIZATION) * cm.f_He * local_x_e * HeII_ion_crosssec(nu);
        return s * pw(nu);
      };
    } else if (FLAG == 1) {
      f = [&](double nu) {
        auto Fi = [&](double e0) {
          const float en = (float)((nu - e0) / NU_over_EV);
          return interp_x_int(t, t.nion_HI, en, xf, 0.0f) + interp_x_int(t, t.nion_HeI, en, xf, 0.0f) +
                 interp_x_int(t, t.nion_HeII, en, xf, 0.0f) + 1;
        };
        double s = Fi(NUIONIZATION) * cm.f_H * (1 - local_x_e) * HI_ion_crosssec(nu);
        s += Fi(HeI_NUIONIZATION) * cm.f_He * (1 - local_x_e) * HeI_ion_crosssec(nu);
        s += Fi(HeII_NUIONIZATION) * cm.f_He * local_x_e * HeII_ion_crosssec(nu);
        return s * pw(nu);
      };
    } else {
      f = [&](double nu) {
        double s = interp_x_int(t, t.n_Lya, (float)((nu - NUIONIZATION) / NU_over_EV), xf, 0.0f) * cm.f_H *
                   (1 - local_x_e) * HI_ion_crosssec(nu);
        s += interp_x_int(t, t.n_Lya, (float)((nu - HeI_NUIONIZATION) / NU_over_EV), xf, 0.0f) * cm.f_He *
             (1 - local_x_e) * HeI_ion_crosssec(nu);
        s += interp_x_int(t, t.n_Lya, (float)((nu - HeII_NUIONIZATION) / NU_over_EV), xf, 0.0f) * cm.f_He *
             local_x_e * HeII_ion_crosssec(nu);
        return s * pw(nu);
      };
    }
    double result, error;
    const int status = qag61(f, lo, hi, 0, 0.01, 1000, &result, &error);
    if (status != 0) return 0.0;
    if (FLAG == 2) return result * SPEED_OF_LIGHT / (4 * M_PI) / NU_LA / cm.hubble((float)zp);
    return result;
  };

  double filling_factor_of_HI_zp = 1. - p->ReionEfficiency * collapse_fraction / (1.0 - x_e_ave);
  // shells are independent: spread them over the host cores
  std::vector<double> ntone(nS, 0);
  auto shell_work = [&](int R_ct) {
    const double prev_zpp = R_ct == 0 ? zp : sh.zpp_edge[R_ct - 1];
    const double zpp = (sh.zpp_edge[R_ct] + prev_zpp) * 0.5;
    const double nu_tau_one_zpp = nu_tau_one(zp, zpp, x_e_ave);
    (void)filling_factor_of_HI_zp;
    ntone[R_ct] = nu_tau_one_zpp;
    const double lower = std::fmax(nu_tau_one_zpp, thresh * NU_over_EV);
    const double upper = p->NuXrayMax * NU_over_EV;
    const double alpha = p->SpecIndexXrayGal;
    for (int x_e_ct = 0; x_e_ct < x_int_NXHII; x_e_ct++) {
      const double xe = t.x_int_XHII[x_e_ct];
      out->heat[(size_t)x_e_ct * nS + R_ct] = integrate_over_nu(xe, lower, upper, 0, alpha);
      out->ion[(size_t)x_e_ct * nS + R_ct] = integrate_over_nu(xe, lower, upper, 1, alpha);
      out->lya[(size_t)x_e_ct * nS + R_ct] = integrate_over_nu(xe, lower, upper, 2, alpha);
    }
    // AGN bands: limits redshifted from zpp to zp (ComputeTs.c:834-897)
    const double zf = (1. + zp) / (1. + zpp);
    for (int b = 0; b < 2; ++b) {
      if (out->agn[b][0].empty()) continue;
      const double lo_b = std::fmax(nu_tau_one_zpp, (b ? p->NuXraySoftCut : thresh) * NU_over_EV * zf);
      const double hi_b = (b ? p->NuXrayMax : p->NuXraySoftCut) * NU_over_EV * zf;
      const double a_b = b ? p->SpecIndexXrayAGNHard : p->SpecIndexXrayAGNSoft;
      for (int x_e_ct = 0; x_e_ct < x_int_NXHII; x_e_ct++) {
        const double xe = t.x_int_XHII[x_e_ct];
        for (int kind = 0; kind < 3; ++kind)
          out->agn[b][kind][(size_t)x_e_ct * nS + R_ct] = integrate_over_nu(xe, lo_b, hi_b, kind, a_b);
      }
    }
  };
  const int agn_flag = p->Flag_IncludeAGNXray;
  for (int b = 0; b < 2; ++b) {
    const bool on = b == 0 ? (agn_flag == 1 || agn_flag == 3) : (agn_flag == 1 || agn_flag == 2);
    for (int kind = 0; kind < 3; ++kind) {
      if (on)
        out->agn[b][kind].assign((size_t)x_int_NXHII * nS, 0);
      else
        out->agn[b][kind].clear();
    }
  }
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nth = (int)std::min<unsigned>(hw, (unsigned)nS);
  std::vector<std::thread> pool;
  for (int w = 0; w < nth; ++w)
    pool.emplace_back([&, w]() {
      for (int r = w; r < nS; r += nth) shell_work(r);
    });
  for (auto& th : pool) th.join();
  out->nu_tau_one_min = *std::min_element(ntone.begin(), ntone.end());
  out->nu_tau_one_max = *std::max_element(ntone.begin(), ntone.end());

  // Lyman-n sums with the kink correction (ComputeTs.c:900-1011), in shell order
  bool first_radii = true, first_zero = true;
  // the C reuses the history weight variable: without a crossing in the trial loop the
  // correction multiplies by the weight the history loop left behind
  double weight = sh.final_weight;
  const int n_pts_radii = 1000;
  for (int R_ct = 0; R_ct < nS; R_ct++) {
    const double prev_zpp = R_ct == 0 ? zp : sh.zpp_edge[R_ct - 1];
    const double prev_R = R_ct == 0 ? 0 : sh.R[R_ct - 1];
    const double zpp = (sh.zpp_edge[R_ct] + prev_zpp) * 0.5;
    out->sum_lyn[R_ct] = 0;
    for (int n_ct = NSPEC_MAX; n_ct >= 2; n_ct--) {
      if (zpp > zmax((float)zp, n_ct)) continue;
      const double nuprime = nu_n(n_ct) * (1 + zpp) / (1.0 + zp);
      out->sum_lyn[R_ct] += frecycle(n_ct) * spectral_emissivity(t, nuprime);
    }
    if (R_ct > 2 && out->sum_lyn[R_ct] == 0.0 && out->sum_lyn[R_ct - 1] > 0. && first_radii) {
      const double trial_zpp_max = (prev_zpp - (sh.R[R_ct] - prev_R) * MPC / cm.drdz((float)prev_zpp) + prev_zpp) * 0.5;
      const double trial_zpp_min =
          (sh.zpp_edge[R_ct - 2] - (sh.R[R_ct - 1] - sh.R[R_ct - 2]) * MPC / cm.drdz((float)sh.zpp_edge[R_ct - 2]) +
           sh.zpp_edge[R_ct - 2]) *
          0.5;
      for (int ii = 0; ii < n_pts_radii; ii++) {
        const double trial_zpp =
            trial_zpp_min + (trial_zpp_max - trial_zpp_min) * (float)ii / ((float)n_pts_radii - 1.);
        int counter = 0;
        for (int n_ct = NSPEC_MAX; n_ct >= 2; n_ct--) {
          if (trial_zpp > zmax((float)zp, n_ct)) continue;
          counter += 1;
        }
        if (counter == 0 && first_zero) {
          first_zero = false;
          weight = (float)ii / (float)n_pts_radii;
        }
      }
      out->sum_lyn[R_ct] = weight * out->sum_lyn[R_ct - 1];
      first_radii = false;
    }
  }
  (void)msg;
  return RG_OK;
}

TsPrefactors ts_prefactors(const rg_params* p, double zp) {
  const Cosmo cm(p);
  TsPrefactors f;
  f.growth_factor_zp = cm.dicke(zp);
  f.dgrowth_factor_dzp = cm.ddicke_dz(zp);
  f.dt_dzp = cm.dtdz((float)zp);
  double L;
  if (std::fabs(p->SpecIndexXrayGal - 1.0) < (double)REL_TOL) {
    L = (p->NuXrayThreshold * NU_over_EV) * std::log(p->NuXraySoftCut / p->NuXrayThreshold);
    L = 1. / L;
  } else {
    L = std::pow(p->NuXraySoftCut * NU_over_EV, 1. - p->SpecIndexXrayGal) -
        std::pow(p->NuXrayThreshold * NU_over_EV, 1. - p->SpecIndexXrayGal);
    L = 1. / L;
    L *= std::pow(p->NuXrayThreshold * NU_over_EV, -p->SpecIndexXrayGal) * (1 - p->SpecIndexXrayGal);
  }
  L *= 1.0 / PLANCK;
  f.Luminosity_conversion_factor_GAL = L;
  f.const_zp_prefactor_GAL =
      L / (p->NuXrayThreshold * NU_over_EV) * SPEED_OF_LIGHT * std::pow(1 + zp, p->SpecIndexXrayGal + 3);
  // AGN bands: soft NuXrayThreshold..NuXraySoftCut, hard NuXraySoftCut..NuXrayMax, the spectrum
  // normalised at NuXrayThreshold (ComputeTs.c:1049-1081,1116-1131)
  for (int b = 0; b < 2; ++b) {
    const double a = b ? p->SpecIndexXrayAGNHard : p->SpecIndexXrayAGNSoft;
    const double nlo = b ? p->NuXraySoftCut : p->NuXrayThreshold, nhi = b ? p->NuXrayMax : p->NuXraySoftCut;
    double La;
    if (std::fabs(a - 1.0) < (double)REL_TOL) {
      La = (p->NuXrayThreshold * NU_over_EV) * std::log(nhi / nlo);
      La = 1.0 / La;
    } else {
      La = std::pow(nhi * NU_over_EV, 1.0 - a) - std::pow(nlo * NU_over_EV, 1.0 - a);
      La = 1.0 / La;
      La *= std::pow(p->NuXrayThreshold * NU_over_EV, -a) * (1.0 - a);
    }
    La /= PLANCK;
    f.const_zp_prefactor_AGN[b] =
        La / (p->NuXrayThreshold * NU_over_EV) * SPEED_OF_LIGHT * std::pow(1.0 + zp, a + 3.0);
  }
  return f;
}

}  // namespace rg
