// Table readers and the natural cubic spline of the host coefficient engine.
#include "rg_tables.h"

#include <cmath>
#include <cstdio>
#include <cstring>

#include "rg_internal.h"

namespace rg {

bool CubicSpline::init(const std::vector<double>& x, const std::vector<double>& y) {
  const size_t n = x.size();
  if (n < 3 || y.size() != n) return false;
  x_ = x;
  y_ = y;
  c_.assign(n, 0.0);
  // Natural spline: c_0 = c_{n-1} = 0; for 1 <= i <= n-2
  //   h_{i-1} c_{i-1} + 2 (h_{i-1} + h_i) c_i + h_i c_{i+1} = 3 (s_i - s_{i-1}),
  // s_i the slope of interval i.  Solved by the Thomas algorithm (the system is
  // symmetric and diagonally dominant).
  const size_t m = n - 2;
  std::vector<double> diag(m), off(m), rhs(m);
  for (size_t i = 0; i < m; ++i) {
    const double h0 = x[i + 1] - x[i], h1 = x[i + 2] - x[i + 1];
    if (!(h0 > 0.0) || !(h1 > 0.0)) return false;
    diag[i] = 2.0 * (h0 + h1);
    off[i] = h1;
    rhs[i] = 3.0 * ((y[i + 2] - y[i + 1]) / h1 - (y[i + 1] - y[i]) / h0);
  }
  for (size_t i = 1; i < m; ++i) {
    const double w = off[i - 1] / diag[i - 1];
    diag[i] -= w * off[i - 1];
    rhs[i] -= w * rhs[i - 1];
  }
  std::vector<double> sol(m);
  sol[m - 1] = rhs[m - 1] / diag[m - 1];
  for (size_t i = m - 1; i-- > 0;) sol[i] = (rhs[i] - off[i] * sol[i + 1]) / diag[i];
  for (size_t i = 0; i < m; ++i) c_[i + 1] = sol[i];
  return true;
}

size_t CubicSpline::locate(double x) const {
  // index i with x_i <= x < x_{i+1}; the last interval is closed
  size_t lo = 0, hi = x_.size() - 1;
  while (hi > lo + 1) {
    const size_t mid = (lo + hi) / 2;
    if (x_[mid] > x)
      hi = mid;
    else
      lo = mid;
  }
  return lo;
}

void CubicSpline::coeffs(size_t i, double* a, double* b, double* c, double* d) const {
  const double h = x_[i + 1] - x_[i];
  const double dy = y_[i + 1] - y_[i];
  *a = y_[i];
  *b = dy / h - h * (c_[i + 1] + 2.0 * c_[i]) / 3.0;
  *c = c_[i];
  *d = (c_[i + 1] - c_[i]) / (3.0 * h);
}

double CubicSpline::eval(double x) const {
  const size_t i = locate(x);
  double a, b, c, d;
  coeffs(i, &a, &b, &c, &d);
  const double dx = x - x_[i];
  return a + dx * (b + dx * (c + dx * d));
}

static std::string join(const std::string& d, const char* f) { return d + "/" + f; }

std::string load_tables(const std::string& dir, double pop2_ion, Tables* t) {
  *t = Tables();
  t->dir = dir;
  // recfast_LCDM.dat: 501 rows "z xion trash TK", stored from high z to low z
  {
    FILE* f = std::fopen(join(dir, "recfast_LCDM.dat").c_str(), "r");
    if (!f) return "cannot open " + join(dir, "recfast_LCDM.dat");
    t->rec_z.assign(RECFAST_NPTS, 0.0);
    t->rec_xion.assign(RECFAST_NPTS, 0.0);
    t->rec_tk.assign(RECFAST_NPTS, 0.0);
    for (int i = RECFAST_NPTS - 1; i >= 0; --i) {
      float z, xion, trash, tk;
      if (std::fscanf(f, "%f %E %E %E", &z, &xion, &trash, &tk) != 4) {
        std::fclose(f);
        return "short read in recfast_LCDM.dat";
      }
      t->rec_z[i] = z;
      t->rec_xion[i] = xion;
      t->rec_tk[i] = tk;
    }
    std::fclose(f);
    if (!t->T_spline.init(t->rec_z, t->rec_tk) || !t->x_spline.init(t->rec_z, t->rec_xion))
      return "recfast spline setup failed";
  }
  // kappa_10 (Zygelman 2005, Table 2 column 4), XRayHeatingFunctions.c:1737-1797
  {
    static const double tk[KAPPA_10_NPTS] = {1.0,   2.0,   4.0,   6.0,   8.0,    10.0,   15.0,   20.0,   25.0,
                                             30.0,  40.0,  50.0,  60.0,  70.0,   80.0,   90.0,   100.0,  200.0,
                                             300.0, 501.0, 701.0, 1000.0, 2000.0, 3000.0, 5000.0, 7000.0, 10000.0};
    static const double kap[KAPPA_10_NPTS] = {1.38e-13, 1.43e-13, 2.71e-13, 6.60e-13, 1.47e-12, 2.88e-12, 9.10e-12,
                                              1.78e-11, 2.73e-11, 3.67e-11, 5.38e-11, 6.86e-11, 8.14e-11, 9.25e-11,
                                              1.02e-10, 1.11e-10, 1.19e-10, 1.75e-10, 2.09e-10, 2.565e-10, 2.91e-10,
                                              3.31e-10, 4.27e-10, 4.97e-10, 6.03e-10, 6.87e-10, 7.87e-10};
    for (int i = 0; i < KAPPA_10_NPTS; ++i) {
      t->k10_lT.push_back(std::log(tk[i]));
      t->k10_lk.push_back(std::log(kap[i]));
    }
    if (!t->k10.init(t->k10_lT, t->k10_lk)) return "kappa_10 spline setup failed";
  }
  auto read_kappa = [&](const char* name, int npts, std::vector<double>* lT, std::vector<double>* lk,
                        CubicSpline* sp) -> std::string {
    FILE* f = std::fopen(join(dir, name).c_str(), "r");
    if (!f) return std::string("cannot open ") + join(dir, name);
    for (int i = 0; i < npts; ++i) {
      float a, b;
      if (std::fscanf(f, "%f %e", &a, &b) != 2) {
        std::fclose(f);
        return std::string("short read in ") + name;
      }
      lT->push_back(std::log((double)a));
      lk->push_back(std::log((double)b));
    }
    std::fclose(f);
    if (!sp->init(*lT, *lk)) return std::string("spline setup failed for ") + name;
    return "";
  };
  std::string e = read_kappa("kappa_eH_table.dat", KAPPA_10_elec_NPTS, &t->kel_lT, &t->kel_lk, &t->kel);
  if (!e.empty()) return e;
  e = read_kappa("kappa_pH_table.dat", KAPPA_10_pH_NPTS, &t->kpH_lT, &t->kpH_lk, &t->kpH);
  if (!e.empty()) return e;
  // stellar_spectra.dat, spectral_emissivity(flag=1), XRayHeatingFunctions.c:670-707
  {
    FILE* f = std::fopen(join(dir, "stellar_spectra.dat").c_str(), "r");
    if (!f) return "cannot open " + join(dir, "stellar_spectra.dat");
    t->spec_n.assign(NSPEC_MAX, 0);
    t->spec_nu.assign(NSPEC_MAX, 0.f);
    t->spec_alpha2.assign(NSPEC_MAX, 0.f);
    t->spec_N0_2.assign(NSPEC_MAX, 0.f);
    for (int i = 1; i < NSPEC_MAX; ++i) {
      float n02, a2, n03, a3;
      if (std::fscanf(f, "%i %e %e %e %e", &t->spec_n[i], &n02, &a2, &n03, &a3) != 5) {
        std::fclose(f);
        return "short read in stellar_spectra.dat";
      }
      t->spec_N0_2[i] = n02;
      t->spec_alpha2[i] = a2;
    }
    std::fclose(f);
    for (int i = 1; i < NSPEC_MAX; ++i)
      t->spec_nu[i] = (float)(4.0 / 3.0 * (1.0 - 1.0 / std::pow((double)t->spec_n[i], 2.0)));
    for (int i = 1; i < NSPEC_MAX - 1; ++i) {
      const double n0_fac = std::pow((double)t->spec_nu[i + 1], (double)t->spec_alpha2[i] + 1) -
                            std::pow((double)t->spec_nu[i], (double)t->spec_alpha2[i] + 1);
      t->spec_N0_2[i] = (float)((double)t->spec_N0_2[i] * (((double)t->spec_alpha2[i] + 1) / n0_fac * pop2_ion));
    }
  }
  // x_int_tables (initialize_interp_arrays, XRayHeatingFunctions.c:861-960)
  {
    static const float xhii[x_int_NXHII] = {1.0e-4f, 2.318e-4f, 4.677e-4f, 1.0e-3f, 2.318e-3f, 4.677e-3f, 1.0e-2f,
                                            2.318e-2f, 4.677e-2f, 1.0e-1f, 0.5f, 0.9f, 0.99f, 0.999f};
    t->x_int_XHII.assign(xhii, xhii + x_int_NXHII);
    const size_t sz = (size_t)x_int_NXHII * x_int_NENERGY;
    t->x_int_Energy.assign(x_int_NENERGY, 0.f);
    t->fheat.assign(sz, 0.f);
    t->n_Lya.assign(sz, 0.f);
    t->nion_HI.assign(sz, 0.f);
    t->nion_HeI.assign(sz, 0.f);
    t->nion_HeII.assign(sz, 0.f);
    for (int ion = 0; ion < x_int_NXHII; ++ion) {
      char name[128];
      if (xhii[ion] < 0.3)
        std::snprintf(name, sizeof(name), "x_int_tables/log_xi_%1.1f.dat", std::log10((double)xhii[ion]));
      else
        std::snprintf(name, sizeof(name), "x_int_tables/xi_%1.3f.dat", (double)xhii[ion]);
      FILE* f = std::fopen(join(dir, name).c_str(), "r");
      if (!f) return std::string("cannot open ") + join(dir, name);
      char label[64];
      for (int i = 0; i < 5; ++i)
        if (std::fscanf(f, "%63s", label) != 1) { std::fclose(f); return std::string("bad header in ") + name; }
      float a, b, c, d, e2;
      if (std::fscanf(f, "%g %g %g %g %g", &a, &b, &c, &d, &e2) != 5) { std::fclose(f); return "bad header"; }
      for (int i = 0; i < 11; ++i)
        if (std::fscanf(f, "%63s", label) != 1) { std::fclose(f); return std::string("bad header in ") + name; }
      for (int i = 0; i < x_int_NENERGY; ++i) {
        float en, tr1, fh, tr2, nl, nh, nhe, nhe2, tr3;
        if (std::fscanf(f, "%g %g %g %g %g %g %g %g %g", &en, &tr1, &fh, &tr2, &nl, &nh, &nhe, &nhe2, &tr3) != 9) {
          std::fclose(f);
          return std::string("short read in ") + name;
        }
        t->x_int_Energy[i] = en;
        const size_t k = (size_t)ion * x_int_NENERGY + i;
        t->fheat[k] = fh;
        t->n_Lya[k] = nl;
        t->nion_HI[k] = nh;
        t->nion_HeI[k] = nhe;
        t->nion_HeII[k] = nhe2;
      }
      std::fclose(f);
    }
  }
  t->loaded = true;
  return "";
}

double T_RECFAST(const Tables& t, float z) {
  if ((double)z > t.rec_z.back()) return -1.0;
  return t.T_spline.eval((double)z);
}

double xion_RECFAST(const Tables& t, float z) {
  if ((double)z > t.rec_z.back()) return -1.0;
  return t.x_spline.eval((double)z);
}

}  // namespace rg
