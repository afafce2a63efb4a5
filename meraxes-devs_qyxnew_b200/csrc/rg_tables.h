// Host-side FP64 coefficient engine: the 21cmFAST data tables, natural cubic splines,
// adaptive Gauss-Kronrod quadrature and Brent root finding that the reference takes
// from GSL (src/core/XRayHeatingFunctions.c), written from the published methods.
#pragma once

#include <string>
#include <vector>

namespace rg {

// Natural cubic spline (the interpolant gsl_interp_cspline builds): second
// derivatives from the tridiagonal system with zero end curvature.
class CubicSpline {
 public:
  CubicSpline() = default;
  bool init(const std::vector<double>& x, const std::vector<double>& y);
  double eval(double x) const;        // caller keeps x inside [x0, x_{n-1}]
  size_t size() const { return x_.size(); }
  const std::vector<double>& xs() const { return x_; }
  const std::vector<double>& half_curvature() const { return c_; }   // c_i = y''_i / 2
  // per interval i: y = a + dx (b + dx (c + dx d)), dx = x - x_i
  void coeffs(size_t i, double* a, double* b, double* c, double* d) const;

 private:
  size_t locate(double x) const;
  std::vector<double> x_, y_, c_;     // c_ = half the second derivative
};

struct Tables {
  bool loaded = false;
  std::string dir;
  // recfast_LCDM.dat, ascending z
  std::vector<double> rec_z, rec_xion, rec_tk;
  CubicSpline T_spline, x_spline;
  // kappa tables in log-log (XRayHeatingFunctions.c:1728-1966)
  std::vector<double> k10_lT, k10_lk, kel_lT, kel_lk, kpH_lT, kpH_lk;
  CubicSpline k10, kel, kpH;
  // stellar spectra (spectral_emissivity), indices 1..NSPEC_MAX-1
  std::vector<int> spec_n;
  std::vector<float> spec_nu, spec_alpha2, spec_N0_2;
  // electron interpolation tables [14][258] (initialize_interp_arrays)
  std::vector<float> x_int_XHII, x_int_Energy, fheat, n_Lya, nion_HI, nion_HeI, nion_HeII;
};

// Load every table from dir; returns an empty string or an error message.
std::string load_tables(const std::string& dir, double ReionNionPhotPerBary, Tables* t);

double T_RECFAST(const Tables& t, float z);      // -1 when z is beyond the table
double xion_RECFAST(const Tables& t, float z);

}  // namespace rg
