// Host FP64 coefficient engine of the spin-temperature step (ComputeTs), restating the
// scalar parts of src/core/ComputeTs.c and src/core/XRayHeatingFunctions.c: the shell
// schedule, the SFR-history weights, the frequency-integral tables, the Lyman-n sums and
// the per-snapshot prefactors.  GSL's QAG (Gauss-Kronrod 61) and Brent solver are written
// here from the published QUADPACK and Brent algorithms.
#pragma once

#include <functional>
#include <string>
#include <vector>

#include "../../include/rg_b200.h"
#include "rg_tables.h"

namespace rg {

// QAG: adaptive bisection with the 61-point Gauss-Kronrod rule; returns 0 on success,
// nonzero when the tolerance was not met (like a GSL error status).
int qag61(const std::function<double(double)>& f, double a, double b, double epsabs, double epsrel, int limit,
          double* result, double* abserr);
// Brent's method on [lo, hi]; iterates until |hi - lo| < epsabs + epsrel min(|lo|,|hi|) or
// max_iter; returns the last estimate.
double brent_root(const std::function<double(double)>& f, double lo, double hi, double epsabs, double epsrel,
                  int max_iter, int* status);

// cosmology and atomic physics of the reference
struct Cosmo {
  const rg_params* p;
  double No, He_No, N_b0, f_H, f_He;
  explicit Cosmo(const rg_params* prm);
  double dtdz(float z) const;
  double drdz(float z) const;
  double hubble(float z) const;
  double dicke(double z) const;
  double ddicke_dz(double z) const;
};

double HI_ion_crosssec(double nu);
double HeI_ion_crosssec(double nu);
double HeII_ion_crosssec(double nu);
float interp_x_int(const Tables& t, const std::vector<float>& tab, float En, float xHII_call, float below);
int locate_xHII_index(const Tables& t, float xHII_call);
float zmax(float z, int n);
double nu_n(int n);
double frecycle(int n);
double spectral_emissivity(const Tables& t, double nu_norm);  // flag 0, Pop II

// One snapshot's inhomogeneous shell set-up (ComputeTs.c:339-478 and :760-1132)
struct TsShells {
  int nS = 0;
  std::vector<double> R, zpp_edge, zpp, dzpp, dt_dzpp, sum_lyn;
  // linear combination of source grids per shell: coefficient of source k for shell r is
  // coef[r * nsrc + k]; source 0 = this snapshot's sfr/xray grids, source 1 + h = history slot h
  int nsrc = 0;
  std::vector<float> coef;
  // value of the history weight after the last shell; the Lyman-n kink correction starts from it
  double final_weight = 1;
  bool error = false;
  std::string msg;
};

// Shell radii, zpp edges and the SFR-history combination (ComputeTs.c:339-478).
TsShells ts_shells(const rg_params* p, const double* ZZ, int n_snap, int snapshot, int n_hist);

// Frequency-integral tables [kind][x_e node][shell] for kind = heat, ion, lya
// (ComputeTs.c:761-808) and the Lyman-n sums with the kink correction (:900-1011).
struct TsTables {
  std::vector<double> heat, ion, lya;   // [14][nS]
  // AGN X-ray bands (Flag_IncludeAGNXray), [band 0 soft, 1 hard][kind heat, ion, lya][14][nS]
  // (ComputeTs.c:834-897); empty for a band that is off
  std::vector<double> agn[2][3];
  std::vector<double> sum_lyn;          // [nS]
  double nu_tau_one_min = 0, nu_tau_one_max = 0;
};
int ts_tables(const rg_params* p, const Tables& t, const TsShells& sh, double zp, double x_e_ave,
              double collapse_fraction, const double* ZZ, const double* stored_fcoll, int snapshot, TsTables* out,
              std::string* msg);

// Per-snapshot prefactors (ComputeTs.c:1014-1109)
struct TsPrefactors {
  double growth_factor_zp, dgrowth_factor_dzp, dt_dzp, const_zp_prefactor_GAL, Luminosity_conversion_factor_GAL;
  double const_zp_prefactor_AGN[2];   // soft, hard (ComputeTs.c:1049-1081,1116-1131)
};
TsPrefactors ts_prefactors(const rg_params* p, double zp);

}  // namespace rg
