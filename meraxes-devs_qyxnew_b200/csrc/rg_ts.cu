// Spin-temperature step (_ComputeTs, src/core/ComputeTs.c:85-1554) on sm_100a, without the
// AGN and mini-halo channels.
//
// Inhomogeneous branch, per snapshot:
//   1. FP64 reductions of the collapse fraction and <x_e> (ComputeTs.c:585-677)
//   2. host: frequency-integral tables, Lyman-n sums, prefactors (rg_xray.cpp)
//   3. forward r2c of every source grid (this snapshot's sfr / xray_luminosity and the
//      history slots the shells use); each shell's source is a linear combination of them
//      (the history re-weighting of :366-478), formed in k-space on load
//   4. shells in batches: x pass (combination, TsHeatingFilterType window), y pass, z pass
//      that turns both grids of every shell of the batch into the four per-cell sums of
//      evolveInt (X-ray heating, ionisation and Lyman-alpha integrands, stellar Lyman-alpha)
//      without storing the reference's SMOOTHED_*[nS N^3] arrays
//   5. per cell, FP64: evolveInt, the Euler step of x_e and T_K, get_Ts, and the FP64 sums
// Homogeneous branch (zp >= ReionMaxHeatingRedshift): RECFAST x_e and T_K, get_Ts with no
// Lyman-alpha coupling (:252-331).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "rg_internal.h"
#include "rg_pass.cuh"
#include "rg_xray.h"

namespace rg {

constexpr int TS_KB = 8;        // shells per batch
constexpr int TS_MAXSRC = 4;    // sources combined into one shell
constexpr int TS_NSUM = 8;      // evolve sums
constexpr int KSPL = 27;        // knots of the largest kappa table

struct KappaSpline {
  int n;
  double x[KSPL], y[KSPL], b[KSPL], c[KSPL], d[KSPL];
};

struct TsDev {
  KappaSpline k10, kel, kpH;
  double No, N_b0, f_H, f_He, h, OMm, OMr, OMl;
};

__device__ __forceinline__ double spline_eval(const KappaSpline& s, double x) {
  int lo = 0, hi = s.n - 1;
  while (hi > lo + 1) {
    const int mid = (lo + hi) >> 1;
    if (s.x[mid] > x)
      hi = mid;
    else
      lo = mid;
  }
  const double dx = x - s.x[lo];
  return s.y[lo] + dx * (s.b[lo] + dx * (s.c[lo] + dx * s.d[lo]));
}

// kappa_10 (XRayHeatingFunctions.c:1728-1822)
__device__ double kappa_10(const TsDev& C, double TK) {
  const KappaSpline& s = C.k10;
  double ans;
  if (log(TK) < s.x[0]) {
    ans = s.y[0];
  } else if (log(TK) > s.x[s.n - 1]) {
    ans = log(exp(s.y[s.n - 1]) * pow(TK / exp(s.x[s.n - 1]), 0.381));
  } else {
    ans = spline_eval(s, log(TK));
  }
  return exp(ans);
}

// kappa_10_elec and kappa_10_pH (XRayHeatingFunctions.c:1827-1966)
__device__ double kappa_table(const KappaSpline& s, double T) {
  T = log(T);
  double ans;
  if (T < s.x[0]) {
    ans = s.y[0];
  } else if (T > s.x[s.n - 1]) {
    ans = s.y[s.n - 1] + ((s.y[s.n - 1] - s.y[s.n - 2]) / (s.x[s.n - 1] - s.x[s.n - 2]) * (T - s.x[s.n - 1]));
  } else {
    ans = spline_eval(s, T);
  }
  return exp(ans);
}

__device__ __forceinline__ double d_hubble(const TsDev& C, float z) {
  const double opz = (double)(1.0f + z);
  return HUBBLE * C.h * sqrt(C.OMm * pow(opz, 3) + C.OMr * pow(opz, 4) + C.OMl);
}

// xcoll (XRayHeatingFunctions.c:1686-1726)
__device__ double xcoll(const TsDev& C, double z, double TK, double delta, double xe) {
  const double Trad = TCMB * (1.0 + z);
  const double opz3 = pow(1.0 + z, 3.0);
  const double nH = (1.0 - xe) * C.No * opz3 * (1.0 + delta);
  const double ne = xe * C.N_b0 * opz3 * (1.0 + delta);
  const double np = xe * C.No * opz3 * (1.0 + delta);
  return T21 / Trad * nH * kappa_10(C, TK) / A10_HYPERFINE + T21 / Trad * ne * kappa_table(C.kel, TK) / A10_HYPERFINE +
         T21 / Trad * np * kappa_table(C.kpH, TK) / A10_HYPERFINE;
}

// get_Ts and the Wouthuysen-Field coupling (XRayHeatingFunctions.c:1639-1684, 1973-2008); the
// fixed-point loop is capped at 10000 iterations (a cell that hits the cap counts in *nonconv)
__device__ float get_Ts(const TsDev& C, float z, float delta, float TK, float xe, float Jalpha, float* curr_xalpha,
                        int* nonconv) {
  const double Trad = TCMB * (1.0 + (double)z);
  const double xc = xcoll(C, (double)z, (double)TK, (double)delta, (double)xe);
  double TS, TSinv;
  if ((double)Jalpha > 1.0e-20) {
    TS = Trad;
    double TSold = 0.0, xa_tilde = 0.0;
    const double zz = (double)z;
    const double tgp = 1.342881e-7 / d_hubble(C, (float)zz) * C.No * pow(1 + zz, 3) * (1.0 + (double)delta) *
                       (1.0 - (double)xe);
    const double tk = (double)TK;
    int it = 0;
    while (fabs(TS - TSold) / TS > 1.0e-3) {
      if (++it > 10000) {
        *nonconv += 1;
        break;
      }
      TSold = TS;
      // Salpha_tilde and xalpha_tilde
      const double xi = pow(1.0e-7 * tgp / tk / tk, 1.0 / 3.0);
      double st = 1.0 - 0.0631789 / tk + 0.115995 / tk / tk - 0.401403 / TS / tk;
      st += 0.336463 / TS / tk / tk;
      st /= 1.0 + 2.98394 * xi + 1.53583 * xi * xi + 3.85289 * xi * xi * xi;
      xa_tilde = 1.66e11 / (1.0 + zz) * st * (double)Jalpha;
      // Tc_eff
      double tce = 1.0 / tk + 0.405535 / tk * (1.0 / TS - 1.0 / tk);
      tce = 1.0 / tce;
      TSinv = (1.0 / Trad + xa_tilde / tce + xc / tk) / (1.0 + xa_tilde + xc);
      TS = 1.0 / TSinv;
    }
    *curr_xalpha = (float)xa_tilde;
  } else {
    TSinv = (1.0 / Trad + xc / (double)TK) / (1.0 + xc);
    TS = 1.0 / TSinv;
    *curr_xalpha = 0;
  }
  if (TS < 0.) TS = fabs(TS);
  return (float)TS;
}

// alpha_A (XRayHeatingFunctions.c:1576-1584)
__device__ double alpha_A(double T) {
  const double logT = log(T / (double)1.1604505e4);
  return exp(-28.6130338 - 0.72411256 * logT - 2.02604473e-2 * pow(logT, 2) - 2.38086188e-3 * pow(logT, 3) -
             3.21260521e-4 * pow(logT, 4) - 1.42150291e-5 * pow(logT, 5) + 4.98910892e-6 * pow(logT, 6) +
             5.75561414e-7 * pow(logT, 7) - 1.85676704e-8 * pow(logT, 8) - 3.07113524e-9 * pow(logT, 9));
}

// dT_comp (XRayHeatingFunctions.c:1564-1573)
__device__ double dT_comp(const TsDev& C, double z, double TK, double xe) {
  const double Trad = TCMB * (1.0 + z);
  double ans = (-1.51e-4) * (xe / (1.0 + xe + C.f_He)) / (d_hubble(C, (float)z) / (HUBBLE * C.h)) / C.h *
               pow(Trad, 4.0) / (1.0 + z);
  ans *= Trad - TK;
  return ans;
}

// ---------------------------------------------------------------------------
// block sums (deterministic) -> partials[block][K]

template <int K>
__device__ __forceinline__ void block_sum_dyn(double (&acc)[K], double* out) {
  __shared__ double s_red[32][K];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < K; ++i) {
    double v = acc[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) s_red[wid][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += s_red[w][threadIdx.x];
    out[threadIdx.x] = v;
  }
}

// collapse fraction and <x_e> over the box (ComputeTs.c:585-677)
__global__ void __launch_bounds__(256) k_ts_reduce0(const float* __restrict__ stars, const float* __restrict__ deltax,
                                                    const float* __restrict__ xe, int n, double Mh2,
                                                    double fourthirds_pi_R3_over_pv, double* partials) {
  const int padw = 2 * (n / 2 + 1);
  const size_t rows = (size_t)n * n;
  double acc[2] = {0.0, 0.0};
  for (size_t row = blockIdx.x; row < rows; row += gridDim.x)
    for (int z = threadIdx.x; z < n; z += blockDim.x) {
      const size_t ip = row * padw + z;
      const double density_over_mean = 1.0 + (double)deltax[ip];
      double c = (double)stars[ip] / (Mh2 * density_over_mean) * fourthirds_pi_R3_over_pv;
      if (c > 1.0) c = 1.0;
      acc[0] += c;
      acc[1] += (double)xe[ip];
    }
  block_sum_dyn<2>(acc, partials + (size_t)blockIdx.x * 2);
}

// ---------------------------------------------------------------------------
// shell x pass: output (r, g) = sum_i cs[r][i] spec[ks[r][i]][g] x window_r, transformed along x

struct TsBatch {
  int nr;
  int nk[TS_KB];
  int ks[TS_KB][TS_MAXSRC];
  float cs[TS_KB][TS_MAXSRC];
  int filtered[TS_KB];
  int wrow[TS_KB];
};

template <int N>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::BX, RG_MINB(Cfg<N>::T* Cfg<N>::BX))
    k_ts_x(const cf* __restrict__ spec, size_t stride, cf* __restrict__ work, TsBatch bt,
           const float* __restrict__ wtab, int wpitch, const cf* __restrict__ g_tw) {
  constexpr int T = Cfg<N>::T, B = Cfg<N>::BX, V = Cfg<N>::V;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  const int kz = blockIdx.y;
  const int b = threadIdx.x % B, t = threadIdx.x / B;
  const int y = blockIdx.x * B + b;
  const size_t col = (size_t)kz * N * N + y;
  load_twiddles<N>(s_tw, g_tw);
  int n2[V];
  const int ny = y > N / 2 ? y - N : y;
#pragma unroll
  for (int sl = 0; sl < V; ++sl) {
    const int p = stage0_pos<N>(t, sl);
    const int nx = p > N / 2 ? p - N : p;
    n2[sl] = nx * nx + ny * ny + kz * kz;
  }
  __syncthreads();
  for (int r = 0; r < bt.nr; ++r) {
    float wv[V];
    if (!bt.filtered[r]) {
#pragma unroll
      for (int sl = 0; sl < V; ++sl) wv[sl] = 1.f;
    } else {
      const float* wr = wtab + (size_t)bt.wrow[r] * wpitch;
#pragma unroll
      for (int sl = 0; sl < V; ++sl) wv[sl] = __ldg(wr + n2[sl]);
    }
    const int nk = bt.nk[r];
    for (int g = 0; g < 2; ++g) {
      cf* dst = work + ((size_t)r * 2 + g) * stride;
      line_fft<N, true>(
          t, xbuf, s_tw,
          [&](int p, int sl) {
            float ax = 0.f, ay = 0.f;
            for (int i = 0; i < nk; ++i) {
              const cf v = spec[((size_t)bt.ks[r][i] * 2 + g) * stride + col + (size_t)p * N];
              ax = fmaf(bt.cs[r][i], v.x, ax);
              ay = fmaf(bt.cs[r][i], v.y, ay);
            }
            return cf{ax * wv[sl], ay * wv[sl]};
          },
          [&](int p) { return line_addr<N, B>(p, b); }, [&](int p, cf v) { dst[col + (size_t)p * N] = v; });
    }
  }
}

// ---------------------------------------------------------------------------
// shell z pass: c2r of the sfr and xray grids of every shell of the batch, accumulated per cell
// into the four evolveInt sums (FP32 within a batch, FP64 across batches)

struct TsCoef {
  // per shell of the batch: P/Q of the x_e interpolation for heat, ion, lya (scaled), and the
  // scaled stellar Lyman-alpha coefficient; fi_k = P_k[lo] + (x_e - X[lo]) Q_k[lo]
  float P[TS_KB][3][x_int_NXHII];
  float Q[TS_KB][3][x_int_NXHII];
  float cstar[TS_KB];
  float X[x_int_NXHII];           // x_int_XHII (float, as in the reference)
  double inv_scale[4];            // undo the FP32 scaling when flushing to FP64
  int nr;
  int first;                      // first batch: the FP64 sums start at zero
};

template <int N>
struct TsZ {
  using PL = Plan8<N>;
  static constexpr int T = PL::T;
  static constexpr int Q = pow2_div(N / 2, cmax(256 / T, 1));
  static constexpr int NTH = T * Q;
  static constexpr int V = N / T;            // 8
  static constexpr int R0 = PL::R[0];
  static constexpr size_t smem() { return sizeof(cf) * (N + (size_t)line_buf_r0<N, R0, Q>()); }
};

template <int N>
__global__ void __launch_bounds__(TsZ<N>::NTH, RG_MINB(TsZ<N>::NTH))
    k_ts_z(const cf* __restrict__ work, size_t stride, const cf* __restrict__ g_tw, const TsCoef* __restrict__ gco,
           const float* __restrict__ xe_box, double* __restrict__ acc_g) {
  using Z = TsZ<N>;
  using PL = typename Z::PL;
  constexpr int T = Z::T, Q = Z::Q, V = Z::V;
  constexpr int PADW = 2 * (N / 2 + 1);
  constexpr size_t N3 = (size_t)N * N * N;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  __shared__ TsCoef co;
  const int x = blockIdx.y, y0 = blockIdx.x * 2 * Q;
  const int q = threadIdx.x % Q, t = threadIdx.x / Q;
  load_twiddles<N>(s_tw, g_tw);
  {
    const int* src = reinterpret_cast<const int*>(gco);
    int* dst = reinterpret_cast<int*>(&co);
    for (int i = threadIdx.x; i < (int)(sizeof(TsCoef) / sizeof(int)); i += Z::NTH) dst[i] = src[i];
  }
  __syncthreads();
  // cells of this thread: rows y0 + 2q + h, positions last_pos(t, s)
  float dxe[2 * V];
  uint64_t lopack = 0;
#pragma unroll
  for (int s = 0; s < V; ++s) {
    const int z = last_pos<PL>(t, s);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      double xc = (double)__ldg(xe_box + ((size_t)x * N + y0 + 2 * q + h) * PADW + z);
      // ComputeTs.c:1198-1208
      if (xc > (double)co.X[x_int_NXHII - 1] * 0.999)
        xc = (double)co.X[x_int_NXHII - 1] * 0.999;
      else if (xc < (double)co.X[0])
        xc = 1.001 * (double)co.X[0];
      const float xf = (float)xc;
      int m = x_int_NXHII - 1;
      while (xf < co.X[m]) m--;
      lopack |= (uint64_t)m << (4 * (2 * s + h));
      dxe[2 * s + h] = (float)(xc - (double)co.X[m]);
    }
  }
  float a_heat[2 * V], a_ion[2 * V], a_lya[2 * V], a_star[2 * V];
#pragma unroll
  for (int c = 0; c < 2 * V; ++c) a_heat[c] = a_ion[c] = a_lya[c] = a_star[c] = 0.f;
  const size_t colpair = (size_t)x * N + y0 + 2 * q;
  auto addr = [&](int p) { return line_addr_r0<Z::R0, Q>(p, q); };
  for (int r = 0; r < co.nr; ++r) {
    // sfr: stellar Lyman-alpha sum, SFR clamped at 0 (ComputeTs.c:700)
    const cf* gs = work + ((size_t)r * 2 + 0) * stride;
    const float cst = co.cstar[r];
    line_fft_p<PL, true>(
        t, xbuf, s_tw, [&](int p, int) { return build_c2r_input<N>(gs, colpair, p); }, addr,
        [&](int, cf v, int sl) {
          a_star[2 * sl] = fmaf(fmaxf(v.x, 0.f), cst, a_star[2 * sl]);
          a_star[2 * sl + 1] = fmaf(fmaxf(v.y, 0.f), cst, a_star[2 * sl + 1]);
        });
    // xray: heating, ionisation and Lyman-alpha integrands, not clamped
    const cf* gx = work + ((size_t)r * 2 + 1) * stride;
    line_fft_p<PL, true>(
        t, xbuf, s_tw, [&](int p, int) { return build_c2r_input<N>(gx, colpair, p); }, addr,
        [&](int, cf v, int sl) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int c = 2 * sl + h;
            const int lo = (int)((lopack >> (4 * c)) & 15u);
            const float d = dxe[c];
            const float xr = h ? v.y : v.x;
            a_heat[c] = fmaf(xr, fmaf(d, co.Q[r][0][lo], co.P[r][0][lo]), a_heat[c]);
            a_ion[c] = fmaf(xr, fmaf(d, co.Q[r][1][lo], co.P[r][1][lo]), a_ion[c]);
            a_lya[c] = fmaf(xr, fmaf(d, co.Q[r][2][lo], co.P[r][2][lo]), a_lya[c]);
          }
        });
  }
  // flush to the FP64 sums
#pragma unroll
  for (int s = 0; s < V; ++s) {
    const int z = last_pos<PL>(t, s);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = 2 * s + h;
      const size_t ir = ((size_t)x * N + y0 + 2 * q + h) * N + z;
      const double v0 = (double)a_heat[c] * co.inv_scale[0], v1 = (double)a_ion[c] * co.inv_scale[1];
      const double v2 = (double)a_lya[c] * co.inv_scale[2], v3 = (double)a_star[c] * co.inv_scale[3];
      if (co.first) {
        acc_g[ir] = v0;
        acc_g[N3 + ir] = v1;
        acc_g[2 * N3 + ir] = v2;
        acc_g[3 * N3 + ir] = v3;
      } else {
        acc_g[ir] += v0;
        acc_g[N3 + ir] += v1;
        acc_g[2 * N3 + ir] += v2;
        acc_g[3 * N3 + ir] += v3;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// per-cell evolution (evolveInt + the Euler step + get_Ts, ComputeTs.c:1171-1407)

struct TsEvolve {
  float zp_f;
  double zp, dzp, dt_dzp, growth, dgrowth, const_zp, conv_star;
  int no_light;
};

__global__ void __launch_bounds__(256) k_ts_evolve(const TsDev* __restrict__ gC, TsEvolve e, int n,
                                                   const double* __restrict__ acc_g, const float* __restrict__ deltax,
                                                   float* __restrict__ xe_prev, float* __restrict__ xe_box,
                                                   float* __restrict__ Tk, float* __restrict__ TS,
                                                   double* __restrict__ partials, int* __restrict__ nonconv) {
  __shared__ TsDev C;
  {
    const int* src = reinterpret_cast<const int*>(gC);
    int* dst = reinterpret_cast<int*>(&C);
    for (int i = threadIdx.x; i < (int)(sizeof(TsDev) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int padw = 2 * (n / 2 + 1);
  const size_t rows = (size_t)n * n, n3 = rows * n;
  double acc[TS_NSUM];
#pragma unroll
  for (int i = 0; i < TS_NSUM; ++i) acc[i] = 0.0;
  int nc = 0;
  for (size_t row = blockIdx.x; row < rows; row += gridDim.x)
    for (int z = threadIdx.x; z < n; z += blockDim.x) {
      const size_t ir = row * n + z, ip = row * padw + z;
      const float delta = deltax[ip];
      const float xef = xe_prev[ip];
      const double x_e = (double)xef, T = (double)Tk[ir];
      const double n_b = C.N_b0 * pow((double)(1.0f + e.zp_f), 3) * (double)(1.0f + delta);
      double dxheat_dt = 0, dxion_src = 0, dxlya = 0, dstarlya = 0;
      if (!e.no_light) {
        dxheat_dt = acc_g[ir] * e.const_zp;
        dxion_src = acc_g[n3 + ir] * e.const_zp;
        dxlya = acc_g[2 * n3 + ir] * (e.const_zp * n_b);
        dstarlya = acc_g[3 * n3 + ir] * e.conv_star;
      }
      const double dxion_sink = alpha_A(T) * CLUMPING_FACTOR * x_e * x_e * C.f_H * n_b;
      const double dxe_dzp = e.dt_dzp * (dxion_src - dxion_sink);
      double dadia = 3 / (1.0 + (double)e.zp_f);
      if (fabs((double)delta) > FRACT_FLOAT_ERR) dadia += e.dgrowth / (1.0 / (double)delta + e.growth);
      dadia *= (2.0 / 3.0) * T;
      const double dspec = -dxe_dzp * T / (1 + x_e);
      const double dcomp = dT_comp(C, (double)e.zp_f, T, x_e);
      const double dxheat_dzp = dxheat_dt * e.dt_dzp * 2.0 / 3.0 / BOLTZMANN / (1.0 + x_e);
      const double d1 = dxheat_dzp + dcomp + dspec + dadia;
      const double d2 = dxlya + dstarlya;
      const double d4 = e.dt_dzp * dxion_src;
      float xn = (float)((double)xef + dxe_dzp * e.dzp);
      if (xn > 1)
        xn = (float)(1 - FRACT_FLOAT_ERR);
      else if (xn < 0)
        xn = 0;
      float tk = Tk[ir];
      if (tk < MAX_TK) tk = (float)((double)tk + d1 * e.dzp);
      if (tk < MIN_TK) tk = (float)(TCMB * (1 + e.zp));
      float xa;
      const float ts = get_Ts(C, e.zp_f, delta, tk, xn, (float)d2, &xa, &nc);
      xe_prev[ip] = xn;
      xe_box[ip] = xn;
      Tk[ir] = tk;
      TS[ir] = ts;
      acc[0] += d2;
      acc[1] += (double)xa;
      acc[2] += dxheat_dzp;
      acc[3] += d4;
      acc[4] += (double)ts;
      acc[5] += (double)tk;
      acc[6] += (double)xn;
    }
  if (nc) atomicAdd(nonconv, nc);
  block_sum_dyn<TS_NSUM>(acc, partials + (size_t)blockIdx.x * TS_NSUM);
}

// homogeneous branch (ComputeTs.c:252-278) and the closing averages (:1459-1494)
__global__ void __launch_bounds__(256) k_ts_homog(const TsDev* __restrict__ gC, float zp_f, float xe0, float TK0,
                                                  float cT_ad, int n, const float* __restrict__ deltax,
                                                  float* __restrict__ xe_prev, float* __restrict__ xe_box,
                                                  float* __restrict__ Tk, float* __restrict__ TS,
                                                  double* __restrict__ partials, int* __restrict__ nonconv) {
  __shared__ TsDev C;
  {
    const int* src = reinterpret_cast<const int*>(gC);
    int* dst = reinterpret_cast<int*>(&C);
    for (int i = threadIdx.x; i < (int)(sizeof(TsDev) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int padw = 2 * (n / 2 + 1);
  const size_t rows = (size_t)n * n;
  double acc[TS_NSUM];
#pragma unroll
  for (int i = 0; i < TS_NSUM; ++i) acc[i] = 0.0;
  int nc = 0;
  for (size_t row = blockIdx.x; row < rows; row += gridDim.x)
    for (int z = threadIdx.x; z < n; z += blockDim.x) {
      const size_t ir = row * n + z, ip = row * padw + z;
      const float delta = deltax[ip];
      const float tk = (float)((double)TK0 * (1.0 + (double)(cT_ad * delta)));
      float xa;
      const float ts = get_Ts(C, zp_f, delta, tk, xe0, 0.f, &xa, &nc);
      xe_prev[ip] = xe0;
      xe_box[ip] = xe0;
      Tk[ir] = tk;
      TS[ir] = ts;
      acc[4] += (double)ts;
      acc[5] += (double)tk;
      acc[6] += (double)xe0;
    }
  if (nc) atomicAdd(nonconv, nc);
  block_sum_dyn<TS_NSUM>(acc, partials + (size_t)blockIdx.x * TS_NSUM);
}

// ---------------------------------------------------------------------------
// host side

// knots (log T, log kappa) and per-interval coefficients of one kappa table
static void fill_spline(const CubicSpline& sp, const std::vector<double>& lx, const std::vector<double>& ly,
                        KappaSpline* k) {
  std::memset(k, 0, sizeof(*k));
  k->n = (int)lx.size();
  for (int i = 0; i < k->n; ++i) {
    k->x[i] = lx[i];
    k->y[i] = ly[i];
    if (i + 1 < k->n) {
      double a;
      sp.coeffs((size_t)i, &a, &k->b[i], &k->c[i], &k->d[i]);
    }
  }
}

template <typename T>
static int ensure_mem(rg_context* ctx, T** ptr, size_t* have, size_t need) {
  if (*ptr && *have >= need) return RG_OK;
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  *have = 0;
  cudaError_t e = cudaMalloc((void**)ptr, sizeof(T) * need);
  if (e != cudaSuccess) return set_error(ctx, RG_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  *have = need;
  return RG_OK;
}

template <int N>
static int launch_ts_batch(rg_context* ctx, const cf* spec, cf* work, size_t stride, const TsBatch& bt,
                           const float* wtab, int wpitch, const TsCoef* d_co, const float* xe_box, double* acc,
                           cudaStream_t st) {
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  using C = Cfg<N>;
  const double nzc = (double)C::NZ * N * N, n3 = (double)N * N * N;
  const size_t smx = sizeof(cf) * (N + (size_t)line_buf<N, C::BX>());
  RG_CUDA_TRY(ctx, cudaFuncSetAttribute(k_ts_x<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
  prof_begin(ctx, "ts_x_c2c_combine_window", st);
  k_ts_x<N><<<dim3(N / C::BX, C::NZ), C::T * C::BX, smx, st>>>(spec, stride, work, bt, wtab, wpitch, tw);
  double src_reads = 0;
  for (int r = 0; r < bt.nr; ++r) src_reads += bt.nk[r];
  prof_end(ctx, 2 * 8.0 * nzc * (src_reads + bt.nr), st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  const size_t smy = sizeof(cf) * (N + (size_t)C::BY * C::PITCH_P);
  RG_CUDA_TRY(ctx, cudaFuncSetAttribute(k_pass_y<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smy));
  prof_begin(ctx, "ts_y_c2c", st);
  k_pass_y<N, true><<<dim3(N / C::BY, C::NZ, 2 * bt.nr), C::T * C::BY, smy, st>>>(work, stride, tw);
  prof_end(ctx, 2 * bt.nr * 16.0 * nzc, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  using Z = TsZ<N>;
  const size_t smz = Z::smem();
  RG_CUDA_TRY(ctx, cudaFuncSetAttribute(k_ts_z<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz));
  prof_begin(ctx, "ts_z_c2r_accumulate", st);
  k_ts_z<N><<<dim3(N / (2 * Z::Q), N), Z::NTH, smz, st>>>(work, stride, tw, d_co, xe_box, acc);
  // Hermitian halves of both grids per shell, x_e read, four FP64 sums read (after the first
  // batch) and written
  prof_end(ctx, bt.nr * 2 * 8.0 * nzc + 4.0 * n3 + 32.0 * n3 * 2, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

static int ts_batch(rg_context* ctx, int n, const cf* spec, cf* work, size_t stride, const TsBatch& bt,
                    const float* wtab, int wpitch, const TsCoef* d_co, const float* xe_box, double* acc,
                    cudaStream_t st) {
  switch (n) {
    case 8: return launch_ts_batch<8>(ctx, spec, work, stride, bt, wtab, wpitch, d_co, xe_box, acc, st);
    case 16: return launch_ts_batch<16>(ctx, spec, work, stride, bt, wtab, wpitch, d_co, xe_box, acc, st);
    case 32: return launch_ts_batch<32>(ctx, spec, work, stride, bt, wtab, wpitch, d_co, xe_box, acc, st);
    case 64: return launch_ts_batch<64>(ctx, spec, work, stride, bt, wtab, wpitch, d_co, xe_box, acc, st);
    case 128: return launch_ts_batch<128>(ctx, spec, work, stride, bt, wtab, wpitch, d_co, xe_box, acc, st);
    case 256: return launch_ts_batch<256>(ctx, spec, work, stride, bt, wtab, wpitch, d_co, xe_box, acc, st);
    case 512: return launch_ts_batch<512>(ctx, spec, work, stride, bt, wtab, wpitch, d_co, xe_box, acc, st);
    default: return set_error(ctx, RG_EUNSUPPORTED, "ComputeTs needs a power-of-two ReionGridDim");
  }
}

static double pow2_scale(double maxabs) {
  if (!(maxabs > 0) || !std::isfinite(maxabs)) return 1.0;
  return std::ldexp(1.0, -std::ilogb(maxabs));
}

int ts_snapshot(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g, rg_ts_scalars* out,
                const rg_grids* src_host) {
  int rc;
  cudaStream_t st = ctx->stream;
  const int N = ctx->N;
  const size_t n3 = (size_t)N * N * N;
  const Cosmo cm(p);
  const Units u = make_units(p);
  const double zp = s->ZZ[s->snapshot];
  const double box_size = p->BoxSize / p->Hubble_h;  // Mpc
  const double pixel_volume = std::pow(box_size / (double)N, 3);
  std::memset(out, 0, sizeof(*out));

  // device constants: kappa splines and number densities
  TsDev hc;
  std::memset(&hc, 0, sizeof(hc));
  fill_spline(ctx->tables.k10, ctx->tables.k10_lT, ctx->tables.k10_lk, &hc.k10);
  fill_spline(ctx->tables.kel, ctx->tables.kel_lT, ctx->tables.kel_lk, &hc.kel);
  fill_spline(ctx->tables.kpH, ctx->tables.kpH_lT, ctx->tables.kpH_lk, &hc.kpH);
  hc.No = cm.No;
  hc.N_b0 = cm.N_b0;
  hc.f_H = cm.f_H;
  hc.f_He = cm.f_He;
  hc.h = p->Hubble_h;
  hc.OMm = p->OmegaM;
  hc.OMr = p->OmegaR;
  hc.OMl = p->OmegaLambda;
  // device constants, the non-convergence counter and the per-batch coefficients live in one
  // context buffer: [TsDev][int + pad][TsCoef x batches]
  const int nS_all = p->TsNumFilterSteps;
  const int nbatch_max = (nS_all + TS_KB - 1) / TS_KB;
  const size_t off_co = (sizeof(TsDev) + 16 + 255) / 256 * 256;
  if ((rc = ensure_mem(ctx, &ctx->ts_const, &ctx->ts_const_elems, off_co + sizeof(TsCoef) * nbatch_max))) return rc;
  TsDev* d_hc = reinterpret_cast<TsDev*>(ctx->ts_const);
  int* d_nonconv = reinterpret_cast<int*>(ctx->ts_const + sizeof(TsDev));
  TsCoef* d_co_all = reinterpret_cast<TsCoef*>(ctx->ts_const + off_co);
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(d_hc, &hc, sizeof(TsDev), cudaMemcpyHostToDevice, st));
  RG_CUDA_TRY(ctx, cudaMemsetAsync(d_nonconv, 0, sizeof(int), st));
  const int nblk = 148 * 8;
  double* partials = ensure_partials(ctx, (size_t)nblk * TS_NSUM);
  if (!partials) return set_error(ctx, RG_ENOMEM, "partials");

  const double R0 = L_FACTOR * box_size / (float)N;
  const double Mh2 = rtom(p, R0) * p->Hubble_h * p->Hubble_h;
  const double ftpr3 = (4.0 / 3.0) * M_PI * std::pow(R0, 3.0) / pixel_volume;

  auto finish = [&](bool homog) -> int {
    if ((rc = reduce_partials(ctx, partials, nblk, TS_NSUM, ctx->d_sums, st))) return rc;
    RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_sums, ctx->d_sums, sizeof(double) * TS_NSUM, cudaMemcpyDeviceToHost, st));
    int nonconv = 0;
    RG_CUDA_TRY(ctx, cudaMemcpyAsync(&nonconv, d_nonconv, sizeof(int), cudaMemcpyDeviceToHost, st));
    RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    prof_resolve(ctx);
    const double* S = ctx->h_sums;
    const double nn = (double)n3;
    if (!homog) {
      out->volume_ave_J_alpha = S[0] / nn;
      out->volume_ave_xalpha = S[1] / nn;
      out->volume_ave_Xheat = S[2] / nn;
      out->volume_ave_Xion = S[3] / nn;
    }
    out->volume_ave_TS = S[4] / nn;
    out->volume_ave_TK = S[5] / nn;
    out->volume_ave_xe = S[6] / nn;
    out->homogeneous = homog;
    if (nonconv) return set_error(ctx, RG_ETIMEDOUT, "get_Ts did not converge in 10000 iterations for some cells");
    return RG_OK;
  };

  // collapse fraction and <x_e> (both branches compute the collapse fraction)
  prof_begin(ctx, "ts_reduce0", st);
  k_ts_reduce0<<<nblk, 256, 0, st>>>(g->stars, g->deltax, g->x_e_box_prev, N, Mh2, ftpr3, partials);
  prof_end(ctx, 12.0 * n3, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  if ((rc = reduce_partials(ctx, partials, nblk, 2, ctx->d_sums, st))) return rc;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_sums, ctx->d_sums, sizeof(double) * 2, cudaMemcpyDeviceToHost, st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  const double collapse_fraction = ctx->h_sums[0] / (double)n3;
  const double x_e_ave = ctx->h_sums[1] / (double)n3;
  out->collapse_fraction = collapse_fraction;
  out->x_e_ave = x_e_ave;

  if ((zp - p->ReionMaxHeatingRedshift) >= -0.0001) {
    const float xe0 = (float)xion_RECFAST(ctx->tables, (float)zp);
    const float TK0 = (float)T_RECFAST(ctx->tables, (float)zp);
    prof_begin(ctx, "ts_homog", st);
    k_ts_homog<<<nblk, 256, 0, st>>>(d_hc, (float)zp, xe0, TK0, cT_approx((float)zp), N, g->deltax, g->x_e_box_prev,
                                      g->x_e_box, g->Tk_box, g->TS_box, partials, d_nonconv);
    prof_end(ctx, 28.0 * n3, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
    return finish(true);
  }

  // inhomogeneous branch
  TsShells sh = ts_shells(p, s->ZZ, s->n_snapshots, s->snapshot, src_host ? src_host->n_hist : g->n_hist);
  if (sh.error) return set_error(ctx, RG_EINVAL, sh.msg);
  const int nS = sh.nS;
  const bool no_light = !(collapse_fraction > 0.0);
  const TsPrefactors pf = ts_prefactors(p, zp);
  const double prev_redshift = s->snapshot == 0 ? s->ZZ[s->snapshot] : s->ZZ[s->snapshot - 1];
  const size_t nc = (size_t)(N / 2 + 1) * N * N;
  const size_t npad = (size_t)N * N * 2 * (N / 2 + 1);
  if ((rc = ensure_mem(ctx, &ctx->ts_acc, &ctx->ts_acc_elems, 4 * n3))) return rc;

  if (!no_light) {
    if (!s->stored_fcoll && s->snapshot > 0)
      return set_error(ctx, RG_EINVAL, "ComputeTs needs stored_fcoll of the previous snapshot");
    TsTables tb;
    std::string msg;
    if ((rc = ts_tables(p, ctx->tables, sh, zp, x_e_ave, collapse_fraction, s->ZZ, s->stored_fcoll, s->snapshot, &tb,
                        &msg)))
      return set_error(ctx, rc, msg);
    // sources used by any shell
    std::vector<int> slot_of(sh.nsrc, -1), used;
    for (int r = 0; r < nS; ++r)
      for (int k = 0; k < sh.nsrc; ++k)
        if (sh.coef[(size_t)r * sh.nsrc + k] != 0.f && slot_of[k] < 0) {
          slot_of[k] = (int)used.size();
          used.push_back(k);
        }
    for (int r = 0; r < nS; ++r) {
      int nk = 0;
      for (int k = 0; k < sh.nsrc; ++k) nk += sh.coef[(size_t)r * sh.nsrc + k] != 0.f;
      if (nk > TS_MAXSRC) return set_error(ctx, RG_EUNSUPPORTED, "a shell combines more than 4 history snapshots");
    }
    const int nused = std::max(1, (int)used.size());
    if ((rc = ensure_mem(ctx, &ctx->spec, &ctx->spec_elems, nc * 2 * nused))) return rc;
    const int kb = std::min(TS_KB, nS);
    if ((rc = ensure_mem(ctx, &ctx->work, &ctx->work_elems, nc * 2 * kb))) return rc;
    // source grid `which` (0 sfr, 1 xray) of source k, on the device
    const rg_grids* sg = src_host ? src_host : g;
    auto src_grid = [&](int k, int which) -> const float* {
      if (k == 0) return which ? sg->xray_luminosity : sg->sfr;
      return (which ? sg->xray_luminosity_histories : sg->sfr_histories) + (size_t)(k - 1) * npad;
    };
    if (src_host) {
      if ((rc = ensure_mem(ctx, &ctx->ts_stage, &ctx->ts_stage_elems, npad * 2 * used.size()))) return rc;
      for (size_t j = 0; j < used.size(); ++j)
        for (int which = 0; which < 2; ++which)
          RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->ts_stage + (j * 2 + which) * npad, src_grid(used[j], which),
                                           sizeof(float) * npad, cudaMemcpyHostToDevice, st));
    }
    auto dev_grid = [&](size_t j, int which) -> const float* {
      return src_host ? ctx->ts_stage + (j * 2 + which) * npad : src_grid(used[j], which);
    };
    // forward transforms of the used sources: spec[(slot * 2 + g)]
    for (size_t i = 0; i < used.size(); i += 4) {
      const float* srcs[8];
      int ng = 0;
      for (size_t j = i; j < used.size() && j < i + 4; ++j) {
        srcs[ng++] = dev_grid(j, 0);
        srcs[ng++] = dev_grid(j, 1);
      }
      if ((rc = fft_forward(ctx, N, srcs, ng, ctx->spec + nc * 2 * i, nc, 1.0 / std::pow((double)N, 3), st))) return rc;
    }
    // window rows for the shells (filter() takes BoxSize in Mpc/h and R in Mpc, ComputeTs.c:532)
    const int n2max = 3 * (N / 2) * (N / 2);
    if ((rc = ensure_mem(ctx, &ctx->d_radii, &ctx->d_radii_elems, (size_t)nS))) return rc;
    RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_radii, sh.R.data(), sizeof(double) * nS, cudaMemcpyHostToDevice, st));
    if ((rc = ensure_mem(ctx, &ctx->wtab, &ctx->wtab_elems, (size_t)nS * (n2max + 1)))) return rc;
    if ((rc = window_table(ctx, p->BoxSize, ctx->d_radii, nS, p->TsHeatingFilterType, ctx->wtab, n2max, st))) return rc;

    // per-shell coefficients.  evolveInt sums over shells R (XRayHeatingFunctions.c:1379-1432):
    //   heat/ion/lya: dt_dzpp dzpp XRAY_R (1+zpp)^-alpha fi_k(x_e)     (times const_zp later)
    //   star        : SFR_R (1+zp)^2 (1+zpp) sum_lyn dt_dzpp dzpp      (times the conversion)
    // with XRAY_R = xray / pv * 1e40 UL^-3 and SFR_R = max(sfr,0) / pv * (UM/UT) UL^-3 / Msun.
    const double convX = 1.0 / pixel_volume * XRAY_LUMINOSITY_UNIT * std::pow(p->UnitLength_in_cm, -3.);
    const double convS = 1.0 / pixel_volume * (p->UnitMass_in_g / u.UnitTime_in_s) *
                         std::pow(p->UnitLength_in_cm, -3.) / SOLAR_MASS;
    const float zpf = (float)zp;
    const double opzf2 = std::pow((double)(1.0f + zpf), 2);
    std::vector<double> Pd((size_t)nS * 3 * x_int_NXHII), Qd((size_t)nS * 3 * x_int_NXHII), cs(nS);
    double maxk[4] = {0, 0, 0, 0};
    const float* X = ctx->tables.x_int_XHII.data();
    for (int r = 0; r < nS; ++r) {
      const double a = sh.dt_dzpp[r] * sh.dzpp[r];
      const double pw = std::pow(1 + sh.zpp[r], -p->SpecIndexXrayGal);
      for (int kind = 0; kind < 3; ++kind) {
        const std::vector<double>& tb_k = kind == 0 ? tb.heat : kind == 1 ? tb.ion : tb.lya;
        for (int m = 0; m < x_int_NXHII; ++m) {
          const double t_lo = tb_k[(size_t)m * nS + r];
          const double t_hi = m + 1 < x_int_NXHII ? tb_k[(size_t)(m + 1) * nS + r] : t_lo;
          const double slope = m + 1 < x_int_NXHII ? (t_hi - t_lo) / ((double)X[m + 1] - (double)X[m]) : 0.0;
          Pd[((size_t)r * 3 + kind) * x_int_NXHII + m] = a * convX * pw * t_lo;
          Qd[((size_t)r * 3 + kind) * x_int_NXHII + m] = a * convX * pw * slope;
          maxk[kind] = std::max({maxk[kind], std::fabs(a * convX * pw * t_lo), std::fabs(a * convX * pw * t_hi)});
        }
      }
      cs[r] = convS * opzf2 * (1 + sh.zpp[r]) * tb.sum_lyn[r] * a;
      maxk[3] = std::max(maxk[3], std::fabs(cs[r]));
    }
    // FP32 within a batch: scale each sum by a power of two that brings its largest
    // per-shell coefficient near 1 (values of order 1e-30 would lose range in float)
    double scale[4];
    for (int k = 0; k < 4; ++k) scale[k] = pow2_scale(maxk[k]);
    TsCoef* d_co = d_co_all;
    const int nbatch = (nS + kb - 1) / kb;
    std::vector<TsCoef> hco(nbatch);
    for (int bi = 0; bi < nbatch; ++bi) {
      const int r0 = bi * kb, cnt = std::min(kb, nS - r0);
      TsCoef& co = hco[bi];
      std::memset(&co, 0, sizeof(co));
      co.nr = cnt;
      co.first = bi == 0;
      for (int m = 0; m < x_int_NXHII; ++m) co.X[m] = X[m];
      for (int k = 0; k < 4; ++k) co.inv_scale[k] = 1.0 / scale[k];
      TsBatch bt;
      std::memset(&bt, 0, sizeof(bt));
      bt.nr = cnt;
      for (int j = 0; j < cnt; ++j) {
        const int r = r0 + j;
        for (int kind = 0; kind < 3; ++kind)
          for (int m = 0; m < x_int_NXHII; ++m) {
            co.P[j][kind][m] = (float)(Pd[((size_t)r * 3 + kind) * x_int_NXHII + m] * scale[kind]);
            co.Q[j][kind][m] = (float)(Qd[((size_t)r * 3 + kind) * x_int_NXHII + m] * scale[kind]);
          }
        co.cstar[j] = (float)(cs[r] * scale[3]);
        int nk = 0;
        for (int k = 0; k < sh.nsrc; ++k) {
          const float c = sh.coef[(size_t)r * sh.nsrc + k];
          if (c != 0.f) {
            bt.ks[j][nk] = slot_of[k];
            bt.cs[j][nk] = c;
            nk++;
          }
        }
        bt.nk[j] = nk;
        bt.filtered[j] = r > 0;  // no filter on the first shell (ComputeTs.c:529)
        bt.wrow[j] = r;
      }
      RG_CUDA_TRY(ctx, cudaMemcpyAsync(d_co + bi, &co, sizeof(TsCoef), cudaMemcpyHostToDevice, st));
      if ((rc = ts_batch(ctx, N, ctx->spec, ctx->work, nc, bt, ctx->wtab, n2max + 1, d_co + bi, g->x_e_box_prev,
                         ctx->ts_acc, st)))
        return rc;
    }
    RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));  // hco outlives the copies
  }

  TsEvolve e;
  e.zp_f = (float)zp;
  e.zp = zp;
  e.dzp = zp - prev_redshift;
  e.dt_dzp = pf.dt_dzp;
  e.growth = pf.growth_factor_zp;
  e.dgrowth = pf.dgrowth_factor_dzp;
  e.const_zp = pf.const_zp_prefactor_GAL;
  // Conversion_factor (XRayHeatingFunctions.c:1331-1332)
  e.conv_star = (SPEED_OF_LIGHT / (4. * M_PI)) / (PROTONMASS / SOLAR_MASS);
  e.no_light = no_light;
  prof_begin(ctx, "ts_evolve", st);
  k_ts_evolve<<<nblk, 256, 0, st>>>(d_hc, e, N, ctx->ts_acc, g->deltax, g->x_e_box_prev, g->x_e_box, g->Tk_box,
                                     g->TS_box, partials, d_nonconv);
  prof_end(ctx, (double)n3 * (32 + 4 + 4 + 4 + 4 + 4 + 4 + 4), st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return finish(false);
}

}  // namespace rg
