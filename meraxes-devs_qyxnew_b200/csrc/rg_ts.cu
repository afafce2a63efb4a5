// Spin-temperature step (_ComputeTs, src/core/ComputeTs.c:85-1554) on sm_100a, with the AGN
// X-ray channels (Flag_IncludeAGNXray) and without the mini-halo channels.
//
// Inhomogeneous branch, per snapshot:
//   1. FP64 reductions of the collapse fraction and <x_e> (ComputeTs.c:585-677)
//   2. host: frequency-integral tables, Lyman-n sums, prefactors (rg_xray.cpp)
//   3. forward r2c of every source grid (this snapshot's sfr / xray_luminosity and the
//      history slots the shells use); each shell's source is a linear combination of them
//      (the history re-weighting of :366-478), formed in k-space on load
//   4. shells in batches: x pass (combination, TsHeatingFilterType window), y pass, z pass
//      that turns the grids of every shell (sfr, X-ray, then the AGN soft and / or hard
//      emissivity) into the four per-cell sums of
//      evolveInt (X-ray heating, ionisation and Lyman-alpha integrands, stellar Lyman-alpha)
//      without storing the reference's SMOOTHED_*[nS N^3] arrays
//   5. per cell, FP64: evolveInt, the Euler step of x_e and T_K, get_Ts, and the FP64 sums
// Homogeneous branch (zp >= ReionMaxHeatingRedshift): RECFAST x_e and T_K, get_Ts with no
// Lyman-alpha coupling (:252-331).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstring>
#include <vector>

#include "rg_internal.h"
#include "rg_pass.cuh"
#include "rg_tma.cuh"
#include "rg_xray.h"

namespace rg {

constexpr int TS_KB = 8;        // shells per batch
constexpr int TS_MAXSRC = 4;    // sources combined into one shell
constexpr int TS_NSUM = 9;      // evolve sums (7, 8: the AGN heating of the two AGN units)
constexpr int KSPL = 27;        // knots of the largest kappa table

struct KappaSpline {
  int n;
  double x[KSPL], y[KSPL], b[KSPL], c[KSPL], d[KSPL];
};

// per-snapshot constants of the per-cell physics (the factors of xcoll, taugp, xalpha_tilde,
// dT_comp and evolveInt that depend on the redshift only), computed on the host in FP64
struct TsZConst {
  double Trad, inv_Trad;       // TCMB (1 + z), z the float redshift
  double xc_H, xc_e, xc_p;     // T21 / Trad / A10 x {No, N_b0, No} (1 + z)^3   (xcoll_HI/elec/prot)
  double tgp0;                 // 1.342881e-7 / hubble(z) No (1 + z)^3          (taugp)
  double xa0;                  // 1.66e11 / (1 + z)                             (xalpha_tilde)
  double nb0;                  // N_b0 (1 + z)^3                                (evolveInt n_b)
  double comp0;                // -1.51e-4 / (H(z) / H0) / h Trad^4 / (1 + z)    (dT_comp)
  double dadia0;               // 3 / (1 + z)
  double f_H, f_He;
};

struct TsDev {
  KappaSpline k10, kel, kpH;
  TsZConst z;
  int max_iter;   // get_Ts fixed-point iterations before a cell counts as not converged
  int pad_;
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

// log kappa_10 at log T (XRayHeatingFunctions.c:1728-1822): below the table its first value,
// above it the T^0.381 power law log(exp(y_n) (T / exp(x_n))^0.381) = y_n + 0.381 (log T - x_n)
__device__ __forceinline__ double log_kappa_10(const KappaSpline& s, double lt) {
  if (lt < s.x[0]) return s.y[0];
  if (lt > s.x[s.n - 1]) return s.y[s.n - 1] + 0.381 * (lt - s.x[s.n - 1]);
  return spline_eval(s, lt);
}

// log kappa_10_elec / kappa_10_pH at log T (XRayHeatingFunctions.c:1827-1966): linear
// extrapolation of the last segment above the table
__device__ __forceinline__ double log_kappa_table(const KappaSpline& s, double lt) {
  if (lt < s.x[0]) return s.y[0];
  if (lt > s.x[s.n - 1])
    return s.y[s.n - 1] + ((s.y[s.n - 1] - s.y[s.n - 2]) / (s.x[s.n - 1] - s.x[s.n - 2]) * (lt - s.x[s.n - 1]));
  return spline_eval(s, lt);
}

// get_Ts with xcoll and the Wouthuysen-Field coupling (XRayHeatingFunctions.c:1639-1726,
// 1973-2008).  The factors that do not change across the fixed-point iterations (xcoll, the
// S_alpha terms in T_K only, xi) are evaluated once per cell.  The loop is capped at
// C.max_iter iterations (10000 unless a test lowers it); a cell that reaches the cap counts in
// *nonconv.
__device__ float get_Ts(const TsDev& C, float delta, float TK, float xe, float Jalpha, float* curr_xalpha,
                        int* nonconv) {
  const TsZConst& Z = C.z;
  const double tk = (double)TK, d1 = 1.0 + (double)delta, x = (double)xe;
  const double lt = log(tk);
  const double xc = Z.xc_H * (1.0 - x) * d1 * exp(log_kappa_10(C.k10, lt)) +
                    Z.xc_e * x * d1 * exp(log_kappa_table(C.kel, lt)) +
                    Z.xc_p * x * d1 * exp(log_kappa_table(C.kpH, lt));
  const double itk = 1.0 / tk;
  double TS;
  if ((double)Jalpha > 1.0e-20) {
    const double tgp = Z.tgp0 * d1 * (1.0 - x);
    const double xi = cbrt(1.0e-7 * tgp * itk * itk);
    const double den = 1.0 + 2.98394 * xi + 1.53583 * xi * xi + 3.85289 * xi * xi * xi;
    const double sa = 1.0 - 0.0631789 * itk + 0.115995 * itk * itk;    // S_alpha terms in T_K only
    const double sb = (-0.401403 + 0.336463 * itk) * itk;                 // times 1 / T_S
    const double xaj = Z.xa0 * (double)Jalpha / den;
    const double ctc = 0.405535 * itk;
    TS = Z.Trad;
    double TSold = 0.0, xa_tilde = 0.0;
    int it = 0;
    while (fabs(TS - TSold) / TS > 1.0e-3) {
      if (++it > C.max_iter) {
        *nonconv += 1;
        break;
      }
      TSold = TS;
      const double u = 1.0 / TS;
      xa_tilde = xaj * (sa + sb * u);
      const double tce_inv = itk + ctc * (u - itk);                        // 1 / Tc_eff
      TS = (1.0 + xa_tilde + xc) / (Z.inv_Trad + xa_tilde * tce_inv + xc * itk);
    }
    *curr_xalpha = (float)xa_tilde;
  } else {
    TS = (1.0 + xc) / (Z.inv_Trad + xc * itk);
    *curr_xalpha = 0;
  }
  if (TS < 0.) TS = fabs(TS);
  return (float)TS;
}

// alpha_A (XRayHeatingFunctions.c:1576-1584): exp of a degree-9 polynomial in
// log(T / 1.1604505e4), evaluated by Horner's rule
__device__ __forceinline__ double alpha_A(double T) {
  const double l = log(T / 1.1604505e4);
  const double poly =
      -28.6130338 +
      l * (-0.72411256 +
           l * (-2.02604473e-2 +
                l * (-2.38086188e-3 +
                     l * (-3.21260521e-4 +
                          l * (-1.42150291e-5 +
                               l * (4.98910892e-6 + l * (5.75561414e-7 + l * (-1.85676704e-8 + l * -3.07113524e-9))))))));
  return exp(poly);
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
  int ng;             // grids per shell: sfr, X-ray, then 0 to 2 AGN bands
};

template <int N>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::BX, (x_pass_minb<N>()))
    k_ts_x(const cf* __restrict__ spec, size_t stride, cf* __restrict__ work, TsBatch bt,
           const float* __restrict__ wtab, int wpitch, const int* __restrict__ wcut, const cf* __restrict__ g_tw) {
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
      if (wcut) {
        // sharp-k: the row is the step W = (n2 <= cut), no gathers
        const int cut = __ldg(wcut + bt.wrow[r]);
#pragma unroll
        for (int sl = 0; sl < V; ++sl) wv[sl] = n2[sl] <= cut ? 1.f : 0.f;
      } else {
        const float* wr = wtab + (size_t)bt.wrow[r] * wpitch;
#pragma unroll
        for (int sl = 0; sl < V; ++sl) wv[sl] = __ldg(wr + n2[sl]);
      }
    }
    const int nk = bt.nk[r];
    const int G = bt.ng;
    for (int g = 0; g < G; ++g) {
      cf* dst = work + ((size_t)r * G + g) * stride;
      // the combination sum_i c_i spec_i of this thread's V input positions, source by source:
      // the V loads of a source are independent and in flight together (per element the same
      // fmaf sequence in the order of i)
      cf in[V];
#pragma unroll
      for (int sl = 0; sl < V; ++sl) in[sl] = cf{0.f, 0.f};
      for (int i = 0; i < nk; ++i) {
        const float c = bt.cs[r][i];
        const cf* src = spec + ((size_t)bt.ks[r][i] * G + g) * stride + col;
        cf v[V];
#pragma unroll
        for (int sl = 0; sl < V; ++sl) v[sl] = src[(size_t)stage0_pos<N>(t, sl) * N];
#pragma unroll
        for (int sl = 0; sl < V; ++sl) {
          in[sl].x = fmaf(c, v[sl].x, in[sl].x);
          in[sl].y = fmaf(c, v[sl].y, in[sl].y);
        }
      }
      line_fft<N, true>(
          t, xbuf, s_tw, [&](int, int sl) { return cf{in[sl].x * wv[sl], in[sl].y * wv[sl]}; },
          [&](int p) { return line_addr<N, B>(p, b); }, [&](int p, cf v) { dst[col + (size_t)p * N] = v; });
    }
  }
}

// ---------------------------------------------------------------------------
// per-cell evolution (evolveInt + the Euler step + get_Ts, ComputeTs.c:1171-1407)

struct TsEvolve {
  double zp, dzp, dt_dzp, growth, dgrowth, const_zp, conv_star;
  double heat_conv;            // dt_dzp 2 / 3 / k_B
  int no_light;
};

// One cell: sums[0..3] = the four evolveInt shell sums (heat, ion, lya, stellar lya) before
// their snapshot prefactors; updates x_e and T_K, returns T_S and adds the cell to acc[0..6].
__device__ __forceinline__ void evolve_cell(const TsDev& C, const TsEvolve& e, float delta, float xef, float tk0,
                                            const double (&sums)[4], float* xn_out, float* tk_out, float* ts_out,
                                            double (&acc)[TS_NSUM], int* nc) {
  const TsZConst& Z = C.z;
  const double x_e = (double)xef, T = (double)tk0;
  const double n_b = Z.nb0 * (double)(1.0f + delta);
  double dxheat_dt = 0, dxion_src = 0, dxlya = 0, dstarlya = 0;
  if (!e.no_light) {
    dxheat_dt = sums[0] * e.const_zp;
    dxion_src = sums[1] * e.const_zp;
    dxlya = sums[2] * (e.const_zp * n_b);
    dstarlya = sums[3] * e.conv_star;
  }
  const double inv1x = 1.0 / (1.0 + x_e);
  const double dxion_sink = alpha_A(T) * CLUMPING_FACTOR * x_e * x_e * Z.f_H * n_b;
  const double dxe_dzp = e.dt_dzp * (dxion_src - dxion_sink);
  double dadia = Z.dadia0;
  if (fabs((double)delta) > FRACT_FLOAT_ERR) {
    const double dl = (double)delta;
    dadia += e.dgrowth * dl / (1.0 + e.growth * dl);      // dgrowth / (1 / delta + growth)
  }
  dadia *= (2.0 / 3.0) * T;
  const double dspec = -dxe_dzp * T * inv1x;
  const double dcomp = Z.comp0 * (x_e / (1.0 + x_e + Z.f_He)) * (Z.Trad - T);
  const double dxheat_dzp = dxheat_dt * e.heat_conv * inv1x;
  const double d1 = dxheat_dzp + dcomp + dspec + dadia;
  const double d2 = dxlya + dstarlya;
  const double d4 = e.dt_dzp * dxion_src;
  float xn = (float)((double)xef + dxe_dzp * e.dzp);
  if (xn > 1)
    xn = (float)(1 - FRACT_FLOAT_ERR);
  else if (xn < 0)
    xn = 0;
  float tk = tk0;
  if (tk < MAX_TK) tk = (float)((double)tk + d1 * e.dzp);
  if (tk < MIN_TK) tk = (float)(TCMB * (1 + e.zp));
  float xa;
  const float ts = get_Ts(C, delta, tk, xn, (float)d2, &xa, nc);
  *xn_out = xn;
  *tk_out = tk;
  *ts_out = ts;
  acc[0] += d2;
  acc[1] += (double)xa;
  acc[2] += dxheat_dzp;
  acc[3] += d4;
  acc[4] += (double)ts;
  acc[5] += (double)tk;
  acc[6] += (double)xn;
}

// ---------------------------------------------------------------------------
// shell z pass: for every shell r the c2r along z of its sfr and X-ray grids, accumulated per
// cell into the four evolveInt shell sums in registers over all shells, then stored once as a
// float4 per cell.  Two shells share one complex line (the two-for-one c2r of two real rows:
// shell r in the real part, shell r + 1 in the imaginary part; both rows are the same grid,
// filtered at neighbouring radii).
//
// Per shell: P_k[m], Q_k[m] (k = heat, ion, lya; m = x_e node) so that the cell's term is
// xray x (P_k[lo] + (x_e - X[lo]) Q_k[lo]), and cstar for max(sfr, 0); all scaled by a power of
// two per sum kind so FP32 keeps its range (the scale is undone in FP64 by the update kernel).

struct TsShellCoef {
  float P[3][x_int_NXHII];
  float Q[3][x_int_NXHII];
  float cstar;
  float pad;
  // AGN units j = 0, 1 (the bands in use, soft first): max(grid, 0) x (PA + dx QA), with the
  // ratio of the band's prefactor to the galaxies' folded in so the terms join the same sums
  float PA[2][3][x_int_NXHII];
  float QA[2][3][x_int_NXHII];
};

struct TsZev {
  int nS;
  float X[x_int_NXHII];           // x_int_XHII (float, as in the reference)
  double inv_scale[4];            // undo the FP32 scaling
};

template <int N>
struct TsZ {
  using PL = Plan8<N>;
  static constexpr int T = PL::T;
  static constexpr int V = N / T;            // 8
  static constexpr int R0 = PL::R[0];
  static constexpr int Q = pow2_div(N, cmax(256 / T, 4));   // rows per block
  static constexpr int NTH = T * Q;
  static constexpr int MINB = NTH >= 512 ? 1 : 512 / NTH;   // 2 blocks of 256: at most 128 registers
  static constexpr int NZ = N / 2 + 1;
  // kz rows per tensor box (at most 256): one box, or for N = 512 two of (NZ + 1) / 2 rows at kz 0
  // and NZ - KZB that overlap in one row, so the second lands on a 128-byte boundary
  static constexpr int KZB = NZ <= 256 ? NZ : (NZ + 1) / 2;
  static constexpr int NBOX = NZ <= 256 ? 1 : 2;
  static constexpr int TS = round_up(NZ * Q, 16);            // one shell's rows, a 128-byte multiple
  static constexpr size_t tile_elems() { return (size_t)2 * TS; }   // two shells' rows
  static constexpr uint32_t SHELL_TX = (uint32_t)(NBOX * KZB * Q * sizeof(cf));
  static constexpr int STAGES = 3;           // tiles in flight: units u + 1 and u + 2 load during u
  static constexpr size_t smem() {
    return 128 + sizeof(cf) * (STAGES * tile_elems() + (size_t)line_buf_r0<N, R0, Q>() + N) +
           sizeof(uint64_t) * STAGES;
  }
  static_assert(Q % 2 == 0 && 2 * Q <= 256, "tensor box of 2Q floats, x a 16-byte multiple");
  static_assert(NBOX == 1 || ((NZ - KZB) * Q * sizeof(cf)) % 128 == 0, "second box off a 128-byte boundary");
};

constexpr int TS_TMA_WAIT_LIMIT = 1 << 22;   // polls of an mbarrier before a wait gives up

// complex line of row q of the two shells in a tile (shell a real part, shell b imaginary part);
// the tile holds tile[s][k][j] = (s ? b : a)[k][x][y0 + j], shell b at TS
template <int N, int Q>
__device__ __forceinline__ cf ts_tile_input(const cf* tile, int q, int p) {
  constexpr int TS = TsZ<N>::TS;
  const int k = p <= N / 2 ? p : N - p;
  const cf A = tile[k * Q + q], B = tile[TS + k * Q + q];
  if (p == 0 || p == N / 2) return cf{A.x, B.x};
  if (p < N / 2) return cf{A.x - B.y, A.y + B.x};
  return cf{A.x + B.y, B.x - A.y};
}

// G grids per shell: 0 sfr, 1 X-ray, 2 and 3 the AGN bands in use (their per-cell heating
// terms also go to agn_heat, for the AGN heating averages)
// The shells' Hermitian column tiles arrive by tensor loads (the spectra as the tensor `tmap`:
// floats y innermost, then x, then kz of spectrum r G + g at (r G + g)(N/2 + 1) + kz), STAGES
// tiles in flight, one mbarrier each.
template <int N, int G>
__global__ void __launch_bounds__(TsZ<N>::NTH, TsZ<N>::MINB)
    k_ts_zsum(const __grid_constant__ CUtensorMap tmap, const cf* __restrict__ g_tw,
              const TsShellCoef* __restrict__ gco, TsZev zv, const float* __restrict__ xe_prev,
              float4* __restrict__ sums, float2* __restrict__ agn_heat, uint32_t* err) {
  using Z = TsZ<N>;
  using PL = typename Z::PL;
  constexpr int Q = Z::Q, V = Z::V, NZ = Z::NZ, KZB = Z::KZB;
  constexpr int PADW = 2 * (N / 2 + 1);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  cf* tiles = reinterpret_cast<cf*>(sm);
  cf* xbuf = tiles + Z::STAGES * Z::tile_elems();
  cf* s_tw = xbuf + line_buf_r0<N, Z::R0, Q>();
  uint64_t* bars = reinterpret_cast<uint64_t*>(s_tw + N);
  __shared__ TsShellCoef sc[2];
  const int x = blockIdx.y, y = blockIdx.x * Q + threadIdx.x % Q;
  const int t = threadIdx.x / Q;
  if (threadIdx.x == 0) {
    for (int b = 0; b < Z::STAGES; ++b) mbar_init(&bars[b], 1);
    mbar_init_fence();
  }
  load_twiddles_p<PL>(s_tw, g_tw);
  const size_t row = (size_t)x * N + y;
  // this thread's cells: z = last_pos(t, s); x_e interpolation node and offset
  // (ComputeTs.c:1198-1209)
  float dxe[V];
  uint32_t lopack = 0;
#pragma unroll
  for (int sl = 0; sl < V; ++sl) {
    double xc = (double)__ldg(xe_prev + row * PADW + last_pos<PL>(t, sl));
    if (xc > (double)zv.X[x_int_NXHII - 1] * 0.999)
      xc = (double)zv.X[x_int_NXHII - 1] * 0.999;
    else if (xc < (double)zv.X[0])
      xc = 1.001 * (double)zv.X[0];
    // locate_xHII_index: the last node not above x_e (constant indices keep zv in the
    // parameter bank)
    const float xf = (float)xc;
    int m = 0;
    float xm = zv.X[0];
#pragma unroll
    for (int j = 1; j < x_int_NXHII; ++j)
      if (!(xf < zv.X[j])) {
        m = j;
        xm = zv.X[j];
      }
    lopack |= (uint32_t)m << (4 * sl);
    dxe[sl] = (float)(xc - (double)xm);
  }
  // every thread's cells each on one x_e node of their own (the common case early in
  // reionization): the coefficient reads leave the per-cell loops.  The choice is the block's, as
  // both paths run transforms with block barriers.
  static_assert(V == 8, "eight x_e node indices in one 32-bit word");
  const uint32_t lo0 = lopack & 15u;
  const bool uni = __syncthreads_and(lopack == lo0 * 0x11111111u) != 0;
  float a_heat[V], a_ion[V], a_lya[V], a_star[V];
  float a_agn0[G > 2 ? V : 1], a_agn1[G > 3 ? V : 1];
#pragma unroll
  for (int sl = 0; sl < V; ++sl) a_heat[sl] = a_ion[sl] = a_lya[sl] = a_star[sl] = 0.f;
#pragma unroll
  for (int sl = 0; sl < (G > 2 ? V : 1); ++sl) a_agn0[sl] = 0.f;
#pragma unroll
  for (int sl = 0; sl < (G > 3 ? V : 1); ++sl) a_agn1[sl] = 0.f;
  auto addr = [&](int p) { return line_addr_r0<Z::R0, Q>(p, threadIdx.x % Q); };
  // units u = G (r / 2) + g: the pair of shells (r, r + 1), grid g; the tiles of units u + 1 and
  // u + 2 load while unit u is transformed (three buffers).  A pair without its second shell (an
  // odd count) gets zeros there, written by the block.
  constexpr int S = Z::STAGES;
  const int y0 = blockIdx.x * Q, q = threadIdx.x % Q;
  const int nunits = G * ((zv.nS + 1) / 2);
  auto has_b = [&](int u) { return 2 * (u / G) + 1 < zv.nS; };
  // thread 0: tensor loads of unit u into its buffer
  auto issue = [&](int u) {
    const int b = u % S;
    const bool two = has_b(u);
    mbar_arrive_expect_tx(&bars[b], (two ? 2u : 1u) * Z::SHELL_TX);
    for (int sh = 0; sh < (two ? 2 : 1); ++sh) {
      const int spec = (2 * (u / G) + sh) * G + u % G;
#pragma unroll
      for (int k = 0; k < Z::NBOX; ++k) {
        const int k0 = k ? NZ - KZB : 0;
        tma_load_3d(tiles + b * Z::tile_elems() + sh * Z::TS + k0 * Q, &tmap, 2 * y0, x, spec * NZ + k0, &bars[b]);
      }
    }
  };
  auto zero_b = [&](int u) {
    cf* tb = tiles + (u % S) * Z::tile_elems() + Z::TS;
    for (int i = threadIdx.x; i < NZ * Q; i += Z::NTH) tb[i] = cf{0.f, 0.f};
  };
  __syncthreads();   // barriers initialised
  if (threadIdx.x == 0)
    for (int u = 0; u < S - 1 && u < nunits; ++u) issue(u);
  for (int u = 0; u < S - 1 && u < nunits; ++u)
    if (!has_b(u)) zero_b(u);
  bool waited = true;
  // an AGN unit j: clamped at 0 (ComputeTs.c:615-630), its own band tables
  auto agn_unit = [&](const cf* tile, int j, float (&ah)[G > 2 ? V : 1]) {
    line_fft_p<PL, true>(
        t, xbuf, s_tw, [&](int p, int) { return ts_tile_input<N, Q>(tile, q, p); }, addr,
        [&](int, cf v, int sl) {
          const int lo = (int)((lopack >> (4 * sl)) & 15u);
          const float d = dxe[sl];
          const float vx = fmaxf(v.x, 0.f), vy = fmaxf(v.y, 0.f);
          const float h = vx * fmaf(d, sc[0].QA[j][0][lo], sc[0].PA[j][0][lo]) +
                          vy * fmaf(d, sc[1].QA[j][0][lo], sc[1].PA[j][0][lo]);
          a_heat[sl] += h;
          ah[sl] += h;
          a_ion[sl] += vx * fmaf(d, sc[0].QA[j][1][lo], sc[0].PA[j][1][lo]) +
                       vy * fmaf(d, sc[1].QA[j][1][lo], sc[1].PA[j][1][lo]);
          a_lya[sl] += vx * fmaf(d, sc[0].QA[j][2][lo], sc[0].PA[j][2][lo]) +
                       vy * fmaf(d, sc[1].QA[j][2][lo], sc[1].PA[j][2][lo]);
        });
  };
  for (int u = 0; u < nunits; ++u) {
    const int r = 2 * (u / G), g = u % G;
    if (g == 0) {
      __syncthreads();  // readers of the previous pair's coefficients are done
      const bool two = r + 1 < zv.nS;
      const int* src = reinterpret_cast<const int*>(gco + r);
      int* dst = reinterpret_cast<int*>(sc);
      // words per shell: the AGN tables only when there are AGN units
      constexpr int SW = (int)(sizeof(TsShellCoef) / sizeof(int));
      constexpr int W = G > 2 ? SW : (int)(offsetof(TsShellCoef, PA) / sizeof(int));
      for (int i = threadIdx.x; i < 2 * W; i += Z::NTH) {
        const int sh = i / W, w = sh * SW + i % W;
        dst[w] = (sh == 0 || two) ? src[w] : 0;
      }
    }
    // buffer (u + 2) % 3 was consumed by unit u - 1 (the barrier at the end of its iteration)
    if (u + S - 1 < nunits) {
      if (threadIdx.x == 0) issue(u + S - 1);
      if (!has_b(u + S - 1)) zero_b(u + S - 1);
    }
    if (!mbar_wait(&bars[u % S], (uint32_t)((u / S) & 1), TS_TMA_WAIT_LIMIT)) waited = false;
    __syncthreads();  // unit u's tile (and the pair's coefficients) are visible to every thread
    const cf* tile = tiles + (u % S) * Z::tile_elems();
    if (g == 0) {
      // sfr: stellar Lyman-alpha sum, SFR clamped at 0 (ComputeTs.c:700)
      const float c0 = sc[0].cstar, c1 = sc[1].cstar;
      line_fft_p<PL, true>(
          t, xbuf, s_tw, [&](int p, int) { return ts_tile_input<N, Q>(tile, q, p); }, addr,
          [&](int, cf v, int sl) { a_star[sl] += fmaxf(v.x, 0.f) * c0 + fmaxf(v.y, 0.f) * c1; });
    } else if (g == 1) {
      // X-ray: heating, ionisation and Lyman-alpha integrands, not clamped
      if (uni) {
        // every cell of this thread on the same x_e node: its twelve coefficients read once
        float c[2][3][2];
#pragma unroll
        for (int sh = 0; sh < 2; ++sh)
#pragma unroll
          for (int kd = 0; kd < 3; ++kd) {
            c[sh][kd][0] = sc[sh].P[kd][lo0];
            c[sh][kd][1] = sc[sh].Q[kd][lo0];
          }
        line_fft_p<PL, true>(
            t, xbuf, s_tw, [&](int p, int) { return ts_tile_input<N, Q>(tile, q, p); }, addr,
            [&](int, cf v, int sl) {
              const float d = dxe[sl];
              a_heat[sl] += v.x * fmaf(d, c[0][0][1], c[0][0][0]) + v.y * fmaf(d, c[1][0][1], c[1][0][0]);
              a_ion[sl] += v.x * fmaf(d, c[0][1][1], c[0][1][0]) + v.y * fmaf(d, c[1][1][1], c[1][1][0]);
              a_lya[sl] += v.x * fmaf(d, c[0][2][1], c[0][2][0]) + v.y * fmaf(d, c[1][2][1], c[1][2][0]);
            });
      } else {
        line_fft_p<PL, true>(
            t, xbuf, s_tw, [&](int p, int) { return ts_tile_input<N, Q>(tile, q, p); }, addr,
            [&](int, cf v, int sl) {
              const int lo = (int)((lopack >> (4 * sl)) & 15u);
              const float d = dxe[sl];
              a_heat[sl] +=
                  v.x * fmaf(d, sc[0].Q[0][lo], sc[0].P[0][lo]) + v.y * fmaf(d, sc[1].Q[0][lo], sc[1].P[0][lo]);
              a_ion[sl] +=
                  v.x * fmaf(d, sc[0].Q[1][lo], sc[0].P[1][lo]) + v.y * fmaf(d, sc[1].Q[1][lo], sc[1].P[1][lo]);
              a_lya[sl] +=
                  v.x * fmaf(d, sc[0].Q[2][lo], sc[0].P[2][lo]) + v.y * fmaf(d, sc[1].Q[2][lo], sc[1].P[2][lo]);
            });
      }
    } else if constexpr (G > 2) {
      if (g == 2) {
        agn_unit(tile, 0, a_agn0);
      } else if constexpr (G > 3) {
        agn_unit(tile, 1, a_agn1);
      }
    }
    // the tile is consumed (generic reads ordered before the tensor load that refills it)
    fence_proxy_async_smem();
    __syncthreads();
  }
  if (!waited && threadIdx.x % 32 == 0) atomicExch(err, 1u);
#pragma unroll
  for (int sl = 0; sl < V; ++sl) {
    const size_t ic = row * N + last_pos<PL>(t, sl);
    sums[ic] = make_float4(a_heat[sl], a_ion[sl], a_lya[sl], a_star[sl]);
    if constexpr (G > 2) agn_heat[ic] = make_float2(a_agn0[sl], G > 3 ? a_agn1[G > 3 ? sl : 0] : 0.f);
  }
}

// the per-cell update (ComputeTs.c:1171-1407) from the shell sums; sums == nullptr: no light
__global__ void __launch_bounds__(256) k_ts_evolve(const TsDev* __restrict__ gC, TsEvolve e, double4 inv_scale, int n,
                                                   const float4* __restrict__ sums,
                                                   const float2* __restrict__ agn_heat,
                                                   const float* __restrict__ deltax, float* __restrict__ xe_prev,
                                                   float* __restrict__ xe_box, float* __restrict__ Tk,
                                                   float* __restrict__ TS, double* __restrict__ partials,
                                                   int* __restrict__ nonconv) {
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
      double sm[4] = {0.0, 0.0, 0.0, 0.0};
      if (sums) {
        const float4 v = __ldg(sums + ir);
        sm[0] = (double)v.x * inv_scale.x;
        sm[1] = (double)v.y * inv_scale.y;
        sm[2] = (double)v.z * inv_scale.z;
        sm[3] = (double)v.w * inv_scale.w;
      }
      float xn, tk, ts;
      const float xe0 = xe_prev[ip];
      if (agn_heat) {
        // the AGN heating terms of dT_K/dz (XRayHeatingFunctions.c:1519-1520) for their averages
        const float2 a = __ldg(agn_heat + ir);
        const double f = inv_scale.x * e.const_zp * e.heat_conv / (1.0 + (double)xe0);
        acc[7] += (double)a.x * f;
        acc[8] += (double)a.y * f;
      }
      evolve_cell(C, e, __ldg(deltax + ip), xe0, Tk[ir], sm, &xn, &tk, &ts, acc, &nc);
      xe_prev[ip] = xn;
      xe_box[ip] = xn;
      Tk[ir] = tk;
      TS[ir] = ts;
    }
  if (nc) atomicAdd(nonconv, nc);
  block_sum_dyn<TS_NSUM>(acc, partials + (size_t)blockIdx.x * TS_NSUM);
}

// homogeneous branch (ComputeTs.c:252-278) and the closing averages (:1459-1494)
__global__ void __launch_bounds__(256) k_ts_homog(const TsDev* __restrict__ gC, float xe0, float TK0,
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
      const float ts = get_Ts(C, delta, tk, xe0, 0.f, &xa, &nc);
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

// The combination of a shell that reads more than TS_MAXSRC history slots:
// spec[spare][g] = sum_i cs[i] spec[ks[i]][g] for every grid g, accumulated with fmaf in the order
// of i as the x pass does (1 x value is exact, so the shell's x pass then reads the same numbers).
// Sources go in chunks of TS_COMB; later chunks continue from the partial sums.
constexpr int TS_COMB = 32;
struct TsComb {
  int n;
  int first;   // the chunk starts the sums (else it adds to the spare slot)
  int ks[TS_COMB];
  float cs[TS_COMB];
};

__global__ void __launch_bounds__(256) k_ts_combine(cf* __restrict__ spec, size_t stride, int G, TsComb cb,
                                                    int spare) {
  const size_t total = stride * (size_t)G;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const size_t g = e / stride, i = e - g * stride;
    cf* out = spec + ((size_t)spare * G + g) * stride + i;
    float ax = 0.f, ay = 0.f;
    if (!cb.first) {
      ax = out->x;
      ay = out->y;
    }
    for (int k = 0; k < cb.n; ++k) {
      const cf v = spec[((size_t)cb.ks[k] * G + g) * stride + i];
      ax = fmaf(cb.cs[k], v.x, ax);
      ay = fmaf(cb.cs[k], v.y, ay);
    }
    *out = cf{ax, ay};
  }
}

static int ts_combine(rg_context* ctx, int n, cf* spec, size_t stride, int G, const std::vector<int>& ks,
                      const std::vector<float>& cs, int spare, cudaStream_t st) {
  (void)n;
  const int blocks = 4 * ctx->num_sms;
  for (size_t i0 = 0; i0 < ks.size(); i0 += TS_COMB) {
    TsComb cb;
    std::memset(&cb, 0, sizeof(cb));
    cb.first = i0 == 0;
    cb.n = (int)std::min((size_t)TS_COMB, ks.size() - i0);
    for (int k = 0; k < cb.n; ++k) {
      cb.ks[k] = ks[i0 + k];
      cb.cs[k] = cs[i0 + k];
    }
    prof_begin(ctx, "ts_combine_sources", st);
    k_ts_combine<<<blocks, 256, 0, st>>>(spec, stride, G, cb, spare);
    prof_end(ctx, 8.0 * stride * G * (cb.n + (cb.first ? 1 : 2)), st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  return RG_OK;
}

// x and y passes of a batch of shells: work_base + (j * bt.ng + g) * stride, j < bt.nr.  (The
// fused x/y kernel of find_HII_bubbles, run on these batches, measured slower at 512^3: 48.8 ms
// against 43.5 ms for the two passes; the x pass here reads its history spectra mostly from L2.)
template <int N>
static int launch_ts_xy(rg_context* ctx, const cf* spec, cf* work_base, size_t stride, const TsBatch& bt,
                        const float* wtab, int wpitch, const int* wcut, cudaStream_t st) {
  using C = Cfg<N>;
  const double nzc = (double)C::NZ * N * N;
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  const size_t smx = sizeof(cf) * (N + (size_t)line_buf<N, C::BX>());
  RG_CUDA_TRY(ctx, cudaFuncSetAttribute(k_ts_x<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
  prof_begin(ctx, "ts_x_c2c_combine_window", st);
  k_ts_x<N><<<dim3(N / C::BX, C::NZ), C::T * C::BX, smx, st>>>(spec, stride, work_base, bt, wtab, wpitch, wcut, tw);
  double src_reads = 0;
  for (int r = 0; r < bt.nr; ++r) src_reads += bt.nk[r];
  prof_end(ctx, bt.ng * 8.0 * nzc * (src_reads + bt.nr), st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  prof_begin(ctx, "ts_y_c2c", st);
  RG_CUDA_TRY(ctx, (launch_pass_y<N, true>(work_base, stride, bt.ng * bt.nr, tw, st)));
  prof_end(ctx, bt.ng * bt.nr * 16.0 * nzc, st);
  return RG_OK;
}

// the z pass over all nS shells: per-cell shell sums
template <int N, int G>
static int launch_ts_zsum_g(rg_context* ctx, const cf* work, size_t stride, const TsShellCoef* d_co, const TsZev& zv,
                            const float* xe_prev, float4* sums, float2* agn_heat, cudaStream_t st) {
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  using Z = TsZ<N>;
  const double n3 = (double)N * N * N, nzc = (double)(N / 2 + 1) * N * N;
  if (stride != (size_t)Z::NZ * N * N) return set_error(ctx, RG_EINVAL, "Ts z pass: shell spectra must be contiguous");
  // every shell's G spectra (S[kz][x][y], one after another) as a 3-D float tensor
  CUtensorMap tmap;
  const uint64_t dims[3] = {2ull * N, (uint64_t)N, (uint64_t)Z::NZ * zv.nS * G};
  const uint64_t strides[2] = {8ull * N, 8ull * N * N};
  const uint32_t box[3] = {2u * Z::Q, 1u, (uint32_t)Z::KZB};
  const int mrc = tma_map_3d(&tmap, work, dims, strides, box);
  if (mrc != 0) return set_error(ctx, RG_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(mrc) + ")");
  const size_t smz = Z::smem();
  RG_CUDA_TRY(ctx, cudaFuncSetAttribute(k_ts_zsum<N, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smz));
  prof_begin(ctx, "ts_z_c2r_sums", st);
  k_ts_zsum<N, G><<<dim3(N / Z::Q, N), Z::NTH, smz, st>>>(tmap, tw, d_co, zv, xe_prev, sums, agn_heat, ctx->xy_ctrl);
  // Hermitian halves of the G grids of every shell, x_e read, four float sums (and the AGN
  // heating pair) written
  prof_end(ctx, zv.nS * G * 8.0 * nzc + 4.0 * n3 + 16.0 * n3 + (G > 2 ? 8.0 * n3 : 0.0), st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

template <int N>
static int launch_ts_zsum(rg_context* ctx, const cf* work, size_t stride, int ng, const TsShellCoef* d_co,
                          const TsZev& zv, const float* xe_prev, float4* sums, float2* agn_heat, cudaStream_t st) {
  if (ng == 2) return launch_ts_zsum_g<N, 2>(ctx, work, stride, d_co, zv, xe_prev, sums, nullptr, st);
  if (ng == 3) return launch_ts_zsum_g<N, 3>(ctx, work, stride, d_co, zv, xe_prev, sums, agn_heat, st);
  return launch_ts_zsum_g<N, 4>(ctx, work, stride, d_co, zv, xe_prev, sums, agn_heat, st);
}

#define RG_TS_DISPATCH(n, call)                                                           \
  switch (n) {                                                                            \
    case 8: { constexpr int NN = 8; return call; }                                        \
    case 16: { constexpr int NN = 16; return call; }                                      \
    case 32: { constexpr int NN = 32; return call; }                                      \
    case 64: { constexpr int NN = 64; return call; }                                      \
    case 128: { constexpr int NN = 128; return call; }                                    \
    case 256: { constexpr int NN = 256; return call; }                                    \
    case 512: { constexpr int NN = 512; return call; }                                    \
    default: return set_error(ctx, RG_EUNSUPPORTED, "ComputeTs needs a power-of-two ReionGridDim"); \
  }

static int ts_xy(rg_context* ctx, int n, const cf* spec, cf* work_base, size_t stride, const TsBatch& bt,
                 const float* wtab, int wpitch, const int* wcut, cudaStream_t st) {
  RG_TS_DISPATCH(n, launch_ts_xy<NN>(ctx, spec, work_base, stride, bt, wtab, wpitch, wcut, st));
}

static int ts_zsum(rg_context* ctx, int n, const cf* work, size_t stride, int ng, const TsShellCoef* d_co,
                   const TsZev& zv, const float* xe_prev, float4* sums, float2* agn_heat, cudaStream_t st) {
  RG_TS_DISPATCH(n, launch_ts_zsum<NN>(ctx, work, stride, ng, d_co, zv, xe_prev, sums, agn_heat, st));
}

static double pow2_scale(double maxabs) {
  if (!(maxabs > 0) || !std::isfinite(maxabs)) return 1.0;
  return std::ldexp(1.0, -std::ilogb(maxabs));
}

int ts_snapshot(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g, rg_ts_scalars* out,
                const rg_grids* src_host, const Staging* stg) {
  int rc;
  const Staging none;
  if (!stg) stg = &none;
  bool kicked = false;
  auto kick = [&]() -> int {
    if (kicked || !stg->after_sources) return RG_OK;
    kicked = true;
    return stg->after_sources();
  };
  cudaStream_t st = ctx->stream;
  const int N = ctx->N;
  const size_t n3 = (size_t)N * N * N;
  const Cosmo cm(p);
  const Units u = make_units(p);
  const double zp = s->ZZ[s->snapshot];
  const double box_size = p->BoxSize / p->Hubble_h;  // Mpc
  const double pixel_volume = std::pow(box_size / (double)N, 3);
  std::memset(out, 0, sizeof(*out));
  // grids per shell: sfr, X-ray, then the AGN bands in use (0 soft, 1 hard)
  const int agn_flag = p->Flag_IncludeAGNXray;
  int bands[2] = {-1, -1}, nagn = 0;
  if (agn_flag == 1 || agn_flag == 3) bands[nagn++] = 0;
  if (agn_flag == 1 || agn_flag == 2) bands[nagn++] = 1;
  const int G = 2 + nagn;

  // device constants: kappa splines and number densities
  TsDev hc;
  std::memset(&hc, 0, sizeof(hc));
  fill_spline(ctx->tables.k10, ctx->tables.k10_lT, ctx->tables.k10_lk, &hc.k10);
  fill_spline(ctx->tables.kel, ctx->tables.kel_lT, ctx->tables.kel_lk, &hc.kel);
  fill_spline(ctx->tables.kpH, ctx->tables.kpH_lT, ctx->tables.kpH_lk, &hc.kpH);
  hc.max_iter = ctx->ts_iter_limit;
  {
    // per-redshift factors of xcoll / taugp / xalpha_tilde / dT_comp / evolveInt; the C passes
    // the redshift to them as a float
    const float zf = (float)zp;
    const double z = (double)zf;
    TsZConst& Z = hc.z;
    Z.Trad = TCMB * (1.0 + z);
    Z.inv_Trad = 1.0 / Z.Trad;
    const double opz3 = std::pow(1.0 + z, 3.0);
    Z.xc_H = T21 / Z.Trad * cm.No * opz3 / A10_HYPERFINE;
    Z.xc_e = T21 / Z.Trad * cm.N_b0 * opz3 / A10_HYPERFINE;
    Z.xc_p = Z.xc_H;
    Z.tgp0 = 1.342881e-7 / cm.hubble(zf) * cm.No * opz3;
    Z.xa0 = 1.66e11 / (1.0 + z);
    Z.nb0 = cm.N_b0 * std::pow((double)(1.0f + zf), 3);
    Z.comp0 = (-1.51e-4) / (cm.hubble(zf) / (HUBBLE * p->Hubble_h)) / p->Hubble_h * std::pow(Z.Trad, 4.0) / (1.0 + z);
    Z.dadia0 = 3 / (1.0 + z);
    Z.f_H = cm.f_H;
    Z.f_He = cm.f_He;
  }
  // device constants, the non-convergence counter and the per-shell coefficients live in one
  // context buffer: [TsDev][int + pad][TsShellCoef x shells]
  const int nS_all = p->TsNumFilterSteps;
  const size_t off_co = (sizeof(TsDev) + 16 + 255) / 256 * 256;
  if ((rc = ensure_device(ctx, &ctx->ts_const, &ctx->ts_const_elems, off_co + sizeof(TsShellCoef) * (nS_all + 1))))
    return rc;
  TsDev* d_hc = reinterpret_cast<TsDev*>(ctx->ts_const);
  int* d_nonconv = reinterpret_cast<int*>(ctx->ts_const + sizeof(TsDev));
  TsShellCoef* d_co = reinterpret_cast<TsShellCoef*>(ctx->ts_const + off_co);
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(d_hc, &hc, sizeof(TsDev), cudaMemcpyHostToDevice, st));
  RG_CUDA_TRY(ctx, cudaMemsetAsync(d_nonconv, 0, sizeof(int), st));
  const int nblk = 148 * 8;
  double* partials = ensure_partials(ctx, (size_t)nblk * TS_NSUM);
  if (!partials) return set_error(ctx, RG_ENOMEM, "partials");

  const double R0 = L_FACTOR * box_size / (float)N;
  const double Mh2 = rtom(p, R0) * p->Hubble_h * p->Hubble_h;
  const double ftpr3 = (4.0 / 3.0) * M_PI * std::pow(R0, 3.0) / pixel_volume;

  auto finish = [&](bool homog, int nblocks) -> int {
    if ((rc = kick())) return rc;
    if ((rc = reduce_partials(ctx, partials, nblocks, TS_NSUM, ctx->d_sums, st))) return rc;
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
      for (int j = 0; j < nagn; ++j)
        (bands[j] ? out->volume_ave_Xheat_AGN_hard : out->volume_ave_Xheat_AGN_soft) = S[7 + j] / nn;
    }
    out->volume_ave_TS = S[4] / nn;
    out->volume_ave_TK = S[5] / nn;
    out->volume_ave_xe = S[6] / nn;
    out->homogeneous = homog;
    if (nonconv)
      return set_error(ctx, RG_ETIMEDOUT, "get_Ts did not converge in " + std::to_string(ctx->ts_iter_limit) +
                                              " iterations for some cells");
    return RG_OK;
  };

  // collapse fraction and <x_e> (both branches compute the collapse fraction)
  prof_begin(ctx, "ts_reduce0", st);
  if ((rc = stage_wait(ctx, stg->inputs, st))) return rc;
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
    if ((rc = stage_wait(ctx, stg->closing, st))) return rc;   // Tk_box is overwritten
    k_ts_homog<<<nblk, 256, 0, st>>>(d_hc, xe0, TK0, cT_approx((float)zp), N, g->deltax, g->x_e_box_prev,
                                      g->x_e_box, g->Tk_box, g->TS_box, partials, d_nonconv);
    prof_end(ctx, 28.0 * n3, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
    return finish(true, nblk);
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
  TsZev zv;
  std::memset(&zv, 0, sizeof(zv));
  for (int m = 0; m < x_int_NXHII; ++m) zv.X[m] = ctx->tables.x_int_XHII[m];
  for (int k = 0; k < 4; ++k) zv.inv_scale[k] = 1.0;

  if (!no_light) {
    if (!s->stored_fcoll && s->snapshot > 0)
      return set_error(ctx, RG_EINVAL, "ComputeTs needs stored_fcoll of the previous snapshot");
    // sources used by any shell
    std::vector<int> slot_of(sh.nsrc, -1), used;
    for (int r = 0; r < nS; ++r)
      for (int k = 0; k < sh.nsrc; ++k)
        if (sh.coef[(size_t)r * sh.nsrc + k] != 0.f && slot_of[k] < 0) {
          slot_of[k] = (int)used.size();
          used.push_back(k);
        }
    // a shell that combines more than TS_MAXSRC history snapshots gets its combination formed
    // beforehand (k_ts_combine) into one of TS_KB spare slots after the used sources
    bool wide = false;
    for (int r = 0; r < nS; ++r) {
      int nk = 0;
      for (int k = 0; k < sh.nsrc; ++k) nk += sh.coef[(size_t)r * sh.nsrc + k] != 0.f;
      wide = wide || nk > TS_MAXSRC;
    }
    const int nused = std::max(1, (int)used.size());
    const size_t slots = (size_t)nused + (wide ? TS_KB : 0);
    if ((rc = ensure_device(ctx, &ctx->spec, &ctx->spec_elems, nc * G * slots))) return rc;
    // every shell's filtered grids stay in HBM until the fused z pass (G nS spectra)
    if ((rc = ensure_device(ctx, &ctx->work, &ctx->work_elems, nc * G * nS))) return rc;
    // source grid `which` (0 sfr, 1 xray, 2 + j AGN band bands[j]) of source k, on the device
    // (the AGN histories are re-weighted like the sfr ones, load_reion_bh_grids)
    const rg_grids* sg = src_host ? src_host : g;
    auto src_grid = [&](int k, int which) -> const float* {
      if (which >= 2) {
        const bool hard = bands[which - 2] == 1;
        if (k == 0) return hard ? sg->bh_xray_hard : sg->bh_xray_soft;
        return (hard ? sg->bh_xray_histories_hard : sg->bh_xray_histories_soft) + (size_t)(k - 1) * npad;
      }
      if (k == 0) return which ? sg->xray_luminosity : sg->sfr;
      return (which ? sg->xray_luminosity_histories : sg->sfr_histories) + (size_t)(k - 1) * npad;
    };
    if (src_host && (rc = ensure_device(ctx, &ctx->ts_stage, &ctx->ts_stage_elems, npad * G * used.size()))) return rc;
    auto dev_grid = [&](size_t j, int which) -> const float* {
      return src_host ? ctx->ts_stage + (j * G + which) * npad : src_grid(used[j], which);
    };
    // window rows for the shells (filter() takes BoxSize in Mpc/h and R in Mpc, ComputeTs.c:532)
    const int n2max = 3 * (N / 2) * (N / 2);
    if ((rc = ensure_device(ctx, &ctx->d_radii, &ctx->d_radii_elems, (size_t)nS))) return rc;
    RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_radii, sh.R.data(), sizeof(double) * nS, cudaMemcpyHostToDevice, st));
    if ((rc = ensure_device(ctx, &ctx->wtab, &ctx->wtab_elems, (size_t)nS * (n2max + 1)))) return rc;
    if ((rc = ensure_device(ctx, &ctx->wcut, &ctx->wcut_elems, (size_t)nS))) return rc;
    if ((rc = window_table(ctx, p->BoxSize, ctx->d_radii, nS, p->TsHeatingFilterType, ctx->wtab, n2max, st,
                           ctx->wcut)))
      return rc;
    const int* wcut = p->TsHeatingFilterType == 1 ? ctx->wcut : nullptr;

    // Batches of TS_KB shells: the forward transforms of the sources a batch uses first (`used`
    // is in order of first use), then its x and y passes into work[r][g].  From host arrays,
    // each group of sources is copied on the copy stream and its transform waits for the copy,
    // so the copies of later sources overlap the passes of earlier batches.
    size_t next_slot = 0;   // used[0, next_slot) are transformed into spec[slot * G + g]
    for (int r0 = 0; r0 < nS; r0 += TS_KB) {
      const int cnt = std::min(TS_KB, nS - r0);
      size_t need = next_slot;
      for (int r = r0; r < r0 + cnt; ++r)
        for (int k = 0; k < sh.nsrc; ++k)
          if (sh.coef[(size_t)r * sh.nsrc + k] != 0.f) need = std::max(need, (size_t)slot_of[k] + 1);
      while (next_slot < need) {
        const size_t end = std::min(need, next_slot + (size_t)(MAXG / G));
        if (src_host) {
          for (size_t j = next_slot; j < end; ++j)
            for (int which = 0; which < G; ++which)
              RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->ts_stage + (j * G + which) * npad, src_grid(used[j], which),
                                               sizeof(float) * npad, cudaMemcpyHostToDevice, ctx->copy_stream));
          cudaEvent_t e;
          if ((rc = stage_record(ctx, 4 + next_slot, ctx->copy_stream, &e))) return rc;
          if ((rc = stage_wait(ctx, e, st))) return rc;
        }
        const float* srcs[MAXG];
        int ng = 0;
        for (size_t j = next_slot; j < end; ++j)
          for (int which = 0; which < G; ++which) srcs[ng++] = dev_grid(j, which);
        if ((rc = fft_forward(ctx, N, srcs, ng, ctx->spec + nc * G * next_slot, nc, 1.0 / std::pow((double)N, 3), st)))
          return rc;
        next_slot = end;
      }
      TsBatch bt;
      std::memset(&bt, 0, sizeof(bt));
      bt.nr = cnt;
      bt.ng = G;
      for (int j = 0; j < cnt; ++j) {
        const int r = r0 + j;
        std::vector<int> ks;
        std::vector<float> cs;
        for (int k = 0; k < sh.nsrc; ++k) {
          const float c = sh.coef[(size_t)r * sh.nsrc + k];
          if (c != 0.f) {
            ks.push_back(slot_of[k]);
            cs.push_back(c);
          }
        }
        if ((int)ks.size() > TS_MAXSRC) {
          // spare slot nused + j holds sum_i cs[i] spec[ks[i]], accumulated in the x pass's order
          const int spare = nused + j;
          if ((rc = ts_combine(ctx, N, ctx->spec, nc, G, ks, cs, spare, st))) return rc;
          ks.assign(1, spare);
          cs.assign(1, 1.f);
        }
        const int nk = (int)ks.size();
        for (int i = 0; i < nk; ++i) {
          bt.ks[j][i] = ks[i];
          bt.cs[j][i] = cs[i];
        }
        bt.nk[j] = nk;
        bt.filtered[j] = r > 0;  // no filter on the first shell (ComputeTs.c:529)
        bt.wrow[j] = r;
      }
      if ((rc = ts_xy(ctx, N, ctx->spec, ctx->work + (size_t)r0 * G * nc, nc, bt, ctx->wtab, n2max + 1, wcut, st)))
        return rc;
    }
    if ((rc = kick())) return rc;
    // the frequency tables on the host while the device runs the transforms above
    TsTables tb;
    std::string msg;
    if ((rc = ts_tables(p, ctx->tables, sh, zp, x_e_ave, collapse_fraction, s->ZZ, s->stored_fcoll, s->snapshot, &tb,
                        &msg)))
      return set_error(ctx, rc, msg);

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
    // AGN bands: XAGN_R = max(bh, 0) 1e10 L_sun / pv UL^-3 (ComputeTs.c:615-630), the band's
    // (1+zpp)^-alpha and tables, and const_zp_AGN / const_zp_GAL so the terms share the
    // galaxies' prefactor in the update kernel (XRayHeatingFunctions.c:1420-1470)
    const double convA = 1e10 * SOLAR_LUM / pixel_volume * std::pow(p->UnitLength_in_cm, -3.0);
    std::vector<double> PAd((size_t)nS * 2 * 3 * x_int_NXHII, 0.0), QAd(PAd.size(), 0.0);
    for (int j = 0; j < nagn; ++j) {
      const int b = bands[j];
      const double alpha_b = b ? p->SpecIndexXrayAGNHard : p->SpecIndexXrayAGNSoft;
      const double ratio = pf.const_zp_prefactor_AGN[b] / pf.const_zp_prefactor_GAL;
      for (int r = 0; r < nS; ++r) {
        const double a = sh.dt_dzpp[r] * sh.dzpp[r] * convA * std::pow(1 + sh.zpp[r], -alpha_b) * ratio;
        for (int kind = 0; kind < 3; ++kind) {
          const std::vector<double>& tb_k = tb.agn[b][kind];
          for (int m = 0; m < x_int_NXHII; ++m) {
            const double t_lo = tb_k[(size_t)m * nS + r];
            const double t_hi = m + 1 < x_int_NXHII ? tb_k[(size_t)(m + 1) * nS + r] : t_lo;
            const double slope = m + 1 < x_int_NXHII ? (t_hi - t_lo) / ((double)X[m + 1] - (double)X[m]) : 0.0;
            const size_t o = (((size_t)r * 2 + j) * 3 + kind) * x_int_NXHII + m;
            PAd[o] = a * t_lo;
            QAd[o] = a * slope;
            maxk[kind] = std::max({maxk[kind], std::fabs(a * t_lo), std::fabs(a * t_hi)});
          }
        }
      }
    }
    // FP32 sums over the shells: scale each sum by a power of two that brings its largest
    // per-shell coefficient near 1 (values of order 1e-30 would lose range in float)
    double scale[4];
    for (int k = 0; k < 4; ++k) {
      scale[k] = pow2_scale(maxk[k]);
      zv.inv_scale[k] = 1.0 / scale[k];
    }
    std::vector<TsShellCoef> hco(nS + 1);
    std::memset(hco.data(), 0, sizeof(TsShellCoef) * hco.size());
    for (int r = 0; r < nS; ++r) {
      for (int kind = 0; kind < 3; ++kind)
        for (int m = 0; m < x_int_NXHII; ++m) {
          hco[r].P[kind][m] = (float)(Pd[((size_t)r * 3 + kind) * x_int_NXHII + m] * scale[kind]);
          hco[r].Q[kind][m] = (float)(Qd[((size_t)r * 3 + kind) * x_int_NXHII + m] * scale[kind]);
        }
      hco[r].cstar = (float)(cs[r] * scale[3]);
      for (int j = 0; j < nagn; ++j)
        for (int kind = 0; kind < 3; ++kind)
          for (int m = 0; m < x_int_NXHII; ++m) {
            const size_t o = (((size_t)r * 2 + j) * 3 + kind) * x_int_NXHII + m;
            hco[r].PA[j][kind][m] = (float)(PAd[o] * scale[kind]);
            hco[r].QA[j][kind][m] = (float)(QAd[o] * scale[kind]);
          }
    }
    RG_CUDA_TRY(ctx, cudaMemcpyAsync(d_co, hco.data(), sizeof(TsShellCoef) * (nS + 1), cudaMemcpyHostToDevice, st));
    zv.nS = nS;
    if ((rc = ensure_device(ctx, &ctx->ts_sums, &ctx->ts_sums_elems, n3))) return rc;
    if (nagn && (rc = ensure_device(ctx, &ctx->ts_agn, &ctx->ts_agn_elems, n3))) return rc;
    if ((rc = xy_ctrl_reset(ctx, 0, st))) return rc;   // the error word of the tile waits
    if ((rc = ts_zsum(ctx, N, ctx->work, nc, G, d_co, zv, g->x_e_box_prev, ctx->ts_sums, nagn ? ctx->ts_agn : nullptr,
                      st)))
      return rc;
    RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));  // hco outlives the copy
    if ((rc = xy_ctrl_check(ctx, st))) return rc;
  }

  TsEvolve e;
  e.zp = zp;
  e.dzp = zp - prev_redshift;
  e.dt_dzp = pf.dt_dzp;
  e.heat_conv = pf.dt_dzp * 2.0 / 3.0 / BOLTZMANN;
  e.growth = pf.growth_factor_zp;
  e.dgrowth = pf.dgrowth_factor_dzp;
  e.const_zp = pf.const_zp_prefactor_GAL;
  // Conversion_factor (XRayHeatingFunctions.c:1331-1332)
  e.conv_star = (SPEED_OF_LIGHT / (4. * M_PI)) / (PROTONMASS / SOLAR_MASS);
  e.no_light = no_light;
  const double4 inv = make_double4(zv.inv_scale[0], zv.inv_scale[1], zv.inv_scale[2], zv.inv_scale[3]);
  prof_begin(ctx, "ts_evolve", st);
  if ((rc = stage_wait(ctx, stg->closing, st))) return rc;
  k_ts_evolve<<<nblk, 256, 0, st>>>(d_hc, e, inv, N, no_light ? nullptr : ctx->ts_sums,
                                     (no_light || !nagn) ? nullptr : ctx->ts_agn, g->deltax, g->x_e_box_prev,
                                     g->x_e_box, g->Tk_box, g->TS_box, partials, d_nonconv);
  prof_end(ctx, (double)n3 * (16 + 4 + 4 + 4 + 4 + 4 + 4 + 4), st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return finish(false, nblk);
}

}  // namespace rg
