// Excursion-set step (_find_HII_bubbles, src/core/find_HII_bubbles.c:86-710) on sm_100a.
//
// Per snapshot: one forward r2c of each grid the barrier test reads (deltax, stars, [x_e],
// [effective_bhm]); then the filter radii in batches of KB:
//   x pass : each block loads its spectrum tile once and writes KB windowed, x-transformed
//            copies (one per radius of the batch)
//   y pass : in place over the KB x G work grids
//   z pass : per block of rows, for each radius of the batch in order: c2r of the G grids into
//            shared memory, then the aliasing clamp and the barrier test per cell.
// Until the last radius the per-cell state is two bits (ionized this snapshot; z_at_ionization
// still < 0), kept in registers within a batch and in one byte per cell between batches;
// z_at_ionization and J_21 are written only where a cell first ionizes.  The last radius also
// computes the partial xH and runs the closing pass (temperatures and FP64 global sums).
#include <cuda_runtime.h>
#include <math.h>

#include <cstdio>
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

#include "rg_internal.h"
#include "rg_pass.cuh"
#include "rg_tma.cuh"
#include "rg_xyf.cuh"

namespace rg {

// ---------------------------------------------------------------------------
// window table W[r][n2], n2 = nx^2 + ny^2 + nz^2, evaluated in double from the closed
// forms of filter() (src/core/reionization.c:3404-3428)

// sharp-k: k R 0.413566994 > 1 zeroes the mode
__device__ __forceinline__ bool sharpk_zero(double delta_k, int n2, double R) {
  const double kR = delta_k * sqrt((double)n2) * R;
  return kR * 0.413566994 > 1.0;
}

// For the sharp-k filter (ftype 1) the row is a step in n2 (kR grows with n2); wcut[r], when
// given, receives the last n2 of the step (written by that entry alone), so
// W[r][n2] == (n2 <= wcut[r]).
__global__ void k_window_table(float* wtab, int n2max, const double* __restrict__ radii, int nr, double delta_k,
                               int ftype, int* wcut) {
  const int r = blockIdx.y;
  if (r >= nr) return;
  const double R = radii[r];
  for (int n2 = blockIdx.x * blockDim.x + threadIdx.x; n2 <= n2max; n2 += gridDim.x * blockDim.x) {
    const double kR = delta_k * sqrt((double)n2) * R;
    double w = 1.0;
    if (ftype == 0) {
      if (kR > 1e-4) w = 3.0 * (sin(kR) / (kR * kR * kR) - cos(kR) / (kR * kR));
    } else if (ftype == 1) {
      if (sharpk_zero(delta_k, n2, R)) w = 0.0;
    } else {
      const double g = kR * 0.643;
      w = exp(-g * g / 2.0);
    }
    wtab[(size_t)r * (n2max + 1) + n2] = (float)w;
    if (ftype == 1 && wcut && w == 1.0 && (n2 == n2max || sharpk_zero(delta_k, n2 + 1, R))) wcut[r] = n2;
  }
}


// ---------------------------------------------------------------------------
// inverse x pass with the window and a batch of radii: grid g of spec (spec + g * stride) is
// read once per block; radius r of the batch is written to work + (r * ng + g) * stride.
// Radius r uses window row wrows + r * wpitch, or none when r == unfiltered.

template <int N>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::BX, (x_pass_minb<N>()))
    k_hii_x(const cf* __restrict__ spec, size_t stride, int ng, cf* __restrict__ work, int nr,
            const float* __restrict__ wrows, int wpitch, int unfiltered, const cf* __restrict__ g_tw) {
  constexpr int T = Cfg<N>::T, B = Cfg<N>::BX, V = Cfg<N>::V;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  const int kz = blockIdx.y;
  const int b = threadIdx.x % B, t = threadIdx.x / B;
  const int y = blockIdx.x * B + b;
  const size_t col = (size_t)kz * N * N + y;
  load_twiddles<N>(s_tw, g_tw);
  // |k|^2 index of each register slot: nx from the position, ny from the column
  int n2[V];
  const int ny = y > N / 2 ? y - N : y;
#pragma unroll
  for (int sl = 0; sl < V; ++sl) {
    const int p = stage0_pos<N>(t, sl);
    const int nx = p > N / 2 ? p - N : p;
    n2[sl] = nx * nx + ny * ny + kz * kz;
  }
  __syncthreads();
  // Radius outer, grid inner: the window gathers (scattered 4-byte reads of the table) are
  // shared by all grids; a grid's spectrum tile is read from HBM at the first radius and
  // from L1/L2 after that.
  for (int r = 0; r < nr; ++r) {
    float wv[V];
    if (r == unfiltered) {
#pragma unroll
      for (int sl = 0; sl < V; ++sl) wv[sl] = 1.f;
    } else {
      const float* wr = wrows + (size_t)r * wpitch;
#pragma unroll
      for (int sl = 0; sl < V; ++sl) wv[sl] = __ldg(wr + n2[sl]);
    }
    for (int g = 0; g < ng; ++g) {
      const cf* src = spec + g * stride;
      cf* dst = work + ((size_t)r * ng + g) * stride;
      line_fft<N, true>(
          t, xbuf, s_tw,
          [&](int p, int sl) {
            const cf v = src[col + (size_t)p * N];
            return cf{v.x * wv[sl], v.y * wv[sl]};
          },
          [&](int p) { return line_addr<N, B>(p, b); }, [&](int p, cf v) { dst[col + (size_t)p * N] = v; });
    }
  }
}

// ---------------------------------------------------------------------------
// the barrier test

__device__ __forceinline__ float partial_T(float t_hi, float res_xh) {
  // ComputePartiallyIoinizedTemperature (find_HII_bubbles.c:76-84)
  if (res_xh <= 0.f) return (float)T_RE;
  if (res_xh >= 1.f) return t_hi;
  return (float)((double)(t_hi * res_xh) + T_RE * (1.0 - (double)res_xh));
}

__device__ float fully_ionized_T(float z_re, float z, float delta) {
  // ComputeFullyIoinizedTemperature (find_HII_bubbles.c:48-74), with its float/double mix
  float result, delta_re;
  if (fabs((double)(z - z_re)) < 1e-4) {
    result = 1.f;
  } else {
    delta_re = (float)((double)delta * (1.0 + (double)z) / (1.0 + (double)z_re));
    if (delta_re <= -1.f) delta_re = (float)(-1.0 + (double)ABS_TOL);
    if (delta <= -1.f) delta = (float)(-1.0 + (double)ABS_TOL);
    result = (float)pow((1.0 + (double)delta) / (1.0 + (double)delta_re), 1.1333);
    result = (float)((double)result * pow((1.0 + (double)z) / (1.0 + (double)z_re), 3.4));
    result *= expf((float)(pow((1.0 + (double)z) / 7.1, 2.5) - pow((1.0 + (double)z_re) / 7.1, 2.5)));
  }
  result = (float)((double)result * pow(T_RE, 1.7));
  result = (float)((double)result + pow(1e4 * ((1.0 + (double)z) / 4.0), 1.7) * (double)(1.f + delta));
  result = (float)pow((double)result, 0.5882);
  return result;
}

// Block sum of K doubles per thread into out[0..K), deterministic order.
template <int NTH, int K>
__device__ __forceinline__ void block_sum(double (&acc)[K], double* out) {
  if constexpr (NTH % 32 == 0) {
    __shared__ double s_red[NTH / 32][K];
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
      for (int w = 0; w < NTH / 32; ++w) v += s_red[w][threadIdx.x];
      out[threadIdx.x] = v;
    }
  } else {
    __shared__ double s_red[NTH][K];
#pragma unroll
    for (int i = 0; i < K; ++i) s_red[threadIdx.x][i] = acc[i];
    __syncthreads();
    if (threadIdx.x < K) {
      double v = 0.0;
      for (int w = 0; w < NTH; ++w) v += s_red[w][threadIdx.x];
      out[threadIdx.x] = v;
    }
  }
}

struct HiiBatch {
  int nr;             // radii in this batch
  int first;          // the batch starts the snapshot (state comes from z_at_ionization)
  int ng;             // grids per radius (read by the instantiation for 5 to 7 grids)
  double fcoll_pref[KB_MAX];
  float J_aux[KB_MAX], J_aux_bh[KB_MAX];
  float G_pref[KB_MAX], G_pref_bh[KB_MAX], R[KB_MAX];   // recombination branch
  double fcoll_prefIII[KB_MAX];                          // Pop III (mini-halos)
  float J_auxIII[KB_MAX], G_prefIII[KB_MAX];
};

struct HiiState {
  float* xH;
  float* z_in;
  float* J21;
  float* temp;
  const float* Tk_box;
  const float* deltax_unf;   // padded
  const float* wsfr;         // padded
  const float* bhar;         // padded, may be null
  const float* wsfrIII;      // padded, Pop III only
  float* Gamma12;            // recombination branch: written at a cell's first crossing
  float* r_bubble;
  uint8_t* st8;              // per cell between radius batches: bit 0 = z_at_ionization still < 0,
                             // bit 1 = ionised at a radius of this snapshot
  double* partials;          // [nblocks][HII_NSUM]
};

// Shared-memory plan of the z pass: ZB tile buffers of TB complex each; the buffer of the unit
// being transformed is also its FFT exchange buffer (the tile is consumed by the first stage).
// Two buffers let the next grid's tile arrive while this one is transformed.  At 512^3 the
// batches before the last use one buffer instead, which brings a block to 72 KB and 77 registers
// and the SM to three blocks (measured: 46.0 -> 44.0 ms over 7 batches; the closing batch, with
// more registers, keeps two buffers).
template <int N, bool FINAL>
struct HiiZ {
  static constexpr int NTH = Cfg<N>::T * Cfg<N>::QZ;
  static constexpr bool WIDE = N == 512 && !FINAL;
  static constexpr int ZB = WIDE ? 1 : 2;
  static constexpr int TB = round_up(cmax((int)ztile_elems<N>(), line_buf<N, Cfg<N>::QZ>()), 2);
  static constexpr int MINB = WIDE ? 3 : RG_MINB(NTH);
  static constexpr size_t smem(int ng) {
    return sizeof(cf) * (size_t)N + sizeof(float) * (size_t)round_up(ng * 2 * Cfg<N>::QZ * Cfg<N>::RT_PITCH, 4) +
           sizeof(cf) * (size_t)ZB * TB;
  }
};

// z pass of a batch.  FINAL: the batch ends with the snapshot's last (unfiltered) radius.
// Grids in rt: 0 deltax, 1 stars, then x_e (spin temperature), then effective_bhm (BH), then
// starsIII (Pop III), then with recombinations N_rec, weighted_sfr, effective_bhar (BH) and
// weighted_sfrIII (Pop III).  NG is the number of grids; the EXT instantiation (recombinations or
// Pop III) takes any count up to NG from bt.ng.
template <int N, int NG, bool FINAL, bool EXT>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::QZ, (HiiZ<N, FINAL>::MINB))
    k_hii_z(const cf* __restrict__ work, size_t stride, const cf* __restrict__ g_tw, HiiBatch bt, HiiConst c,
            HiiState s) {
  constexpr int T = Cfg<N>::T, Q = Cfg<N>::QZ, NTH = T * Q, ROWS = 2 * Q, RP = Cfg<N>::RT_PITCH;
  constexpr int PADW = 2 * (N / 2 + 1);
  constexpr int IT = ROWS * N / NTH;   // cells per thread
  constexpr int W = (IT + 31) / 32;    // bit words per thread
  static_assert(ROWS * N % NTH == 0, "whole rows per block");
  extern __shared__ __align__(16) unsigned char smem_raw[];  // 16-byte aligned for cp.async
  cf* smem = reinterpret_cast<cf*>(smem_raw);
  constexpr int ZB = HiiZ<N, FINAL>::ZB, TB = HiiZ<N, FINAL>::TB;
  cf* s_tw = smem;
  float* rt = reinterpret_cast<float*>(smem + N);
  // ZB shared tiles (with two, grid u + 1 is copied while grid u is transformed); the tile of
  // unit u is the exchange buffer of its transform
  // (the EXT instantiation lays the tiles out after the row buffers of the grids it has)
  cf* tiles = reinterpret_cast<cf*>(rt + round_up((EXT ? bt.ng : NG) * ROWS * RP, 4));
  const int x = blockIdx.y, y0 = blockIdx.x * ROWS;
  const size_t blk = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
  load_twiddles<N>(s_tw, g_tw);

  // per-cell state bits: A = z_at_ionization still < 0, I = ionized at a radius of this snapshot.
  // Cell it of this thread is block cell threadIdx.x + it * NTH, bit it % 32 of word it / 32;
  // between batches the state is one byte per cell (s.st8, bit 0 = A, bit 1 = I).
  uint32_t A[W], I[W];
#pragma unroll
  for (int w = 0; w < W; ++w) {
    uint32_t a = 0u, iv = 0u;
    const int nb = IT - 32 * w < 32 ? IT - 32 * w : 32;
#pragma unroll 8
    for (int bb = 0; bb < nb; ++bb) {
      const int i = threadIdx.x + (32 * w + bb) * NTH;
      const size_t ir = ((size_t)x * N + y0 + i / N) * N + i % N;
      if (bt.first) {
        if (s.z_in[ir] < 0.f) a |= 1u << bb;
      } else {
        const uint32_t v = s.st8[ir];
        a |= (v & 1u) << bb;
        iv |= ((v >> 1) & 1u) << bb;
      }
    }
    A[w] = a;
    I[w] = iv;
  }
  // the Pop III and recombination grids (only the 9-grid instantiation runs with them, so the
  // others compile without those branches)
  const int ng = EXT ? bt.ng : NG;
  const bool rec = EXT && c.rec, mini = EXT && c.mini;
  int gi = 2;
  const int gx = c.spin ? gi++ : -1;
  const int gb = c.bh ? gi++ : -1;
  const int gm = mini ? gi++ : -1;                 // starsIII
  const int gn = rec ? gi++ : -1;                  // N_rec
  const int gw = rec ? gi++ : -1;                  // weighted_sfr
  const int gr = rec && c.bh ? gi++ : -1;          // effective_bhar
  const int gw3 = rec && mini ? gi++ : -1;         // weighted_sfrIII
  double acc[FINAL ? HII_NSUM : 1];
#pragma unroll
  for (int k = 0; k < (FINAL ? HII_NSUM : 1); ++k) acc[k] = 0.0;

  const int nunits = bt.nr * ng;   // (radius, grid) pairs, unit u = r * ng + g
  ztile_issue<N, Q>(tiles, work, x, y0, NTH);
  cp_async_commit();
  const int q = threadIdx.x % Q, tq = threadIdx.x / Q;
  for (int r = 0; r < bt.nr; ++r) {
    __syncthreads();  // rt of the previous radius is consumed
#pragma unroll 1
    for (int g = 0; g < ng; ++g) {
      const int u = r * ng + g;
      cf* tile = tiles + (ZB == 2 ? (u & 1) : 0) * TB;
      if constexpr (ZB == 2) {
        if (u + 1 < nunits) ztile_issue<N, Q>(tiles + ((u + 1) & 1) * TB, work + (size_t)(u + 1) * stride, x, y0, NTH);
        cp_async_commit();
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();  // unit u's tile is complete for every thread
      float* r0 = rt + (size_t)(g * ROWS + 2 * q) * RP;
      line_fft<N, true>(
          tq, tile, s_tw, [&](int p, int) { return ztile_c2r_input<N, Q>(tile, q, p); },
          [&](int p) { return line_addr<N, Q>(p, q); },
          [&](int p, cf v) {
            r0[p] = v.x;
            r0[RP + p] = v.y;
          });
      __syncthreads();  // the tile is consumed before it is refilled; rt row is written
      if constexpr (ZB == 1) {
        if (u + 1 < nunits) ztile_issue<N, Q>(tiles, work + (size_t)(u + 1) * stride, x, y0, NTH);
        cp_async_commit();
      }
    }
    const bool last = FINAL && r == bt.nr - 1;
    const double pref = bt.fcoll_pref[r];
#pragma unroll
    for (int w = 0; w < W; ++w) {
      uint32_t a = A[w], iw = I[w];
      const int nb = IT - 32 * w < 32 ? IT - 32 * w : 32;
#pragma unroll 4
      for (int bb = 0; bb < nb; ++bb) {
        const int i = threadIdx.x + (32 * w + bb) * NTH;
        const int z = i % N, row = i / N;
        const uint32_t bit = 1u << bb;
        const float dx = fmaxf(rt[row * RP + z], -1.f + REL_TOL);
        float st = fmaxf(rt[(ROWS + row) * RP + z], 0.f);
        if (st < ABS_TOL) st = 0.f;
        float xe = 0.f, bhm = 0.f;
        if (gx >= 0) {
          xe = fmaxf(rt[(gx * ROWS + row) * RP + z], 0.f);
          if (xe < ABS_TOL) xe = 0.f;
          xe = fminf(xe, 0.999f);
        }
        if (gb >= 0) {
          bhm = fmaxf(rt[(gb * ROWS + row) * RP + z], 0.f);
          if (bhm < ABS_TOL) bhm = 0.f;
        }
        float stIII = 0.f;
        if (gm >= 0) {
          stIII = fmaxf(rt[(gm * ROWS + row) * RP + z], 0.f);
          if (stIII < ABS_TOL) stIII = 0.f;
        }
        float nrec = 0.f;
        if (gn >= 0) {
          nrec = fmaxf(rt[(gn * ROWS + row) * RP + z], 0.f);
          if (nrec < ABS_TOL) nrec = 0.f;
        }
        const double dom = 1.0 + (double)dx;  // >= 1e-5 after the clamp
        const double nf = c.spin ? 1.0 - (double)xe : 1.0;
        const double rec = gn >= 0 ? (double)nrec / dom : 0.0;
        // (f_bh + f_stars) * prefactor > nf (1 + rec) with f = grid / dom, tested with both
        // sides times dom: the two forms differ only within a few FP64 ulps of the barrier
        const double num = c.bh ? (double)bhm + (double)st : (double)st;
        const double prefIII = gm >= 0 ? bt.fcoll_prefIII[r] : 0.0;
        const double lhs_dom = gm >= 0 ? num * pref + (double)stIII * prefIII : num * pref;
        const bool ion = lhs_dom > nf * (1.0 + rec) * dom;
        float xH = (iw & bit) ? 0.f : 1.f;   // so far: 0 once ionized at a radius, else 1
        const size_t cellrow = (size_t)x * N + y0 + row;
        const size_t ir = cellrow * N + z;
        float temp_new = -1.f;               // >= 0: partial temperature written this radius
        if (ion) {
          if (gn >= 0 && !(iw & bit)) {
            // first crossing of the snapshot (find_HII_bubbles.c:488-508)
            float wsf = fmaxf(rt[(gw * ROWS + row) * RP + z], 0.f);
            if (wsf < ABS_TOL) wsf = 0.f;
            float G = __fmul_rn(wsf, bt.G_pref[r]);
            if (gw3 >= 0) {
              float w3 = fmaxf(rt[(gw3 * ROWS + row) * RP + z], 0.f);
              if (w3 < ABS_TOL) w3 = 0.f;
              G = __fadd_rn(G, __fmul_rn(w3, bt.G_prefIII[r]));
            }
            if (gr >= 0) {
              float bhr = fmaxf(rt[(gr * ROWS + row) * RP + z], 0.f);
              if (bhr < ABS_TOL) bhr = 0.f;
              G = __fadd_rn(G, __fmul_rn(bhr, bt.G_pref_bh[r]));
            }
            s.Gamma12[ir] = G;
            s.r_bubble[ir] = bt.R[r];
            if (c.uvb == 2) {
              float j = __fmul_rn(st, bt.J_aux[r]);
              if (gm >= 0) j = __fadd_rn(j, __fmul_rn(stIII, bt.J_auxIII[r]));
              if (c.bh) j = __fadd_rn(j, __fmul_rn(bhm, bt.J_aux_bh[r]));
              s.J21[ir] = j;
            }
          }
          xH = 0.f;
          iw |= bit;
        } else if (last && xH > REL_TOL) {
          // partially ionized: temperature of the neutral gas, xH = nf - f_coll prefactor
          float thi;
          if (c.spin) {
            thi = s.Tk_box[ir];
          } else {
            const float du = s.deltax_unf[cellrow * PADW + z];
            thi = (float)((double)c.TK * (1.0 + (double)(c.cT_ad * du)));
          }
          temp_new = partial_T(thi, xH);
          const double fcs = (double)st / dom;
          const double fbh = c.bh ? (double)bhm / dom : 0.0;
          const double lhs = (fbh + fcs) * pref;
          float v = (float)(nf - lhs);
          if (gm >= 0) v -= (float)((double)stIII / dom * prefIII);   // a float subtraction in the C
          xH = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
        }
        float zin_new = -1.f;                // > -1: set this radius
        if (xH < REL_TOL && (a & bit)) {
          // new ionization (find_HII_bubbles.c:531-543)
          a &= ~bit;
          zin_new = c.redshift;
          s.z_in[ir] = zin_new;
          if (c.uvb == 1) {
            float j = st * bt.J_aux[r];
            if (gm >= 0) j = __fadd_rn(j, __fmul_rn(stIII, bt.J_auxIII[r]));
            if (c.bh) j += bhm * bt.J_aux_bh[r];
            s.J21[ir] = j;
          }
        }
        if (FINAL && last) {
          // closing pass (find_HII_bubbles.c:577-645)
          const size_t ip = cellrow * PADW + z;
          s.xH[ir] = xH;
          const float du = s.deltax_unf[ip];
          const double domu = 1.0 + (double)du;
          float temp = temp_new >= 0.f ? temp_new : s.temp[ir];
          if (xH < REL_TOL) {
            const float zin = zin_new > -1.f ? zin_new : s.z_in[ir];
            if (zin > 0.f) temp = fully_ionized_T(zin, c.redshift, du);
          }
          if (c.spin) {
            const float tk = s.Tk_box[ir];
            if (temp < tk) temp = tk;
          } else {
            const float thistk = (float)((double)c.TK * (1.0 + (double)(c.cT_ad * du)));
            if (temp < thistk) temp = thistk;
          }
          s.temp[ir] = temp;
          acc[0] += (double)xH;
          // acc[1] and acc[6]: r_bubble is written only on the recombination branch
          // (find_HII_bubbles.c:490-508); its sums come from k_hii_recomb.
          acc[2] += (double)s.wsfr[ip];
          if (s.bhar != nullptr) acc[3] += (double)s.bhar[ip];
          if (s.wsfrIII != nullptr) acc[9] += (double)s.wsfrIII[ip];
          acc[4] += (double)temp;
          acc[5] += (double)xH * domu;
          acc[7] += (double)temp * domu;
          acc[8] += domu;
        }
      }
      A[w] = a;
      I[w] = iw;
    }
  }

  if constexpr (!FINAL) {
#pragma unroll
    for (int w = 0; w < W; ++w) {
      const int nb = IT - 32 * w < 32 ? IT - 32 * w : 32;
#pragma unroll 8
      for (int bb = 0; bb < nb; ++bb) {
        const int i = threadIdx.x + (32 * w + bb) * NTH;
        const size_t ir = ((size_t)x * N + y0 + i / N) * N + i % N;
        s.st8[ir] = (uint8_t)(((A[w] >> bb) & 1u) | (((I[w] >> bb) & 1u) << 1));
      }
    }
  } else {
    block_sum<NTH, HII_NSUM>(acc, s.partials + blk * HII_NSUM);
  }
}

// deterministic second stage: one block sums the per-block partials in a fixed order
__global__ void k_reduce_partials(const double* __restrict__ partials, int nblocks, int nsum, double* out) {
  __shared__ double sh[256];
  for (int i = 0; i < nsum; ++i) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 256) v += partials[(size_t)b * nsum + i];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[i] = sh[0];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// launchers

// ---------------------------------------------------------------------------
// recombinations in the closing pass (find_HII_bubbles.c:612-644)

struct RecConst {
  double redshift;     // ZZ[snapshot]
  double hubble_h;
  float fabs_dtdz;     // |dt/dz| / h at the snapshot, float as in the reference
  float zstep;         // ZZ[snapshot - 1] - ZZ[snapshot] (0 at snapshot 0)
  int temp_dep;        // Flag_TemperatureDependentRec
};

struct RecState {
  const float* xH;
  const float* temp;         // temp_kinetic_all_gas after the closing pass
  const float* deltax_unf;   // padded
  const float* r_bubble;
  const float* Gamma12;
  float* N_rec;              // padded
  float* residual_xH;
  float* clumping_factor;
  float* t_resp;
};

constexpr int REC_NSUM = 10;   // r_bubble, Gamma12, N_rec, residual_xH, clumping: volume and mass
constexpr int REC_NT = 256;

// splined_recombination (recombinations.c:35-84): the (z, T) row by rounding to the nearest
// sample, then the natural cubic spline in ln Gamma12 of that row.  The sample spacings are
// the float constants of recombinations.h:17-34.
__device__ void splined_recombination(const RecTables& t, double z_eff, double gamma12, double temp, double* rate,
                                      double* rnh, double* cf) {
  int z_ct = (int)((z_eff - (double)0.0f) / (double)0.2f + 0.5);
  int t_ct = (int)((log10(temp) - (double)2.0f) / (double)0.03f + 0.5);
  double lng = log(gamma12);
  if (z_ct < 0)
    z_ct = 0;
  else if (z_ct >= t.nz)
    z_ct = t.nz - 1;
  if (t_ct < 0 || !(lng >= t.lng_lo)) {
    *rate = 0.0;
    *rnh = 1e4;
    *cf = 1.0;
    return;
  }
  if (t_ct >= t.nt) t_ct = t.nt - 1;
  if (lng >= t.lng_hi) lng = t.lng_hi - 1e-7;   // FRACT_FLOAT_ERR
  // interval lo with knots[lo] <= lng < knots[lo + 1]
  int lo = 0, hi = t.ng - 1;
  while (hi > lo + 1) {
    const int mid = (lo + hi) >> 1;
    if (t.knots[mid] > lng)
      hi = mid;
    else
      lo = mid;
  }
  const double xlo = t.knots[lo];
  const double h = t.knots[lo + 1] - xlo, dx = lng - xlo;
  const size_t rows = (size_t)t.nz * t.nt;
  const size_t row = (size_t)z_ct * t.nt + t_ct;
  double v[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const size_t o = ((size_t)k * rows + row) * t.ng + lo;
    const double yl = t.y[o], yh = t.y[o + 1], cl = t.c[o], ch = t.c[o + 1];
    const double b = (yh - yl) / h - h * (ch + 2.0 * cl) / 3.0;
    const double d = (ch - cl) / (3.0 * h);
    v[k] = yl + dx * (b + dx * (cl + dx * d));
  }
  *rate = exp(v[0]);
  *cf = v[1];
  *rnh = exp(v[2]);
}

template <int N>
__global__ void __launch_bounds__(REC_NT) k_hii_recomb(RecTables tab, RecConst c, RecState s, double* partials) {
  constexpr int PADW = 2 * (N / 2 + 1);
  const size_t n3 = (size_t)N * N * N;
  double acc[REC_NSUM];
#pragma unroll
  for (int k = 0; k < REC_NSUM; ++k) acc[k] = 0.0;
  for (size_t ir = (size_t)blockIdx.x * REC_NT + threadIdx.x; ir < n3; ir += (size_t)gridDim.x * REC_NT) {
    const size_t ip = ir / N * PADW + ir % N;
    const float xHf = s.xH[ir];
    const double dom = 1.0 + (double)s.deltax_unf[ip];
    const double z_eff = (1.0 + c.redshift) * pow(dom, 1.0 / 3.0) - 1.0;
    const double temp = c.temp_dep ? (double)s.temp[ir] : 1e4;
    const float G = s.Gamma12[ir];
    const double gh = __dmul_rn(__dmul_rn((double)G, c.hubble_h), c.hubble_h);
    double rate, rnh, cf;
    splined_recombination(tab, z_eff, gh, temp, &rate, &rnh, &cf);
    // N_rec += (float)rate * fabs_dtdz * zstep * (1 - xH): a float product, widened
    const float f = __fmul_rn(__fmul_rn((float)rate, c.fabs_dtdz), c.zstep);
    const float nrec = (float)__dadd_rn((double)s.N_rec[ip], __dmul_rn((double)f, 1.0 - (double)xHf));
    s.N_rec[ip] = nrec;
    const float rnhf = (float)rnh, cff = (float)cf;
    s.residual_xH[ir] = rnhf;
    s.clumping_factor[ir] = cff;
    // t_resp = 1 / (Gamma + rate) in Myr, stored as float first (find_HII_bubbles.c:630-635)
    float tr = (float)__dadd_rn(__dmul_rn(gh, 1e-12), rate);
    tr = tr > 0.f ? (float)(1.0 / (double)tr / SEC_PER_MEGAYEAR) : 1e30f;
    s.t_resp[ir] = tr;
    const double rb = (double)s.r_bubble[ir];
    acc[0] += rb;
    acc[1] += rb * dom;
    acc[2] += (double)G;
    acc[3] += (double)G * dom;
    acc[4] += (double)nrec;
    acc[5] += (double)nrec * dom;
    acc[6] += (double)rnhf;
    acc[7] += (double)rnhf * dom;
    acc[8] += (double)cff;
    acc[9] += (double)cff * dom;
  }
  block_sum<REC_NT, REC_NSUM>(acc, partials + (size_t)blockIdx.x * REC_NSUM);
}

template <int N>
int launch_hii_recomb(rg_context* ctx, const RecTables& tab, const RecConst& c, const RecState& s, double* partials,
                      int nblocks, cudaStream_t st) {
  prof_begin(ctx, "hii_recomb", st);
  k_hii_recomb<N><<<nblocks, REC_NT, 0, st>>>(tab, c, s, partials);
  // xH, temperature, deltax, r_bubble, Gamma12 read; N_rec read and written; three outputs
  prof_end(ctx, 40.0 * (double)N * N * N, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

template <typename K>
static cudaError_t prep(K kernel, size_t smem) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int N>
constexpr size_t smem_x() { return sizeof(cf) * (N + (size_t)line_buf<N, Cfg<N>::BX>()); }

template <int N>
int launch_forward(rg_context* ctx, const float* const* d_real, int ng, cf* spec, size_t stride, double scale,
                   cudaStream_t st) {
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  using C = Cfg<N>;
  GridPtrs src{};
  for (int g = 0; g < ng; ++g) src.p[g] = d_real[g];
  const double nzc = (double)C::NZ * N * N;
  using ZF = ZFCfg<N>;
  RG_CUDA_TRY(ctx, prep(k_fwd_z<N>, ZF::smem()));
  prof_begin(ctx, "fwd_z_r2c", st);
  k_fwd_z<N><<<dim3(N / (2 * ZF::QF), N, ng), ZF::NTH, ZF::smem(), st>>>(src, spec, stride, tw);
  prof_end(ctx, ng * (4.0 * N * N * N + 8.0 * nzc), st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  prof_begin(ctx, "fwd_y_c2c", st);
  RG_CUDA_TRY(ctx, (launch_pass_y<N, false>(spec, stride, ng, tw, st)));
  prof_end(ctx, ng * 16.0 * nzc, st);
  RG_CUDA_TRY(ctx, prep(k_pass_x_fwd<N>, smem_x<N>()));
  prof_begin(ctx, "fwd_x_c2c", st);
  k_pass_x_fwd<N><<<dim3(N / C::BX, C::NZ, ng), C::T * C::BX, smem_x<N>(), st>>>(spec, stride, tw, (float)scale);
  prof_end(ctx, ng * 16.0 * nzc, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}


// f(std::integral_constant<int, I>{}) for I in the sequence, in order
template <class F, int... I>
__device__ __forceinline__ void for_each_index(std::integer_sequence<int, I...>, F&& f) {
  (f(std::integral_constant<int, I>{}), ...);
}

// ---------------------------------------------------------------------------
// z pass of a batch before the last one (no recombination or Pop III grid), with the tiles staged
// by TMA and the barrier test on the transforms' registers.
//
// The block owns rows [y0, y0 + 2Q) of plane x.  For every (radius, grid) unit u of the batch, the
// Hermitian half column tile (all kz, those rows) arrives in shared memory by tensor loads (ZB
// tiles in flight, one mbarrier each); the c2r of its row pairs leaves each thread the same cells
// of every grid (the transform's output positions do not depend on the grid), so the previous
// grids' values are kept in registers and the clamp and barrier test run as the last grid's
// values come out of the transform: no row buffer in shared memory.  The state of a cell
// (z_at_ionization still < 0; ionised at a radius of this snapshot) is two bits in registers
// within the batch and one byte per cell between batches.
template <int N>
struct HiiZR {
  static constexpr int T = Cfg<N>::T, Q = Cfg<N>::QZ, NTH = T * Q, V = N / T;
  static constexpr int NZ = N / 2 + 1;
  // kz rows per tensor box (box dimensions are at most 256): one box, or for N = 512 two boxes of
  // (NZ + 1) / 2 rows at kz 0 and kz NZ - KZB that overlap in one row, so the second box lands on
  // a 128-byte boundary of the tile and no row lies outside the tensor
  static constexpr int KZB = NZ <= 256 ? NZ : (NZ + 1) / 2;
  static constexpr int NBOX = NZ <= 256 ? 1 : 2;
  static constexpr int TB = round_up(cmax(NZ * 2 * Q, line_buf<N, Q>()), 16);   // 128-byte multiple
  static constexpr int ZB = 3;                                 // tiles in flight
  static constexpr uint32_t TX = (uint32_t)(NBOX * KZB * 2 * Q * sizeof(cf));   // bytes the boxes deliver
  static_assert(NBOX == 1 || ((NZ - KZB) * 2 * Q * sizeof(cf)) % 128 == 0, "second box off a 128-byte boundary");
  static constexpr size_t smem() { return 128 + sizeof(cf) * ((size_t)ZB * TB + N) + sizeof(uint64_t) * ZB; }
  // resident blocks: register room for the kept grids (up to 3 x 2V floats) without spills; the
  // closing batch also holds ten FP64 sums (three blocks still fit at 512^3)
  template <bool FINAL>
  static constexpr int minb() { return FINAL ? (NTH >= 256 ? 1 : (N >= 512 ? 3 : 2)) : (NTH >= 256 ? 2 : 3); }
  // the sizes it serves: power-of-two grids of 64^3 and up (at most 16 values per thread)
  static constexpr bool USED = (N == 64 || N == 128 || N == 256 || N == 512);
  static_assert(2 * V <= 64, "two state bits per cell in 64-bit masks");
};

constexpr int TMA_WAIT_LIMIT = 1 << 22;   // polls of an mbarrier before a wait gives up

// FINAL: the batch ends with the snapshot's last (unfiltered) radius: the partial xH of the
// never-ionised cells, and the closing pass (temperatures, xH, FP64 sums into partials) as in
// k_hii_z.
template <int N, bool SPIN, bool BH, bool FINAL>
__global__ void __launch_bounds__(HiiZR<N>::NTH, (HiiZR<N>::template minb<FINAL>()))
    k_hii_zr(const __grid_constant__ CUtensorMap tmap, const cf* __restrict__ g_tw, HiiBatch bt, HiiConst c,
             HiiState s, uint32_t* err) {
  using Z = HiiZR<N>;
  using PL = Plan<N>;
  constexpr int Q = Z::Q, V = Z::V, ZB = Z::ZB, TB = Z::TB, NZ = Z::NZ, KZB = Z::KZB, NBOX = Z::NBOX;
  constexpr int PADW = 2 * (N / 2 + 1);
  constexpr int NG = 2 + SPIN + BH;          // deltax, stars, [x_e], [effective_bhm]
  constexpr int GX = 2, GB = 2 + SPIN;       // grid indices of x_e and effective_bhm
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  cf* tiles = reinterpret_cast<cf*>(sm);
  cf* s_tw = tiles + ZB * TB;
  uint64_t* bars = reinterpret_cast<uint64_t*>(s_tw + N);
  const int x = blockIdx.y, y0 = blockIdx.x * 2 * Q;
  const int q = threadIdx.x % Q, tq = threadIdx.x / Q;
  const int nunits = bt.nr * NG;

  if (threadIdx.x == 0) {
    for (int b = 0; b < ZB; ++b) mbar_init(&bars[b], 1);
    mbar_init_fence();
  }
  load_twiddles<N>(s_tw, g_tw);
  __syncthreads();
  // thread 0: tensor loads of unit u into tile u % ZB (tensor coordinates: y in floats, x, kz of
  // the unit's spectrum stacked after the previous units)
  auto issue = [&](int u) {
    const int b = u % ZB;
    mbar_arrive_expect_tx(&bars[b], Z::TX);
#pragma unroll
    for (int k = 0; k < NBOX; ++k) {
      const int k0 = k ? NZ - KZB : 0;
      tma_load_3d(tiles + b * TB + k0 * 2 * Q, &tmap, 2 * y0, x, u * NZ + k0, &bars[b]);
    }
  };
  if (threadIdx.x == 0)
    for (int u = 0; u < ZB && u < nunits; ++u) issue(u);

  // state of this thread's 2V cells: cell 2 slot + h is row y0 + 2q + h at z = last_pos(tq, slot)
  uint64_t A = 0, I = 0, P = 0;   // P: partly ionised at the closing radius
#pragma unroll
  for (int slot = 0; slot < V; ++slot) {
    const int z = last_pos<PL>(tq, slot);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const size_t ir = ((size_t)x * N + y0 + 2 * q + h) * N + z;
      const uint64_t bit = 1ull << (2 * slot + h);
      if (bt.first) {
        if (s.z_in[ir] < 0.f) A |= bit;
      } else {
        const uint32_t v = s.st8[ir];
        if (v & 1u) A |= bit;
        if (v & 2u) I |= bit;
      }
    }
  }

  const uint64_t A0 = A;
  float vals[NG - 1][2 * V];   // the transformed grids before the last one, for the radius in work
  double acc[FINAL ? HII_NSUM : 1];
#pragma unroll
  for (int k = 0; k < (FINAL ? HII_NSUM : 1); ++k) acc[k] = 0.0;
  bool waited = true;
  int u = 0;
  for (int r = 0; r < bt.nr; ++r) {
    const double pref = bt.fcoll_pref[r];
    const float jaux = bt.J_aux[r], jaux_bh = bt.J_aux_bh[r];
    const bool lastr = FINAL && r == bt.nr - 1;
    // one (radius, grid) unit; the grid index is a compile-time constant (register arrays)
    auto unit = [&](auto gconst) {
      constexpr int g = decltype(gconst)::value;
      const int b = u % ZB;
      cf* tile = tiles + b * TB;
      if (!mbar_wait(&bars[b], (uint32_t)((u / ZB) & 1), TMA_WAIT_LIMIT)) waited = false;
      line_fft_p<PL, true>(
          tq, tile, s_tw, [&](int p, int) { return ztile_c2r_input<N, Q>(tile, q, p); },
          [&](int p) { return line_addr<N, Q>(p, q); },
          [&](int z, cf v, int slot) {
            if constexpr (g < NG - 1) {
              vals[g][2 * slot] = v.x;
              vals[g][2 * slot + 1] = v.y;
            } else {
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                const float last = h ? v.y : v.x;
                auto val = [&](auto gi) -> float {
                  constexpr int gg = decltype(gi)::value;
                  if constexpr (gg == NG - 1) return last;
                  else return vals[gg][2 * slot + h];
                };
                // the aliasing clamp (find_HII_bubbles.c:373-422) and the barrier test of
                // k_hii_z without recombinations or Pop III
                const float dx = fmaxf(val(std::integral_constant<int, 0>{}), -1.f + REL_TOL);
                float st = fmaxf(val(std::integral_constant<int, 1>{}), 0.f);
                if (st < ABS_TOL) st = 0.f;
                float xe = 0.f, bhm = 0.f;
                if constexpr (SPIN) {
                  xe = fmaxf(val(std::integral_constant<int, GX>{}), 0.f);
                  if (xe < ABS_TOL) xe = 0.f;
                  xe = fminf(xe, 0.999f);
                }
                if constexpr (BH) {
                  bhm = fmaxf(val(std::integral_constant<int, GB>{}), 0.f);
                  if (bhm < ABS_TOL) bhm = 0.f;
                }
                const double dom = 1.0 + (double)dx;
                const double nf = SPIN ? 1.0 - (double)xe : 1.0;
                const double num = BH ? (double)bhm + (double)st : (double)st;
                const bool ion = num * pref > nf * (1.0 + 0.0) * dom;
                const uint64_t bit = 1ull << (2 * slot + h);
                const size_t cellrow = (size_t)x * N + y0 + 2 * q + h;
                const size_t ir = cellrow * N + z;
                float xH = (I & bit) ? 0.f : 1.f;   // so far: 0 once ionized at a radius, else 1
                if (ion) {
                  I |= bit;
                  xH = 0.f;
                } else if (lastr && xH > REL_TOL) {
                  // partially ionized: xH = nf - f_coll prefactor; its temperature is that of the
                  // neutral gas (the closing pass below)
                  P |= bit;
                  const double fcs = (double)st / dom;
                  const double fbh = BH ? (double)bhm / dom : 0.0;
                  const float v = (float)(nf - (fbh + fcs) * pref);
                  xH = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
                }
                if (xH < REL_TOL && (A & bit)) {
                  // new ionization (find_HII_bubbles.c:531-543)
                  A &= ~bit;
                  s.z_in[ir] = c.redshift;
                  if (c.uvb == 1) {
                    float j = st * jaux;
                    if (BH) j += bhm * jaux_bh;
                    s.J21[ir] = j;
                  }
                }
                // the cell's deltax is used: its register keeps the final xH for the closing pass
                if constexpr (FINAL) {
                  if (lastr) vals[0][2 * slot + h] = xH;
                }
              }
            }
          });
      // every thread is done with tile b (read by the first stage, exchange buffer after that):
      // order those generic accesses before the tensor load that refills it
      fence_proxy_async_smem();
      __syncthreads();
      if (threadIdx.x == 0 && u + ZB < nunits) issue(u + ZB);
      ++u;
    };
    for_each_index(std::make_integer_sequence<int, NG>{}, unit);
  }
  if (!waited && threadIdx.x % 32 == 0) atomicExch(err, 1u);
  if constexpr (FINAL) {
    // closing pass (find_HII_bubbles.c:577-645) of this thread's cells, four slots at a time with
    // their loads issued together.  z_at_ionization is this snapshot's redshift where this batch
    // set it (A0 & ~A), else it is read (not written by this kernel).  A partly ionised cell's
    // temperature, ComputePartiallyIoinizedTemperature of the neutral gas's T at residual xH 1,
    // is that T: Tk_box with the spin temperature, else the adiabatic T; the floor is the same T.
    constexpr int CH = 4;
#pragma unroll
    for (int s0 = 0; s0 < V; s0 += CH) {
      float du[2 * CH], tk[2 * CH], tp[2 * CH], zi[2 * CH], ws[2 * CH], bh[2 * CH];
#pragma unroll
      for (int j = 0; j < 2 * CH; ++j) {
        const int slot = s0 + j / 2, h = j % 2;
        const uint64_t bit = 1ull << (2 * slot + h);
        const size_t cellrow = (size_t)x * N + y0 + 2 * q + h;
        const int z = last_pos<PL>(tq, slot);
        const size_t ir = cellrow * N + z, ip = cellrow * PADW + z;
        const float xH = vals[0][2 * slot + h];
        du[j] = s.deltax_unf[ip];
        ws[j] = s.wsfr[ip];
        bh[j] = s.bhar != nullptr ? s.bhar[ip] : 0.f;
        tk[j] = SPIN ? s.Tk_box[ir] : 0.f;
        tp[j] = (P & bit) ? 0.f : s.temp[ir];
        zi[j] = (xH < REL_TOL && !((A0 & ~A) & bit)) ? s.z_in[ir] : c.redshift;
      }
#pragma unroll
      for (int j = 0; j < 2 * CH; ++j) {
        const int slot = s0 + j / 2, h = j % 2;
        const uint64_t bit = 1ull << (2 * slot + h);
        const size_t cellrow = (size_t)x * N + y0 + 2 * q + h;
        const size_t ir = cellrow * N + last_pos<PL>(tq, slot);
        const float xH = vals[0][2 * slot + h];
        const float tn = SPIN ? tk[j] : (float)((double)c.TK * (1.0 + (double)(c.cT_ad * du[j])));
        float temp = (P & bit) ? tn : tp[j];
        if (xH < REL_TOL && zi[j] > 0.f) temp = fully_ionized_T(zi[j], c.redshift, du[j]);
        if (temp < tn) temp = tn;
        s.xH[ir] = xH;
        s.temp[ir] = temp;
        const double domu = 1.0 + (double)du[j];
        acc[0] += (double)xH;
        acc[2] += (double)ws[j];
        acc[3] += (double)bh[j];
        acc[4] += (double)temp;
        acc[5] += (double)xH * domu;
        acc[7] += (double)temp * domu;
        acc[8] += domu;
      }
    }
    block_sum<Z::NTH, HII_NSUM>(acc, s.partials + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * HII_NSUM);
  } else {
#pragma unroll
    for (int slot = 0; slot < V; ++slot) {
      const int z = last_pos<PL>(tq, slot);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const size_t ir = ((size_t)x * N + y0 + 2 * q + h) * N + z;
        const int sh = 2 * slot + h;
        s.st8[ir] = (uint8_t)(((A >> sh) & 1ull) | (((I >> sh) & 1ull) << 1));
      }
    }
  }
}

// the batch of the fused x/y pass: grid g of spec windowed for radius r into work (r ng + g)
// The grids may be several snapshots' (ngu grids each, the same radii): the work buffer holds
// snapshot u's block [radius][its grids] at u nr ngu (one snapshot: [radius][grid]).
struct HiiXOp {
  const cf* spec;
  size_t stride;
  int ng;
  int ngu;           // grids per snapshot
  int nr;            // radii of the batch
  cf* work;
  const float* wrows;
  int wpitch;
  int unfiltered;
  const int* wcut;   // sharp-k step ends per radius, or null (window rows are read)
  __device__ int grids() const { return ng; }
  __device__ bool filtered(int r) const { return r != unfiltered; }
  __device__ const float* wrow(int r) const { return wrows + (size_t)r * wpitch; }
  __device__ int cutoff(int r) const { return wcut ? __ldg(wcut + r) : -2; }
  __device__ cf* out(int r, int g) const {
    const int u = g / ngu;
    return work + (((size_t)u * nr + r) * ngu + (g - u * ngu)) * stride;
  }
};

// inverse x (window, batch of nr radii) and y passes: one fused kernel, or (plain mode) the two
// passes as separate kernels
template <int N>
int launch_inverse_xy(rg_context* ctx, const cf* spec, int ng, int ngu, cf* work, size_t stride, int nr,
                      const float* wrows, int wpitch, int unfiltered, cudaStream_t st, const int* wcut = nullptr) {
  using C = Cfg<N>;
  const double nzc = (double)C::NZ * N * N;
  if (ctx->mode == RG_MODE_FUSED) {
    const HiiXOp op{spec, stride, ng, ngu, nr, work, wrows, wpitch, unfiltered, wcut};
    if (stride != (size_t)C::NZ * N * N) return set_error(ctx, RG_EINVAL, "fused x/y pass: spectra must be contiguous");
    return launch_xy_fused<N>(ctx, op, spec, ng, nr, "inv_xy_c2c_window", ng * 8.0 * nzc * (1 + nr), st);
  }
  if (ngu != ng) return set_error(ctx, RG_EINVAL, "several snapshots in one pass need the fused mode");
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  RG_CUDA_TRY(ctx, prep(k_hii_x<N>, smem_x<N>()));
  prof_begin(ctx, "inv_x_c2c_window", st);
  k_hii_x<N><<<dim3(N / C::BX, C::NZ), C::T * C::BX, smem_x<N>(), st>>>(spec, stride, ng, work, nr, wrows, wpitch,
                                                                        unfiltered, tw);
  prof_end(ctx, ng * 8.0 * nzc * (1 + nr), st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  prof_begin(ctx, "inv_y_c2c", st);
  RG_CUDA_TRY(ctx, (launch_pass_y<N, true>(work, stride, ng * nr, tw, st)));
  prof_end(ctx, ng * nr * 16.0 * nzc, st);
  return RG_OK;
}

// grids one EXT z pass can hold at this size: the most, up to 9, whose row buffers fit the
// 227 KB of shared memory a block may use (7 at 384^3, 8 at 192^3)
template <int N>
constexpr int hii_ngx() {
  int ng = 9;
  while (ng > 4 && HiiZ<N, true>::smem(ng) > 227 * 1024) --ng;
  return ng;
}

template <int N, int NG, bool FINAL, bool EXT = false>
int launch_hii_z3(rg_context* ctx, const cf* work, size_t stride, const HiiBatch& bt, const HiiConst& c,
                  const HiiState& s, cudaStream_t st, int* nblocks) {
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  using C = Cfg<N>;
  static_assert(HiiZ<N, FINAL>::smem(NG) <= 227 * 1024, "z pass shared memory above the per-block limit");
  // the EXT instantiation takes the shared memory of the grids it has, not of its maximum
  const size_t sm = HiiZ<N, FINAL>::smem(EXT ? bt.ng : NG);
  RG_CUDA_TRY(ctx, prep(k_hii_z<N, NG, FINAL, EXT>, HiiZ<N, FINAL>::smem(NG)));
  const dim3 grid(N / (2 * C::QZ), N);
  // algorithmic bytes: the Hermitian halves of NG grids per radius, z_at_ionization on the
  // first batch; the closing pass writes xH and temperature and reads deltax, weighted_sfr,
  // [effective_bhar], [Tk_box]
  const double n3 = (double)N * N * N, nzc = (double)C::NZ * N * N;
  double bytes = bt.nr * (EXT ? bt.ng : NG) * 8.0 * nzc + (bt.first ? 4.0 * n3 : 0.0);
  if (FINAL) bytes += 4.0 * n3 * (2 + 2 + (s.bhar != nullptr) + (s.Tk_box != nullptr));
  prof_begin(ctx, FINAL ? "inv_z_c2r_test_final" : "inv_z_c2r_test", st);
  k_hii_z<N, NG, FINAL, EXT><<<grid, C::T * C::QZ, sm, st>>>(work, stride, tw, bt, c, s);
  prof_end(ctx, bytes, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  if (nblocks) *nblocks = (int)(grid.x * grid.y);
  return RG_OK;
}

template <int N, bool SPIN, bool BH, bool FINAL>
int launch_hii_zr3(rg_context* ctx, const cf* work, const HiiBatch& bt, const HiiConst& c, const HiiState& s,
                   cudaStream_t st, int* nblocks) {
  using Z = HiiZR<N>;
  constexpr int NG = 2 + SPIN + BH;
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  // the batch's units as one 3-D float tensor: y (2N floats), x (N), kz of unit u at u NZ + kz
  CUtensorMap map;
  const uint64_t dims[3] = {2ull * N, (uint64_t)N, (uint64_t)Z::NZ * bt.nr * NG};
  const uint64_t strides[2] = {8ull * N, 8ull * N * N};
  const uint32_t box[3] = {4u * Z::Q, 1u, (uint32_t)Z::KZB};
  const int mrc = tma_map_3d(&map, work, dims, strides, box);
  if (mrc != 0) return set_error(ctx, RG_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(mrc) + ")");
  auto kern = k_hii_zr<N, SPIN, BH, FINAL>;
  RG_CUDA_TRY(ctx, prep(kern, Z::smem()));
  const dim3 grid(N / (2 * Z::Q), N);
  const double n3 = (double)N * N * N, nzc = (double)Z::NZ * N * N;
  // algorithmic bytes: the Hermitian halves of NG grids per radius, the state (z_at_ionization on
  // the first batch, one byte per cell read otherwise, one written before the closing batch); the
  // closing pass writes xH and temperature and reads deltax, weighted_sfr, [effective_bhar], the
  // temperature and [Tk_box]
  double bytes = bt.nr * NG * 8.0 * nzc + (bt.first ? 4.0 * n3 : 1.0 * n3) + (FINAL ? 0.0 : 1.0 * n3);
  if (FINAL) bytes += 4.0 * n3 * (2 + 3 + (s.bhar != nullptr) + SPIN);
  prof_begin(ctx, FINAL ? "inv_z_c2r_test_final" : "inv_z_c2r_test", st);
  kern<<<grid, Z::NTH, Z::smem(), st>>>(map, tw, bt, c, s, ctx->xy_ctrl);
  prof_end(ctx, bytes, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  if (nblocks) *nblocks = (int)(grid.x * grid.y);
  return RG_OK;
}

template <int N>
int launch_hii_z(rg_context* ctx, const cf* work, size_t stride, int ng, const HiiBatch& bt, const HiiConst& c,
                 const HiiState& s, bool fin, cudaStream_t st, int* nblocks) {
  // without recombinations or Pop III: TMA tiles, registers
  if constexpr (HiiZR<N>::USED) {
    if (!c.rec && !c.mini) {
      if (fin) {
        if (c.spin && c.bh) return launch_hii_zr3<N, true, true, true>(ctx, work, bt, c, s, st, nblocks);
        if (c.spin) return launch_hii_zr3<N, true, false, true>(ctx, work, bt, c, s, st, nblocks);
        if (c.bh) return launch_hii_zr3<N, false, true, true>(ctx, work, bt, c, s, st, nblocks);
        return launch_hii_zr3<N, false, false, true>(ctx, work, bt, c, s, st, nblocks);
      }
      if (c.spin && c.bh) return launch_hii_zr3<N, true, true, false>(ctx, work, bt, c, s, st, nblocks);
      if (c.spin) return launch_hii_zr3<N, true, false, false>(ctx, work, bt, c, s, st, nblocks);
      if (c.bh) return launch_hii_zr3<N, false, true, false>(ctx, work, bt, c, s, st, nblocks);
      return launch_hii_zr3<N, false, false, false>(ctx, work, bt, c, s, st, nblocks);
    }
  }
  // with recombinations or Pop III (up to 9 grids) one instantiation reads the count from the
  // batch
  if (c.rec || c.mini) {
    constexpr int NGX = hii_ngx<N>();
    if (ng > NGX)
      return set_error(ctx, RG_EUNSUPPORTED,
                       "this combination of grids (recombinations, Pop III, BH feedback, spin temperature) needs "
                       "more row buffers than one z pass holds at this ReionGridDim");
    return fin ? launch_hii_z3<N, NGX, true, true>(ctx, work, stride, bt, c, s, st, nblocks)
               : launch_hii_z3<N, NGX, false, true>(ctx, work, stride, bt, c, s, st, nblocks);
  }
  if (ng == 2)
    return fin ? launch_hii_z3<N, 2, true>(ctx, work, stride, bt, c, s, st, nblocks)
               : launch_hii_z3<N, 2, false>(ctx, work, stride, bt, c, s, st, nblocks);
  if (ng == 3)
    return fin ? launch_hii_z3<N, 3, true>(ctx, work, stride, bt, c, s, st, nblocks)
               : launch_hii_z3<N, 3, false>(ctx, work, stride, bt, c, s, st, nblocks);
  return fin ? launch_hii_z3<N, 4, true>(ctx, work, stride, bt, c, s, st, nblocks)
             : launch_hii_z3<N, 4, false>(ctx, work, stride, bt, c, s, st, nblocks);
}


template <int N>
int launch_debug_inverse(rg_context* ctx, const cf* spec, cf* work, const float* wrow, float* out, cudaStream_t st) {
  const size_t stride = (size_t)Cfg<N>::NZ * N * N;
  int rc = xy_ctrl_reset(ctx, Cfg<N>::NZ, st);
  if (rc) return rc;
  rc = launch_inverse_xy<N>(ctx, spec, 1, 1, work, stride, 1, wrow, 0, wrow ? -1 : 0, st);
  if (rc) return rc;
  const cf* tw;
  if ((rc = twiddles_for(ctx, N, &tw))) return rc;
  using C = Cfg<N>;
  const size_t sm = zfront_smem_bytes<N>(1);
  RG_CUDA_TRY(ctx, prep(k_inv_z_padded<N>, sm));
  k_inv_z_padded<N><<<dim3(N / (2 * C::QZ), N), C::T * C::QZ, sm, st>>>(work, tw, out);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

#define RG_DISPATCH_N(n, call)                                                   \
  switch (n) {                                                                   \
    case 8: { constexpr int NN = 8; return call; }                               \
    case 16: { constexpr int NN = 16; return call; }                             \
    case 24: { constexpr int NN = 24; return call; }                             \
    case 32: { constexpr int NN = 32; return call; }                             \
    case 48: { constexpr int NN = 48; return call; }                             \
    case 64: { constexpr int NN = 64; return call; }                             \
    case 96: { constexpr int NN = 96; return call; }                             \
    case 128: { constexpr int NN = 128; return call; }                           \
    case 192: { constexpr int NN = 192; return call; }                           \
    case 256: { constexpr int NN = 256; return call; }                           \
    case 384: { constexpr int NN = 384; return call; }                           \
    case 512: { constexpr int NN = 512; return call; }                           \
    default: return set_error(ctx, RG_EUNSUPPORTED, "ReionGridDim not in {8,16,24,32,48,64,96,128,192,256,384,512}"); \
  }

#define RG_DISPATCH_N_VAL(n, call, dflt)       \
  switch (n) {                                 \
    case 8: { constexpr int NN = 8; return call; } \
    case 16: { constexpr int NN = 16; return call; } \
    case 24: { constexpr int NN = 24; return call; } \
    case 32: { constexpr int NN = 32; return call; } \
    case 48: { constexpr int NN = 48; return call; } \
    case 64: { constexpr int NN = 64; return call; } \
    case 96: { constexpr int NN = 96; return call; } \
    case 128: { constexpr int NN = 128; return call; } \
    case 192: { constexpr int NN = 192; return call; } \
    case 256: { constexpr int NN = 256; return call; } \
    case 384: { constexpr int NN = 384; return call; } \
    case 512: { constexpr int NN = 512; return call; } \
    default: return dflt;                      \
  }

int fft_forward(rg_context* ctx, int n, const float* const* d_real, int ng, cf* spec, size_t stride, double scale,
                cudaStream_t st) {
  if (ng > MAXG) return set_error(ctx, RG_EINVAL, "too many grids in one forward launch");
  RG_DISPATCH_N(n, launch_forward<NN>(ctx, d_real, ng, spec, stride, scale, st));
}

static int inverse_xy(rg_context* ctx, int n, const cf* spec, int ng, int ngu, cf* work, size_t stride, int nr,
                      const float* wrows, int wpitch, int unfiltered, cudaStream_t st, const int* wcut) {
  RG_DISPATCH_N(n, launch_inverse_xy<NN>(ctx, spec, ng, ngu, work, stride, nr, wrows, wpitch, unfiltered, st, wcut));
}

static int hii_z(rg_context* ctx, int n, const cf* work, size_t stride, int ng, const HiiBatch& bt, const HiiConst& c,
                 const HiiState& s, bool fin, cudaStream_t st, int* nblocks) {
  RG_DISPATCH_N(n, launch_hii_z<NN>(ctx, work, stride, ng, bt, c, s, fin, st, nblocks));
}


static int hii_recomb(rg_context* ctx, int n, const RecTables& tab, const RecConst& c, const RecState& s,
                      double* partials, int nblocks, cudaStream_t st) {
  RG_DISPATCH_N(n, launch_hii_recomb<NN>(ctx, tab, c, s, partials, nblocks, st));
}

int window_table(rg_context* ctx, double box, const double* d_radii, int nr, int ftype, float* d_wtab, int n2max,
                 cudaStream_t st, int* d_wcut) {
  const double delta_k = 2.0 * M_PI / box;
  const int bx = (n2max + 1 + 255) / 256;
  if (ftype != 1) d_wcut = nullptr;
  prof_begin(ctx, "window_table", st);
  k_window_table<<<dim3(bx < 1024 ? bx : 1024, nr), 256, 0, st>>>(d_wtab, n2max, d_radii, nr, delta_k, ftype, d_wcut);
  prof_end(ctx, 4.0 * (n2max + 1) * nr, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

int reduce_partials(rg_context* ctx, const double* partials, int nblocks, int nsum, double* d_out, cudaStream_t st) {
  prof_begin(ctx, "reduce_partials", st);
  k_reduce_partials<<<1, 256, 0, st>>>(partials, nblocks, nsum, d_out);
  prof_end(ctx, 8.0 * nblocks * nsum, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

int xy_ctrl_reset(rg_context* ctx, size_t max_jobs, cudaStream_t st) {
  int rc = ensure_device(ctx, &ctx->xy_ctrl, &ctx->xy_ctrl_elems, max_jobs + 2);
  if (rc) return rc;
  RG_CUDA_TRY(ctx, cudaMemsetAsync(ctx->xy_ctrl, 0, sizeof(uint32_t), st));
  return RG_OK;
}

int xy_ctrl_check(rg_context* ctx, cudaStream_t st) {
  if (!ctx->xy_ctrl) return RG_OK;
  uint32_t err = 0;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(&err, ctx->xy_ctrl, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (err)
    return set_error(ctx, RG_ETIMEDOUT,
                     "a bounded device wait ran out (the fused x/y pass's wait for a plane, or a tensor tile's)");
  return RG_OK;
}

// ---------------------------------------------------------------------------
// the snapshot

// per-snapshot constants of the z passes
static int hii_const(rg_context* ctx, const rg_params* p, double redshift, HiiConst* c) {
  const double tk_d = T_RECFAST(ctx->tables, (float)redshift);
  if (tk_d < 0) return set_error(ctx, RG_ETABLE, "T_RECFAST called beyond its table");
  c->redshift = (float)redshift;
  c->TK = (float)tk_d;
  c->cT_ad = cT_approx((float)redshift);
  c->uvb = p->ReionUVBFlag;
  c->spin = p->Flag_IncludeSpinTemp != 0;
  c->bh = p->Flag_BHFeedback != 0;
  c->rec = p->Flag_IncludeRecombinations != 0;
  c->mini = p->UseMiniHalos != 0;
  return RG_OK;
}

// the per-radius prefactors of radii [r0, r0 + cnt) (find_HII_bubbles.c:430-450)
static void hii_batch_radii(const rg_params* p, double redshift, const std::vector<std::pair<double, bool>>& sched,
                            int r0, int cnt, int ntest, HiiBatch* bt) {
  const int N = p->ReionGridDim;
  const double pixel_volume = std::pow(p->BoxSize / (double)N, 3);
  const Units u = make_units(p);
  const double sfr_timescale = p->ReionSfrTimescale * hubble_time_at(p, redshift);
  std::memset(bt, 0, sizeof(*bt));
  bt->nr = cnt;
  bt->first = (r0 == 0);
  bt->ng = ntest;
  for (int k = 0; k < cnt; ++k) {
    const double R = sched[r0 + k].first;
    const double M_mean = rtom(p, R);
    double Gamma_R_prefactor = (1.0 + redshift) * (1.0 + redshift) * R * p->UnitLength_in_cm / pixel_volume *
                               std::pow(p->UnitLength_in_cm, -3.);
    Gamma_R_prefactor *= (p->UnitMass_in_g / u.UnitTime_in_s) / PROTONMASS * p->ReionNionPhotPerBary;
    bt->J_aux[k] = (float)(Gamma_R_prefactor * PLANCK * 1e21 / (4.0 * M_PI) * p->ReionGammaHaloBias / sfr_timescale *
                           p->ReionAlphaUV);
    bt->J_aux_bh[k] = (float)(Gamma_R_prefactor * PLANCK * 1e21 / (4.0 * M_PI) * p->ReionGammaHaloBias /
                              sfr_timescale * p->ReionAlphaUVBH);
    const double G_bh = Gamma_R_prefactor * (SIGMA_HI * p->ReionAlphaUVBH / (p->ReionAlphaUVBH + 2.75) * 1e12);
    Gamma_R_prefactor *= SIGMA_HI * p->ReionAlphaUV / (p->ReionAlphaUV + 2.75) * 1e12;
    bt->G_pref[k] = (float)Gamma_R_prefactor;
    bt->G_pref_bh[k] = (float)G_bh;
    bt->R[k] = (float)R;
    bt->fcoll_pref[k] = p->ReionEfficiency * (4.0 / 3.0) * M_PI / pixel_volume / M_mean * R * R * R;
    // Pop III (find_HII_bubbles.c:443-450): photons per baryon and efficiency of their own
    bt->J_auxIII[k] = bt->J_aux[k] * (float)(p->ReionNionPhotPerBaryIII / p->ReionNionPhotPerBary);
    bt->G_prefIII[k] = (float)(Gamma_R_prefactor * p->ReionNionPhotPerBaryIII / p->ReionNionPhotPerBary);
    bt->fcoll_prefIII[k] = bt->fcoll_pref[k] / p->ReionEfficiency * p->ReionEfficiencyIII;
  }
}

// the grids the z pass tests, in its order (the first ntest of srcs), then in the plain mode
// without recombinations weighted_sfr; returns the count.  weighted_sfr (and effective_bhar) feed
// only Gamma12 on the recombination branch, so without it their filtered fields are never read;
// the plain mode transforms weighted_sfr anyway, as the reference does.
static int hii_sources(const rg_params* p, const rg_grids* g, bool plain, const float** srcs, int* ntest) {
  const bool spin = p->Flag_IncludeSpinTemp != 0, bh = p->Flag_BHFeedback != 0;
  const bool rec = p->Flag_IncludeRecombinations != 0, mini = p->UseMiniHalos != 0;
  int ng = 0;
  srcs[ng++] = g->deltax;
  srcs[ng++] = g->stars;
  if (spin) srcs[ng++] = g->x_e_box;
  if (bh) srcs[ng++] = g->effective_bhm;
  if (mini) srcs[ng++] = g->starsIII;
  if (rec) {
    srcs[ng++] = g->N_rec;
    srcs[ng++] = g->weighted_sfr;
    if (bh) srcs[ng++] = g->effective_bhar;
    if (mini) srcs[ng++] = g->weighted_sfrIII;
  }
  *ntest = ng;
  if (plain && !rec) srcs[ng++] = g->weighted_sfr;
  return ng;
}

static HiiState hii_state(const rg_params* p, const rg_grids* g, uint8_t* st8, double* partials) {
  const bool bh = p->Flag_BHFeedback != 0, mini = p->UseMiniHalos != 0;
  HiiState hs;
  hs.xH = g->xH;
  hs.z_in = g->z_at_ionization;
  hs.J21 = g->J_21_at_ionization;
  hs.temp = g->temp_kinetic_all_gas;
  hs.Tk_box = p->Flag_IncludeSpinTemp ? g->Tk_box : nullptr;
  hs.deltax_unf = g->deltax;
  hs.wsfr = g->weighted_sfr;
  hs.bhar = bh ? g->effective_bhar : nullptr;
  hs.wsfrIII = mini ? g->weighted_sfrIII : nullptr;
  hs.Gamma12 = g->Gamma12;
  hs.r_bubble = g->r_bubble;
  hs.st8 = st8;
  hs.partials = partials;
  return hs;
}

// the box averages from the reduced sums S (find_HII_bubbles.c:650-700)
static void hii_outputs(const rg_params* p, int nr, const double* S, rg_hii_scalars* out) {
  const bool rec = p->Flag_IncludeRecombinations != 0, mini = p->UseMiniHalos != 0;
  const Units u = make_units(p);
  const double n3 = std::pow((double)p->ReionGridDim, 3);
  const double mass_weight = S[8];
  const double to_msun_yr = p->UnitMass_in_g / u.UnitTime_in_s * SEC_PER_YEAR / SOLAR_MASS;
  out->volume_weighted_global_xH = S[0] / n3;
  out->volume_weighted_global_r_bubble = S[1] / n3;
  out->volume_weighted_global_weighted_sfr = S[2] / n3 * to_msun_yr;
  out->volume_weighted_global_effective_bhar = S[3] / n3 * to_msun_yr;
  out->volume_weighted_global_temp_kinetic_all_gas = S[4] / n3;
  out->mass_weighted_global_xH = S[5] / mass_weight;
  out->mass_weighted_global_r_bubble = S[6] / mass_weight;
  out->mass_weighted_global_temp_kinetic_all_gas = S[7] / mass_weight;
  out->n_radii = nr;
  out->volume_weighted_global_weighted_sfrIII = mini ? S[9] / n3 * to_msun_yr : 0.0;
  const double* R = S + 16;   // recombination sums (find_HII_bubbles.c:666-684)
  out->volume_weighted_global_Gamma12 = rec ? R[2] / n3 : 0.0;
  out->volume_weighted_global_N_rec = rec ? R[4] / n3 : 0.0;
  out->volume_weighted_global_residual_xH = rec ? R[6] / n3 : 0.0;
  out->volume_weighted_global_clumping_factor = rec ? R[8] / n3 : 0.0;
  out->mass_weighted_global_Gamma12 = rec ? R[3] / mass_weight : 0.0;
  out->mass_weighted_global_N_rec = rec ? R[5] / mass_weight : 0.0;
  out->mass_weighted_global_residual_xH = rec ? R[7] / mass_weight : 0.0;
  out->mass_weighted_global_clumping_factor = rec ? R[9] / mass_weight : 0.0;
  if (rec) {
    out->volume_weighted_global_r_bubble = R[0] / n3;
    out->mass_weighted_global_r_bubble = R[1] / mass_weight;
  }
}

// the window table of every radius (and the sharp-k steps) into ctx->wtab / ctx->wcut
static int hii_windows(rg_context* ctx, const rg_params* p, const std::vector<std::pair<double, bool>>& sched,
                       cudaStream_t st) {
  const int N = ctx->N, nr = (int)sched.size();
  const int n2max = 3 * (N / 2) * (N / 2);
  std::vector<double> radii(nr);
  for (int i = 0; i < nr; ++i) radii[i] = sched[i].first;
  int rc;
  if ((rc = ensure_device(ctx, &ctx->d_radii, &ctx->d_radii_elems, (size_t)nr))) return rc;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_radii, radii.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, st));
  if ((rc = ensure_device(ctx, &ctx->wtab, &ctx->wtab_elems, (size_t)nr * (n2max + 1)))) return rc;
  if ((rc = ensure_device(ctx, &ctx->wcut, &ctx->wcut_elems, (size_t)nr))) return rc;
  return window_table(ctx, p->BoxSize, ctx->d_radii, nr, p->ReionFilterType, ctx->wtab, n2max, st, ctx->wcut);
}

int hii_snapshot(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g, rg_hii_scalars* out,
                 const Staging* stg) {
  const Staging none;
  if (!stg) stg = &none;
  int rc;
  cudaStream_t st = ctx->stream;
  const int N = ctx->N;
  const bool rec = p->Flag_IncludeRecombinations != 0;
  const double redshift = s->ZZ[s->snapshot];
  HiiConst c;
  if ((rc = hii_const(ctx, p, redshift, &c))) return rc;

  const float* srcs[10];
  int ntest = 0;
  const bool plain = ctx->mode == RG_MODE_PLAIN;
  const int ng = hii_sources(p, g, plain, srcs, &ntest);

  const size_t nc = (size_t)(N / 2 + 1) * N * N;
  auto sched = radius_schedule(p, redshift);
  const int nr = (int)sched.size();
  int kb = plain ? 1 : (ctx->radius_batch > 0 ? ctx->radius_batch : 8);
  if (kb > KB_MAX) kb = KB_MAX;
  if (kb > nr) kb = nr;
  if ((rc = ensure_device(ctx, &ctx->spec, &ctx->spec_elems, nc * ng))) return rc;
  if ((rc = ensure_device(ctx, &ctx->work, &ctx->work_elems, nc * ng * kb))) return rc;
  // one state byte per cell between radius batches (in words of four)
  if ((rc = ensure_device(ctx, &ctx->bits, &ctx->bits_elems, ((size_t)N * N * N + 3) / 4))) return rc;
  if ((rc = stage_wait(ctx, stg->inputs, st))) return rc;
  for (int g0 = 0; g0 < ng; g0 += MAXG)   // at most MAXG grids per forward launch
    if ((rc = fft_forward(ctx, N, srcs + g0, std::min(MAXG, ng - g0), ctx->spec + nc * g0, nc,
                          1.0 / std::pow((double)N, 3), st)))
      return rc;

  if ((rc = hii_windows(ctx, p, sched, st))) return rc;
  const int n2max = 3 * (N / 2) * (N / 2);
  const int* wcut = p->ReionFilterType == 1 ? ctx->wcut : nullptr;

  // r_bubble is only written on the recombination branch: zero it once
  RG_CUDA_TRY(ctx, cudaMemsetAsync(g->r_bubble, 0, sizeof(float) * (size_t)N * N * N, st));
  if (stg->host_r_bubble && !rec) {
    // final already: the host copy overlaps the radius loop
    cudaEvent_t e;
    if ((rc = stage_record(ctx, 4, st, &e))) return rc;
    RG_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy_stream, e, 0));
    RG_CUDA_TRY(ctx, cudaMemcpyAsync(stg->host_r_bubble, g->r_bubble, sizeof(float) * (size_t)N * N * N,
                                     cudaMemcpyDeviceToHost, ctx->copy_stream));
  }
  double* partials =
      ensure_partials(ctx, std::max((size_t)N * N * HII_NSUM, (size_t)4 * ctx->num_sms * REC_NSUM));
  if (!partials) return set_error(ctx, RG_ENOMEM, "partials");
  const HiiState hs = hii_state(p, g, reinterpret_cast<uint8_t*>(ctx->bits), partials);

  if ((rc = xy_ctrl_reset(ctx, (size_t)(N / 2 + 1) * kb, st))) return rc;
  int nblocks = 0;
  for (int r0 = 0; r0 < nr; r0 += kb) {
    const int cnt = std::min(kb, nr - r0);
    const bool fin = (r0 + cnt == nr);
    HiiBatch bt;
    hii_batch_radii(p, redshift, sched, r0, cnt, ntest, &bt);
    // the snapshot's last radius is unfiltered (find_HII_bubbles.c:313)
    const int unf = fin ? cnt - 1 : -1;
    if ((rc = inverse_xy(ctx, N, ctx->spec, ng, ng, ctx->work, nc, cnt, ctx->wtab + (size_t)r0 * (n2max + 1),
                         n2max + 1, unf, st, wcut ? wcut + r0 : nullptr)))
      return rc;
    if (r0 == 0 && (rc = stage_wait(ctx, stg->state, st))) return rc;
    if (fin && (rc = stage_wait(ctx, stg->closing, st))) return rc;
    if ((rc = hii_z(ctx, N, ctx->work, nc, ntest, bt, c, hs, fin, st, &nblocks))) return rc;
  }
  if ((rc = reduce_partials(ctx, partials, nblocks, HII_NSUM, ctx->d_sums, st))) return rc;
  if (rec) {
    RecTables tab;
    tab.knots = ctx->rec_knots;
    tab.y = ctx->rec_y;
    tab.c = ctx->rec_c;
    tab.nz = ctx->rec_nz;
    tab.nt = ctx->rec_nt;
    tab.ng = ctx->rec_ng;
    // recombinations.c:51-64: the table's bounds as the float expressions of the C
    tab.lng_lo = (double)(-10.0f);
    tab.lng_hi = (double)(-10.0f + 0.1f * (float)(ctx->rec_ng - 1));
    RecConst rcst;
    rcst.redshift = redshift;
    rcst.hubble_h = p->Hubble_h;
    const double prev_z = s->snapshot == 0 ? redshift : s->ZZ[s->snapshot - 1];
    rcst.zstep = (float)(prev_z - redshift);
    rcst.fabs_dtdz = (float)std::fabs(dtdz(p, (float)redshift) / p->Hubble_h);
    rcst.temp_dep = p->Flag_TemperatureDependentRec != 0;
    RecState rs;
    rs.xH = g->xH;
    rs.temp = g->temp_kinetic_all_gas;
    rs.deltax_unf = g->deltax;
    rs.r_bubble = g->r_bubble;
    rs.Gamma12 = g->Gamma12;
    rs.N_rec = g->N_rec;
    rs.residual_xH = g->residual_xH;
    rs.clumping_factor = g->clumping_factor;
    rs.t_resp = g->t_resp;
    const int rb = 4 * ctx->num_sms;
    if ((rc = hii_recomb(ctx, N, tab, rcst, rs, partials, rb, st))) return rc;
    if ((rc = reduce_partials(ctx, partials, rb, REC_NSUM, ctx->d_sums + 16, st))) return rc;
  }
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_sums, ctx->d_sums, sizeof(double) * 32, cudaMemcpyDeviceToHost, st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  prof_resolve(ctx);
  if ((rc = xy_ctrl_check(ctx, st))) return rc;
  hii_outputs(p, nr, ctx->h_sums, out);
  return RG_OK;
}

int hii_batch(rg_context* ctx, int nu, const rg_params* p, const rg_snapshot* s, const rg_grids* g,
              rg_hii_scalars* out) {
  int rc;
  cudaStream_t st = ctx->stream;
  const int N = ctx->N;
  const double z0 = s[0].ZZ[s[0].snapshot];
  auto sched = radius_schedule(&p[0], z0);
  for (int u = 1; u < nu; ++u) {
    auto su = radius_schedule(&p[u], s[u].ZZ[s[u].snapshot]);
    if (su.size() != sched.size()) return set_error(ctx, RG_EINVAL, "batch units with different radius schedules");
    for (size_t i = 0; i < su.size(); ++i)
      if (su[i].first != sched[i].first) return set_error(ctx, RG_EINVAL, "batch units with different radii");
  }
  std::vector<HiiConst> cs(nu);
  for (int u = 0; u < nu; ++u)
    if ((rc = hii_const(ctx, &p[u], s[u].ZZ[s[u].snapshot], &cs[u]))) return rc;
  // the units' grids one after another: unit u's grid k is grid u ngu + k of the batch
  const float* one[10];
  int ntest = 0;
  const int ngu = hii_sources(&p[0], &g[0], false, one, &ntest);
  std::vector<const float*> srcs((size_t)nu * ngu);
  for (int u = 0; u < nu; ++u) {
    hii_sources(&p[u], &g[u], false, one, &ntest);
    for (int k = 0; k < ngu; ++k) srcs[(size_t)u * ngu + k] = one[k];
  }
  const int ng = nu * ngu;
  const size_t nc = (size_t)(N / 2 + 1) * N * N, n3 = (size_t)N * N * N;
  const int nr = (int)sched.size();
  int kb = ctx->radius_batch > 0 ? ctx->radius_batch : 8;
  if (kb > KB_MAX) kb = KB_MAX;
  if (kb > nr) kb = nr;
  if ((rc = ensure_device(ctx, &ctx->spec, &ctx->spec_elems, nc * ng))) return rc;
  if ((rc = ensure_device(ctx, &ctx->work, &ctx->work_elems, nc * ng * kb))) return rc;
  // one state byte per cell of every unit
  if ((rc = ensure_device(ctx, &ctx->bits, &ctx->bits_elems, (n3 * nu + 3) / 4))) return rc;
  if ((rc = ensure_device(ctx, &ctx->batch_sums, &ctx->batch_sums_elems, (size_t)32 * nu))) return rc;
  if ((size_t)nu > ctx->h_batch_sums_elems) {
    if (ctx->h_batch_sums) cudaFreeHost(ctx->h_batch_sums);
    ctx->h_batch_sums = nullptr;
    ctx->h_batch_sums_elems = 0;
    if (cudaMallocHost((void**)&ctx->h_batch_sums, sizeof(double) * 32 * nu) != cudaSuccess)
      return set_error(ctx, RG_ENOMEM, "pinned batch sums");
    ctx->h_batch_sums_elems = (size_t)nu;
  }
  for (int g0 = 0; g0 < ng; g0 += MAXG)
    if ((rc = fft_forward(ctx, N, srcs.data() + g0, std::min(MAXG, ng - g0), ctx->spec + nc * g0, nc,
                          1.0 / std::pow((double)N, 3), st)))
      return rc;
  if ((rc = hii_windows(ctx, &p[0], sched, st))) return rc;
  const int n2max = 3 * (N / 2) * (N / 2);
  const int* wcut = p[0].ReionFilterType == 1 ? ctx->wcut : nullptr;
  for (int u = 0; u < nu; ++u)
    RG_CUDA_TRY(ctx, cudaMemsetAsync(g[u].r_bubble, 0, sizeof(float) * n3, st));
  double* partials = ensure_partials(ctx, (size_t)N * N * HII_NSUM);
  if (!partials) return set_error(ctx, RG_ENOMEM, "partials");
  std::vector<HiiState> hs(nu);
  for (int u = 0; u < nu; ++u)
    hs[u] = hii_state(&p[u], &g[u], reinterpret_cast<uint8_t*>(ctx->bits) + n3 * u, partials);

  if ((rc = xy_ctrl_reset(ctx, (size_t)(N / 2 + 1) * kb, st))) return rc;
  for (int r0 = 0; r0 < nr; r0 += kb) {
    const int cnt = std::min(kb, nr - r0);
    const bool fin = (r0 + cnt == nr);
    const int unf = fin ? cnt - 1 : -1;
    // the windowed inverse x/y passes of every unit's grids in one launch; unit u's block of
    // the work buffer is [radius][its grids], as a single snapshot's
    if ((rc = inverse_xy(ctx, N, ctx->spec, ng, ngu, ctx->work, nc, cnt, ctx->wtab + (size_t)r0 * (n2max + 1),
                         n2max + 1, unf, st, wcut ? wcut + r0 : nullptr)))
      return rc;
    for (int u = 0; u < nu; ++u) {
      HiiBatch bt;
      hii_batch_radii(&p[u], s[u].ZZ[s[u].snapshot], sched, r0, cnt, ntest, &bt);
      int nblocks = 0;
      if ((rc = hii_z(ctx, N, ctx->work + (size_t)u * cnt * ngu * nc, nc, ntest, bt, cs[u], hs[u], fin, st, &nblocks)))
        return rc;
      if (fin && (rc = reduce_partials(ctx, partials, nblocks, HII_NSUM, ctx->batch_sums + 32 * u, st))) return rc;
    }
  }
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_batch_sums, ctx->batch_sums, sizeof(double) * 32 * nu,
                                   cudaMemcpyDeviceToHost, st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  prof_resolve(ctx);
  if ((rc = xy_ctrl_check(ctx, st))) return rc;
  for (int u = 0; u < nu; ++u) hii_outputs(&p[u], nr, ctx->h_batch_sums + 32 * u, &out[u]);
  return RG_OK;
}

static int debug_inverse(rg_context* ctx, int n, const float* wrow, float* d_out, cudaStream_t st) {
  RG_DISPATCH_N(n, launch_debug_inverse<NN>(ctx, ctx->spec, ctx->work, wrow, d_out, st));
}

int spectrum_to_padded(rg_context* ctx, float* d_out, cudaStream_t st) {
  const size_t nc = (size_t)(ctx->N / 2 + 1) * ctx->N * ctx->N;
  int rc;
  if ((rc = ensure_device(ctx, &ctx->work, &ctx->work_elems, nc))) return rc;
  return debug_inverse(ctx, ctx->N, nullptr, d_out, st);
}

int debug_roundtrip(rg_context* ctx, const rg_params* p, const float* d_in, float* d_out, double R, int ftype) {
  int rc;
  cudaStream_t st = ctx->stream;
  const int N = ctx->N;
  const size_t nc = (size_t)(N / 2 + 1) * N * N;
  if ((rc = ensure_device(ctx, &ctx->spec, &ctx->spec_elems, nc))) return rc;
  if ((rc = ensure_device(ctx, &ctx->work, &ctx->work_elems, nc))) return rc;
  const float* srcs[1] = {d_in};
  if ((rc = fft_forward(ctx, N, srcs, 1, ctx->spec, nc, 1.0 / std::pow((double)N, 3), st))) return rc;
  const float* wrow = nullptr;
  if (ftype >= 0) {
    const int n2max = 3 * (N / 2) * (N / 2);
    if ((rc = ensure_device(ctx, &ctx->d_radii, &ctx->d_radii_elems, 1))) return rc;
    RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_radii, &R, sizeof(double), cudaMemcpyHostToDevice, st));
    if ((rc = ensure_device(ctx, &ctx->wtab, &ctx->wtab_elems, (size_t)(n2max + 1)))) return rc;
    if ((rc = window_table(ctx, p->BoxSize, ctx->d_radii, 1, ftype, ctx->wtab, n2max, st))) return rc;
    wrow = ctx->wtab;
  }
  if ((rc = debug_inverse(ctx, N, wrow, d_out, st))) return rc;
  return xy_ctrl_check(ctx, st);
}

}  // namespace rg
