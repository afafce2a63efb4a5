// Excursion-set (find_HII_bubbles) step on sm_100a: the forward r2c of the source grids, and
// per filter radius the inverse chain x (window applied on load) -> y -> z-c2r fused with the
// aliasing clamp and the barrier test, so the per-cell state (xH, z_at_ionization, J_21,
// temperature) is touched once per radius.  The last radius also runs the closing pass
// (temperatures and the FP64 global sums).
#include <cuda_runtime.h>
#include <math.h>

#include <cstdio>
#include <vector>

#include "rg_internal.h"
#include "rg_pass.cuh"

namespace rg {

// ---------------------------------------------------------------------------
// window table W[r][n2], n2 = nx^2 + ny^2 + nz^2, evaluated in double from the closed
// forms of filter() (src/core/reionization.c:3404-3428)

__global__ void k_window_table(float* wtab, int n2max, const double* __restrict__ radii, int nr, double delta_k,
                               int ftype) {
  const int r = blockIdx.y;
  if (r >= nr) return;
  const double R = radii[r];
  for (int n2 = blockIdx.x * blockDim.x + threadIdx.x; n2 <= n2max; n2 += gridDim.x * blockDim.x) {
    const double kR = delta_k * sqrt((double)n2) * R;
    double w = 1.0;
    if (ftype == 0) {
      if (kR > 1e-4) w = 3.0 * (sin(kR) / (kR * kR * kR) - cos(kR) / (kR * kR));
    } else if (ftype == 1) {
      if (kR * 0.413566994 > 1.0) w = 0.0;
    } else {
      const double g = kR * 0.643;
      w = exp(-g * g / 2.0);
    }
    wtab[(size_t)r * (n2max + 1) + n2] = (float)w;
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

// Per-cell clamp and barrier test (find_HII_bubbles.c:373-544); FINAL adds the closing pass
// (:577-645).  Grids in rt: 0 deltax, 1 stars, then x_e (spin temperature), then
// effective_bhm (BH feedback).
template <bool FINAL>
struct EpiHii {
  HiiRadius r;
  HiiConst c;
  HiiState s;

  template <int N, int ROWS, int NTH>
  __device__ __forceinline__ void run(const float* rt, int x, int y0) const {
    constexpr int PADW = 2 * (N / 2 + 1);
    constexpr int RP = N + 1;
    double acc[HII_NSUM];
#pragma unroll
    for (int i = 0; i < HII_NSUM; ++i) acc[i] = 0.0;
    const int gx = c.spin ? 2 : -1;
    const int gb = c.bh ? (c.spin ? 3 : 2) : -1;
    // Cells are taken CH at a time: the global reads of a chunk are issued together before
    // any of its stores, so their latencies overlap (the state pointers may alias as far as
    // the compiler knows, which would otherwise serialise load -> store -> load).
    constexpr int NCELL = ROWS * N;
    constexpr int CH = 8;
    static_assert(NCELL % NTH == 0, "block covers whole rows");
    constexpr int IT = NCELL / NTH;
    constexpr int CHK = IT < CH ? IT : CH;
    static_assert(IT % CHK == 0, "chunking");
    for (int it0 = 0; it0 < IT; it0 += CHK) {
      float xh_in[CHK], zin_in[CHK];
#pragma unroll
      for (int u = 0; u < CHK; ++u) {
        const int i = threadIdx.x + (it0 + u) * NTH;
        const int z = i % N, row = i / N;
        const size_t ir = ((size_t)x * N + y0 + row) * N + z;
        xh_in[u] = r.first ? 1.f : __ldg(s.xH + ir);
        zin_in[u] = __ldg(s.z_in + ir);
      }
#pragma unroll
      for (int u = 0; u < CHK; ++u) {
      const int i = threadIdx.x + (it0 + u) * NTH;
      const int z = i % N, row = i / N;
      const int y = y0 + row;
      const size_t ir = ((size_t)x * N + y) * N + z;
      const size_t ip = ((size_t)x * N + y) * PADW + z;
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
      const double dom = 1.0 + (double)dx;
      const double fcs = (double)st / dom;
      const double fbh = c.bh ? (double)bhm / dom : 0.0;
      const double nf = c.spin ? 1.0 - (double)xe : 1.0;
      const double lhs = (fbh + fcs) * r.fcoll_pref;
      float xH = xh_in[u];
      float zin = zin_in[u];
      if (lhs > nf * (1.0 + 0.0)) {
        xH = 0.f;
      } else if (r.last && xH > REL_TOL) {
        float thi;
        if (c.spin) {
          thi = s.Tk_box[ir];
        } else {
          const float du = s.deltax_unf[ip];
          thi = (float)((double)c.TK * (1.0 + (double)(c.cT_ad * du)));
        }
        s.temp[ir] = partial_T(thi, xH);
        float v = (float)(nf - lhs);
        v = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
        xH = v;
      }
      if (xH < REL_TOL && zin < 0.f) {
        zin = c.redshift;
        s.z_in[ir] = zin;
        if (c.uvb == 1) {
          float j = st * r.J_aux;
          if (c.bh) j += bhm * r.J_aux_bh;
          s.J21[ir] = j;
        }
      }
      s.xH[ir] = xH;
      if (FINAL) {
        const float du = s.deltax_unf[ip];
        const double domu = 1.0 + (double)du;
        float temp = s.temp[ir];
        if (zin > 0.f && xH < REL_TOL) temp = fully_ionized_T(zin, c.redshift, du);
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
        // (find_HII_bubbles.c:490-508), which this library rejects, so it stays 0.
        acc[2] += (double)s.wsfr[ip];
        if (s.bhar != nullptr) acc[3] += (double)s.bhar[ip];
        acc[4] += (double)temp;
        acc[5] += (double)xH * domu;
        acc[7] += (double)temp * domu;
        acc[8] += domu;
      }
      }
    }
    if (FINAL) block_sum<NTH, HII_NSUM>(acc, s.partials + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * HII_NSUM);
  }
};

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
// host-side launchers

template <typename K>
static cudaError_t prep(K kernel, size_t smem) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int N>
size_t smem_x() { return sizeof(cf) * (N + (size_t)N * Cfg<N>::BX); }
template <int N>
size_t smem_y() { return sizeof(cf) * (N + (size_t)Cfg<N>::BY * Cfg<N>::PITCH_Y); }
template <int N>
size_t smem_fz() { return sizeof(cf) * (N + 2 * (size_t)Cfg<N>::QF * Cfg<N>::PITCH_F); }
template <int N>
size_t smem_iz(int ng) {
  return sizeof(cf) * (N + (size_t)N * Cfg<N>::QZ) + sizeof(float) * (size_t)ng * 2 * Cfg<N>::QZ * (N + 1);
}

template <int N>
int launch_forward(rg_context* ctx, const float* const* d_real, cf* const* d_spec, int ng, double scale,
                   cudaStream_t st) {
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  using C = Cfg<N>;
  GridPtrs src{};
  GridPtrsW dst{};
  GridPtrs dsrc{};
  for (int g = 0; g < ng; ++g) {
    src.p[g] = d_real[g];
    dst.p[g] = d_spec[g];
    dsrc.p[g] = d_spec[g];
  }
  const double nzc = (double)C::NZ * N * N;
  {
    const size_t sm = smem_fz<N>();
    RG_CUDA_TRY(ctx, prep(k_fwd_z<N>, sm));
    prof_begin(ctx, "fwd_z_r2c", st);
    k_fwd_z<N><<<dim3(N / (2 * C::QF), N, ng), C::T * C::QF, sm, st>>>(src, dst, tw);
    prof_end(ctx, ng * (4.0 * N * N * N + 8.0 * nzc), st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  {
    const size_t sm = smem_y<N>();
    RG_CUDA_TRY(ctx, prep(k_pass_y<N, false>, sm));
    prof_begin(ctx, "fwd_y_c2c", st);
    k_pass_y<N, false><<<dim3(N / C::BY, C::NZ, ng), C::T * C::BY, sm, st>>>(dst, tw);
    prof_end(ctx, ng * 16.0 * nzc, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  {
    const size_t sm = smem_x<N>();
    RG_CUDA_TRY(ctx, prep(k_pass_x<N, false, LoadPlain>, sm));
    prof_begin(ctx, "fwd_x_c2c", st);
    k_pass_x<N, false, LoadPlain><<<dim3(N / C::BX, C::NZ, ng), C::T * C::BX, sm, st>>>(LoadPlain{dsrc}, dst, tw,
                                                                                          (float)scale);
    prof_end(ctx, ng * 16.0 * nzc, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  return RG_OK;
}

template <int N>
int launch_inverse_xy(rg_context* ctx, cf* const* d_spec, cf* const* d_work, int ng, const float* wrow,
                      cudaStream_t st) {
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  using C = Cfg<N>;
  GridPtrs src{};
  GridPtrsW dst{};
  for (int g = 0; g < ng; ++g) {
    src.p[g] = d_spec[g];
    dst.p[g] = d_work[g];
  }
  const double nzc = (double)C::NZ * N * N;
  {
    const size_t sm = smem_x<N>();
    RG_CUDA_TRY(ctx, prep(k_pass_x<N, true, LoadWindow<N>>, sm));
    prof_begin(ctx, "inv_x_c2c_window", st);
    k_pass_x<N, true, LoadWindow<N>><<<dim3(N / C::BX, C::NZ, ng), C::T * C::BX, sm, st>>>(
        LoadWindow<N>{src, wrow}, dst, tw, 1.f);
    prof_end(ctx, ng * 16.0 * nzc, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  {
    const size_t sm = smem_y<N>();
    RG_CUDA_TRY(ctx, prep(k_pass_y<N, true>, sm));
    prof_begin(ctx, "inv_y_c2c", st);
    k_pass_y<N, true><<<dim3(N / C::BY, C::NZ, ng), C::T * C::BY, sm, st>>>(dst, tw);
    prof_end(ctx, ng * 16.0 * nzc, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  return RG_OK;
}

template <int N, int NG, bool FINAL>
int launch_inv_z_test3(rg_context* ctx, cf* const* d_work, const HiiRadius& r, const HiiConst& c, const HiiState& s,
                       cudaStream_t st, int* nblocks) {
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  using C = Cfg<N>;
  GridPtrs w{};
  for (int g = 0; g < NG; ++g) w.p[g] = d_work[g];
  const size_t sm = smem_iz<N>(NG);
  RG_CUDA_TRY(ctx, prep(k_inv_z<N, NG, EpiHii<FINAL>>, sm));
  const dim3 grid(N / (2 * C::QZ), N);
  // algorithmic bytes: the Hermitian halves read once, xH read (after the first radius)
  // and written, z_at_ionization read; the closing pass adds deltax, weighted_sfr,
  // effective_bhar, Tk_box reads and the temperature read + write.
  const double n3 = (double)N * N * N, nzc = (double)C::NZ * N * N;
  double bytes = NG * 8.0 * nzc + (r.first ? 0.0 : 4.0 * n3) + 4.0 * n3 + 4.0 * n3;
  if (FINAL) bytes += 4.0 * n3 * (2 + (s.bhar != nullptr) + (s.Tk_box != nullptr) + 2);
  prof_begin(ctx, FINAL ? "inv_z_c2r_test_final" : "inv_z_c2r_test", st);
  k_inv_z<N, NG, EpiHii<FINAL>><<<grid, C::T * C::QZ, sm, st>>>(w, tw, EpiHii<FINAL>{r, c, s});
  prof_end(ctx, bytes, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  if (nblocks) *nblocks = (int)(grid.x * grid.y);
  return RG_OK;
}

template <int N>
int launch_inv_z_test(rg_context* ctx, cf* const* d_work, int ngrids, const HiiRadius& r, const HiiConst& c,
                      const HiiState& s, bool fin, cudaStream_t st, int* nblocks) {
  if (ngrids == 2)
    return fin ? launch_inv_z_test3<N, 2, true>(ctx, d_work, r, c, s, st, nblocks)
               : launch_inv_z_test3<N, 2, false>(ctx, d_work, r, c, s, st, nblocks);
  if (ngrids == 3)
    return fin ? launch_inv_z_test3<N, 3, true>(ctx, d_work, r, c, s, st, nblocks)
               : launch_inv_z_test3<N, 3, false>(ctx, d_work, r, c, s, st, nblocks);
  return fin ? launch_inv_z_test3<N, 4, true>(ctx, d_work, r, c, s, st, nblocks)
             : launch_inv_z_test3<N, 4, false>(ctx, d_work, r, c, s, st, nblocks);
}

template <int N>
int launch_debug_inverse(rg_context* ctx, cf* spec, cf* work, const float* wrow, float* out, cudaStream_t st) {
  cf* sp[1] = {spec};
  cf* wk[1] = {work};
  int rc = launch_inverse_xy<N>(ctx, sp, wk, 1, wrow, st);
  if (rc) return rc;
  const cf* tw;
  rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  using C = Cfg<N>;
  GridPtrs w{};
  w.p[0] = work;
  const size_t sm = smem_iz<N>(1);
  RG_CUDA_TRY(ctx, prep(k_inv_z<N, 1, EpiPadded>, sm));
  k_inv_z<N, 1, EpiPadded><<<dim3(N / (2 * C::QZ), N), C::T * C::QZ, sm, st>>>(w, tw, EpiPadded{out});
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

int hii_forward(rg_context* ctx, int n, const float* const* d_real, cf* const* d_spec, int ng, double scale,
                cudaStream_t st) {
  if (ng > MAXG) return set_error(ctx, RG_EINVAL, "too many grids in one forward launch");
  RG_DISPATCH_N(n, launch_forward<NN>(ctx, d_real, d_spec, ng, scale, st));
}

int hii_inverse_xy(rg_context* ctx, int n, cf* const* d_spec, cf* const* d_work, int ng, const float* wrow,
                   cudaStream_t st) {
  if (ng > MAXG) return set_error(ctx, RG_EINVAL, "too many grids in one inverse launch");
  RG_DISPATCH_N(n, launch_inverse_xy<NN>(ctx, d_spec, d_work, ng, wrow, st));
}

int hii_inverse_z_test(rg_context* ctx, int n, cf* const* d_work, int ngrids, const HiiRadius& r, const HiiConst& c,
                       const HiiState& s, bool final_pass, cudaStream_t st, int* nblocks_out) {
  if (ngrids < 2 || ngrids > 4) return set_error(ctx, RG_EINVAL, "the barrier test reads 2 to 4 grids");
  RG_DISPATCH_N(n, launch_inv_z_test<NN>(ctx, d_work, ngrids, r, c, s, final_pass, st, nblocks_out));
}

int debug_inverse_to_padded(rg_context* ctx, int n, cf* d_spec, cf* d_work, const float* wrow, float* d_out,
                            cudaStream_t st) {
  RG_DISPATCH_N(n, launch_debug_inverse<NN>(ctx, d_spec, d_work, wrow, d_out, st));
}

int hii_window_table(rg_context* ctx, int n, double box, const double* d_radii, int nr, int ftype, float* d_wtab,
                     int n2max, cudaStream_t st) {
  (void)n;
  const double delta_k = 2.0 * M_PI / box;
  const int bx = (n2max + 1 + 255) / 256;
  k_window_table<<<dim3(bx < 1024 ? bx : 1024, nr), 256, 0, st>>>(d_wtab, n2max, d_radii, nr, delta_k, ftype);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

int hii_reduce_partials(rg_context* ctx, const double* partials, int nblocks, int nsum, double* d_out,
                        cudaStream_t st) {
  k_reduce_partials<<<1, 256, 0, st>>>(partials, nblocks, nsum, d_out);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

}  // namespace rg
