// Excursion-set (find_HII_bubbles) kernels: 3-D r2c/c2r FFT passes, the k-space window
// and the barrier test, for sm_100a.
//
// Spectrum layout in HBM: complex S[kz][x][y], kz in [0, N/2], x and y in [0, N).  The
// forward chain is z-r2c (rows of the padded real grid, two rows per complex FFT) ->
// y-c2c (contiguous lines) -> x-c2c (lines of stride N, scaled by 1/N^3).  The inverse
// chain per radius is x-c2c with the window applied on load -> y-c2c -> z-c2r fused
// with the aliasing clamp and the barrier test (two neighbouring rows of a grid per complex
// FFT), so the per-cell state (xH, z_at_ionization, J_21, temperature) is touched once per
// radius.
#include <cuda_runtime.h>
#include <math.h>

#include <cstdio>
#include <vector>

#include "rg_fft.cuh"
#include "rg_internal.h"

namespace rg {

constexpr int NT = 256;

struct SrcPack {
  const void* p[HG_COUNT];
};
struct DstPack {
  void* p[HG_COUNT];
};

// ---------------------------------------------------------------------------
// forward z: r2c of pairs of padded rows

template <int N, int B>
__global__ void __launch_bounds__(NT) k_fwd_z(SrcPack srcs, DstPack dsts, const cf* __restrict__ g_tw) {
  constexpr int P = B / 2;  // complex lines (row pairs)
  constexpr int PS = P + 1;
  constexpr int NZ = N / 2 + 1;
  constexpr int PADW = 2 * (N / 2 + 1);
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* buf = smem + N;
  const float* src = static_cast<const float*>(srcs.p[blockIdx.z]);
  cf* dst = static_cast<cf*>(dsts.p[blockIdx.z]);
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * B;
  load_twiddles<N, NT>(s_tw, g_tw);
  for (int t = threadIdx.x; t < N * P; t += NT) {
    const int n = t % N, q = t / N;
    const size_t r0 = ((size_t)x * N + y0 + 2 * q) * PADW;
    buf[n * PS + q] = cf{__ldg(src + r0 + n), __ldg(src + r0 + PADW + n)};
  }
  __syncthreads();
  tile_fft<N, false, P, NT>(buf, s_tw);
  // split the two real transforms and store S[k][x][y0..y0+B)
  for (int t = threadIdx.x; t < NZ * B; t += NT) {
    const int yy = t % B, k = t / B;
    const int q = yy >> 1;
    const cf zk = buf[k * PS + q];
    const cf zn = buf[((N - k) % N) * PS + q];
    cf out;
    if ((yy & 1) == 0) {
      out = cf{0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y)};  // (Z[k] + conj(Z[N-k])) / 2
    } else {
      const float ax = zk.x - zn.x, ay = zk.y + zn.y;         // (Z[k] - conj(Z[N-k])) / (2i)
      out = cf{0.5f * ay, -0.5f * ax};
    }
    dst[((size_t)k * N + x) * N + y0 + yy] = out;
  }
}

// ---------------------------------------------------------------------------
// y: c2c along contiguous lines, S[kz][x][*]

template <int N, int B, bool INV>
__global__ void __launch_bounds__(NT) k_c2c_y(DstPack bufs, const cf* __restrict__ g_tw) {
  constexpr int PS = B + 1;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* buf = smem + N;
  cf* g = static_cast<cf*>(bufs.p[blockIdx.z]);
  const int kz = blockIdx.y;
  const int x0 = blockIdx.x * B;
  load_twiddles<N, NT>(s_tw, g_tw);
  cf* base = g + ((size_t)kz * N + x0) * N;
  for (int t = threadIdx.x; t < N * B; t += NT) {
    const int p = t % N, b = t / N;
    buf[p * PS + b] = base[(size_t)b * N + p];
  }
  __syncthreads();
  tile_fft<N, INV, B, NT>(buf, s_tw);
  for (int t = threadIdx.x; t < N * B; t += NT) {
    const int p = t % N, b = t / N;
    base[(size_t)b * N + p] = buf[p * PS + b];
  }
}

// ---------------------------------------------------------------------------
// x: c2c along lines of stride N.  Forward: scale on store.  Inverse: window on load.

template <int N, int B, bool INV>
__global__ void __launch_bounds__(NT) k_c2c_x(SrcPack srcs, DstPack dsts, const cf* __restrict__ g_tw, float scale,
                                              const float* __restrict__ wrow) {
  constexpr int PS = B + 1;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* buf = smem + N;
  const cf* src = static_cast<const cf*>(srcs.p[blockIdx.z]);
  cf* dst = static_cast<cf*>(dsts.p[blockIdx.z]);
  const int kz = blockIdx.y;
  const int y0 = blockIdx.x * B;
  load_twiddles<N, NT>(s_tw, g_tw);
  const size_t plane = (size_t)kz * N * N;
  for (int t = threadIdx.x; t < N * B; t += NT) {
    const int b = t % B, p = t / B;
    cf v = src[plane + (size_t)p * N + y0 + b];
    if (INV && wrow != nullptr) {
      const int nx = p > N / 2 ? p - N : p;
      const int yy = y0 + b;
      const int ny = yy > N / 2 ? yy - N : yy;
      const float w = __ldg(wrow + nx * nx + ny * ny + kz * kz);
      v.x *= w;
      v.y *= w;
    }
    buf[p * PS + b] = v;
  }
  __syncthreads();
  tile_fft<N, INV, B, NT>(buf, s_tw);
  for (int t = threadIdx.x; t < N * B; t += NT) {
    const int b = t % B, p = t / B;
    cf v = buf[p * PS + b];
    if (!INV) {
      v.x *= scale;
      v.y *= scale;
    }
    dst[plane + (size_t)p * N + y0 + b] = v;
  }
}

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

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Fill a [N][B/2+1] tile with Z_q = X(y0+2q) + i X(y0+2q+1): the full-length spectra of two
// neighbouring rows of ONE grid, whose Hermitian halves sit at src[base + k*pitch_k + y - y0]
// for k in [0, N/2].  After the inverse FFT the real part is row y0+2q and the imaginary part
// row y0+2q+1.  Rows of one grid share a magnitude scale, so the rounding each row picks up
// from its partner stays at the level of a separate transform (pairing two different grids,
// e.g. deltax ~ 1 with stars ~ 1e-3, would leak deltax-sized rounding into stars).  The DC and
// Nyquist terms keep only their real parts, as a c2r transform does.
template <int N, int B>
__device__ __forceinline__ void build_rowpair_tile(cf* buf, const cf* __restrict__ g, size_t base, size_t pitch_k) {
  constexpr int P = B / 2;
  constexpr int PS = P + 1;
  constexpr int NZ = N / 2 + 1;
  for (int t = threadIdx.x; t < NZ * P; t += NT) {
    const int q = t % P, k = t / P;
    const size_t idx = base + (size_t)k * pitch_k + 2 * q;
    const cf a = g[idx];
    const cf bb = g[idx + 1];
    if (k == 0 || k == N / 2) {
      buf[k * PS + q] = cf{a.x, bb.x};
    } else {
      buf[k * PS + q] = cf{a.x - bb.y, a.y + bb.x};
      buf[(N - k) * PS + q] = cf{a.x + bb.y, bb.x - a.y};
    }
  }
}

// value of row y0+b at z in a row-pair tile
template <int B>
__device__ __forceinline__ float rowpair_val(const cf* tile, int z, int b) {
  const cf v = tile[z * (B / 2 + 1) + (b >> 1)];
  return (b & 1) ? v.y : v.x;
}

// z: c2r of each grid (deltax, stars [, x_e] [, effective_bhm]), then per cell the clamp and
// barrier test of find_HII_bubbles.c:373-544; with FINAL also the closing pass of :577-645.
template <int N, int B, int NG, bool FINAL>
__global__ void __launch_bounds__(NT) k_inv_z_test(SrcPack works, const cf* __restrict__ g_tw, HiiRadius r,
                                                   HiiConst c, HiiState s) {
  constexpr int TS = N * (B / 2 + 1);   // one grid's tile
  constexpr int PADW = 2 * (N / 2 + 1);
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* tiles = smem + N;
  __shared__ double s_red[NT / 32][HII_NSUM];
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * B;
  load_twiddles<N, NT>(s_tw, g_tw);
#pragma unroll
  for (int gi = 0; gi < NG; ++gi)
    build_rowpair_tile<N, B>(tiles + gi * TS, static_cast<const cf*>(works.p[gi]), (size_t)x * N + y0,
                             (size_t)N * N);
  __syncthreads();
#pragma unroll
  for (int gi = 0; gi < NG; ++gi) tile_fft<N, true, B / 2, NT>(tiles + gi * TS, s_tw);

  double acc[HII_NSUM];
#pragma unroll
  for (int i = 0; i < HII_NSUM; ++i) acc[i] = 0.0;

  for (int t = threadIdx.x; t < N * B; t += NT) {
    const int z = t % N, b = t / N;
    const int y = y0 + b;
    const size_t ir = ((size_t)x * N + y) * N + z;
    const size_t ip = ((size_t)x * N + y) * PADW + z;
    const float dx = fmaxf(rowpair_val<B>(tiles, z, b), -1.f + REL_TOL);
    float st = fmaxf(rowpair_val<B>(tiles + TS, z, b), 0.f);
    if (st < ABS_TOL) st = 0.f;
    // grids 2.. : x_e with spin temperature, then effective_bhm with BH feedback
    float xe = 0.f, bhm = 0.f;
    if (NG > 2) {
      if (c.spin) {
        xe = fmaxf(rowpair_val<B>(tiles + 2 * TS, z, b), 0.f);
        if (xe < ABS_TOL) xe = 0.f;
        xe = fminf(xe, 0.999f);
      }
      if (c.bh) {
        bhm = fmaxf(rowpair_val<B>(tiles + (c.spin ? 3 : 2) * TS, z, b), 0.f);
        if (bhm < ABS_TOL) bhm = 0.f;
      }
    }
    const double dom = 1.0 + (double)dx;
    const double fcs = (double)st / dom;
    const double fbh = c.bh ? (double)bhm / dom : 0.0;
    const double nf = c.spin ? 1.0 - (double)xe : 1.0;
    const double lhs = (fbh + fcs) * r.fcoll_pref;
    float xH = r.first ? 1.f : s.xH[ir];
    float zin = s.z_in[ir];
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
  if (FINAL) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < HII_NSUM; ++i) {
      const double v = warp_sum(acc[i]);
      if (lane == 0) s_red[wid][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < HII_NSUM) {
      double v = 0.0;
      for (int w = 0; w < NT / 32; ++w) v += s_red[w][threadIdx.x];
      const size_t blk = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
      s.partials[blk * HII_NSUM + threadIdx.x] = v;
    }
  }
}

// deterministic second stage: one block sums the per-block partials in a fixed order
__global__ void k_reduce_partials(const double* __restrict__ partials, int nblocks, int nsum, double* out) {
  __shared__ double sh[NT];
  for (int i = 0; i < nsum; ++i) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += NT) v += partials[(size_t)b * nsum + i];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = NT / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[i] = sh[0];
    __syncthreads();
  }
}

// c2r of one spectrum into a padded real grid (no test): rows y and y+1 share a complex FFT
template <int N, int B>
__global__ void __launch_bounds__(NT) k_inv_z_padded(const cf* __restrict__ work, const cf* __restrict__ g_tw,
                                                     float* __restrict__ out) {
  constexpr int P = B / 2;
  constexpr int PS = P + 1;
  constexpr int NZ = N / 2 + 1;
  constexpr int PADW = 2 * (N / 2 + 1);
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* buf = smem + N;
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * B;
  load_twiddles<N, NT>(s_tw, g_tw);
  for (int t = threadIdx.x; t < NZ * P; t += NT) {
    const int q = t % P, k = t / P;
    const size_t idx = ((size_t)k * N + x) * N + y0 + 2 * q;
    const cf a = work[idx];
    const cf bb = work[idx + 1];
    if (k == 0 || k == N / 2) {
      buf[k * PS + q] = cf{a.x, bb.x};
    } else {
      buf[k * PS + q] = cf{a.x - bb.y, a.y + bb.x};
      buf[(N - k) * PS + q] = cf{a.x + bb.y, bb.x - a.y};
    }
  }
  __syncthreads();
  tile_fft<N, true, P, NT>(buf, s_tw);
  for (int t = threadIdx.x; t < N * B; t += NT) {
    const int z = t % N, b = t / N;
    const cf v = buf[z * PS + (b >> 1)];
    out[((size_t)x * N + y0 + b) * PADW + z] = (b & 1) ? v.y : v.x;
  }
}

// ---------------------------------------------------------------------------
// host-side launchers

template <int N>
struct Tiles {
  static_assert(N % 8 == 0, "grid dimension must be a multiple of 8");
  static constexpr int BZ = (N % 16 == 0) ? 16 : 8;  // rows per forward-z block (even)
  static constexpr int BY = 8;                       // lines per y block
  static constexpr int BX = (N % 16 == 0) ? 16 : 8;  // contiguous y per x block
  static constexpr int BT = 8;                       // y per test block
};

template <typename K>
static cudaError_t prep(K kernel, size_t smem) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int N>
static int forward_n(rg_context* ctx, const float* const* d_real, cf* const* d_spec, int ng, double scale,
                     cudaStream_t st) {
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  constexpr int NZ = N / 2 + 1;
  SrcPack src{};
  DstPack dst{};
  SrcPack dsrc{};
  for (int g = 0; g < ng; ++g) {
    src.p[g] = d_real[g];
    dst.p[g] = d_spec[g];
    dsrc.p[g] = d_spec[g];
  }
  {
    constexpr int B = Tiles<N>::BZ;
    const size_t sm = sizeof(cf) * (N + N * (B / 2 + 1));
    RG_CUDA_TRY(ctx, prep(k_fwd_z<N, B>, sm));
    prof_begin(ctx, "fwd_z_r2c", st);
    k_fwd_z<N, B><<<dim3(N / B, N, ng), NT, sm, st>>>(src, dst, tw);
    prof_end(ctx, ng * (4.0 * N * N * N + 8.0 * NZ * N * N), st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  {
    constexpr int B = Tiles<N>::BY;
    const size_t sm = sizeof(cf) * (N + N * (B + 1));
    RG_CUDA_TRY(ctx, prep(k_c2c_y<N, B, false>, sm));
    prof_begin(ctx, "fwd_y_c2c", st);
    k_c2c_y<N, B, false><<<dim3(N / B, NZ, ng), NT, sm, st>>>(dst, tw);
    prof_end(ctx, ng * 16.0 * NZ * N * N, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  {
    constexpr int B = Tiles<N>::BX;
    const size_t sm = sizeof(cf) * (N + N * (B + 1));
    RG_CUDA_TRY(ctx, prep(k_c2c_x<N, B, false>, sm));
    prof_begin(ctx, "fwd_x_c2c", st);
    k_c2c_x<N, B, false><<<dim3(N / B, NZ, ng), NT, sm, st>>>(dsrc, dst, tw, (float)scale, nullptr);
    prof_end(ctx, ng * 16.0 * NZ * N * N, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  return RG_OK;
}

template <int N>
static int inverse_xy_n(rg_context* ctx, cf* const* d_spec, cf* const* d_work, int ng, const float* wrow,
                        cudaStream_t st) {
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  constexpr int NZ = N / 2 + 1;
  SrcPack src{};
  DstPack dst{};
  for (int g = 0; g < ng; ++g) {
    src.p[g] = d_spec[g];
    dst.p[g] = d_work[g];
  }
  {
    constexpr int B = Tiles<N>::BX;
    const size_t sm = sizeof(cf) * (N + N * (B + 1));
    RG_CUDA_TRY(ctx, prep(k_c2c_x<N, B, true>, sm));
    prof_begin(ctx, "inv_x_c2c_window", st);
    k_c2c_x<N, B, true><<<dim3(N / B, NZ, ng), NT, sm, st>>>(src, dst, tw, 1.f, wrow);
    prof_end(ctx, ng * 16.0 * NZ * N * N, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  {
    constexpr int B = Tiles<N>::BY;
    const size_t sm = sizeof(cf) * (N + N * (B + 1));
    RG_CUDA_TRY(ctx, prep(k_c2c_y<N, B, true>, sm));
    prof_begin(ctx, "inv_y_c2c", st);
    k_c2c_y<N, B, true><<<dim3(N / B, NZ, ng), NT, sm, st>>>(dst, tw);
    prof_end(ctx, ng * 16.0 * NZ * N * N, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  return RG_OK;
}

template <int N, int NG, bool FINAL>
static int inverse_z_test_n3(rg_context* ctx, cf* const* d_work, const HiiRadius& r, const HiiConst& c,
                             const HiiState& s, cudaStream_t st, int* nblocks) {
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  constexpr int B = Tiles<N>::BT;
  SrcPack w{};
  for (int g = 0; g < NG; ++g) w.p[g] = d_work[g];
  const size_t sm = sizeof(cf) * (N + NG * N * (B / 2 + 1));
  RG_CUDA_TRY(ctx, prep(k_inv_z_test<N, B, NG, FINAL>, sm));
  const dim3 grid(N / B, N);
  // algorithmic bytes: the Hermitian halves read once, xH read (after the first radius)
  // and written, z_at_ionization read; the closing pass adds deltax, weighted_sfr,
  // effective_bhar, Tk_box reads and the temperature read + write.
  const double n3 = (double)N * N * N, nzc = (double)(N / 2 + 1) * N * N;
  double bytes = NG * 8.0 * nzc + (r.first ? 0.0 : 4.0 * n3) + 4.0 * n3 + 4.0 * n3;
  if (FINAL) bytes += 4.0 * n3 * (2 + (s.bhar != nullptr) + (s.Tk_box != nullptr) + 2);
  prof_begin(ctx, FINAL ? "inv_z_c2r_test_final" : "inv_z_c2r_test", st);
  k_inv_z_test<N, B, NG, FINAL><<<grid, NT, sm, st>>>(w, tw, r, c, s);
  prof_end(ctx, bytes, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  if (nblocks) *nblocks = (int)(grid.x * grid.y);
  return RG_OK;
}

template <int N>
static int inverse_z_test_n(rg_context* ctx, cf* const* d_work, int ngrids, const HiiRadius& r, const HiiConst& c,
                            const HiiState& s, bool fin, cudaStream_t st, int* nblocks) {
  if (ngrids == 2)
    return fin ? inverse_z_test_n3<N, 2, true>(ctx, d_work, r, c, s, st, nblocks)
               : inverse_z_test_n3<N, 2, false>(ctx, d_work, r, c, s, st, nblocks);
  if (ngrids == 3)
    return fin ? inverse_z_test_n3<N, 3, true>(ctx, d_work, r, c, s, st, nblocks)
               : inverse_z_test_n3<N, 3, false>(ctx, d_work, r, c, s, st, nblocks);
  return fin ? inverse_z_test_n3<N, 4, true>(ctx, d_work, r, c, s, st, nblocks)
             : inverse_z_test_n3<N, 4, false>(ctx, d_work, r, c, s, st, nblocks);
}

template <int N>
static int debug_inverse_n(rg_context* ctx, cf* spec, cf* work, const float* wrow, float* out, cudaStream_t st) {
  cf* sp[1] = {spec};
  cf* wk[1] = {work};
  int rc = inverse_xy_n<N>(ctx, sp, wk, 1, wrow, st);
  if (rc) return rc;
  const cf* tw;
  rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  constexpr int B = Tiles<N>::BZ;
  const size_t sm = sizeof(cf) * (N + N * (B / 2 + 1));
  RG_CUDA_TRY(ctx, prep(k_inv_z_padded<N, B>, sm));
  k_inv_z_padded<N, B><<<dim3(N / B, N), NT, sm, st>>>(work, tw, out);
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
  RG_DISPATCH_N(n, forward_n<NN>(ctx, d_real, d_spec, ng, scale, st));
}

int hii_inverse_xy(rg_context* ctx, int n, cf* const* d_spec, cf* const* d_work, int ng, const float* wrow,
                   cudaStream_t st) {
  RG_DISPATCH_N(n, inverse_xy_n<NN>(ctx, d_spec, d_work, ng, wrow, st));
}

int hii_inverse_z_test(rg_context* ctx, int n, cf* const* d_work, int ngrids, const HiiRadius& r, const HiiConst& c,
                       const HiiState& s, bool final_pass, cudaStream_t st, int* nblocks_out) {
  RG_DISPATCH_N(n, inverse_z_test_n<NN>(ctx, d_work, ngrids, r, c, s, final_pass, st, nblocks_out));
}

int debug_inverse_to_padded(rg_context* ctx, int n, cf* d_spec, cf* d_work, const float* wrow, float* d_out,
                            cudaStream_t st) {
  RG_DISPATCH_N(n, debug_inverse_n<NN>(ctx, d_spec, d_work, wrow, d_out, st));
}

int hii_window_table(rg_context* ctx, int n, double box, const double* d_radii, int nr, int ftype, float* d_wtab,
                     int n2max, cudaStream_t st) {
  (void)n;
  const float box_f = (float)box;
  (void)box_f;
  const double delta_k = 2.0 * M_PI / box;
  const int bx = (n2max + 1 + 255) / 256;
  k_window_table<<<dim3(bx < 1024 ? bx : 1024, nr), 256, 0, st>>>(d_wtab, n2max, d_radii, nr, delta_k, ftype);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

int hii_reduce_partials(rg_context* ctx, const double* partials, int nblocks, int nsum, double* d_out,
                        cudaStream_t st) {
  k_reduce_partials<<<1, NT, 0, st>>>(partials, nblocks, nsum, d_out);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

}  // namespace rg
