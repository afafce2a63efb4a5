// The 3-D r2c / c2r FFT passes over the spectrum layout S[kz][x][y] (complex, kz in [0, N/2],
// x and y in [0, N)), built on line_fft:
//
//   k_fwd_z   : r2c along z of a padded real grid, two neighbouring rows per complex line,
//               split into the two Hermitian halves in shared memory and stored as S[kz][x][y]
//   k_pass_y  : c2c along y (contiguous lines), in place
//   k_pass_x  : c2c along x (lines of stride N); a load hook (window, combination of several
//               spectra) and a scale on store
//   k_inv_z   : c2r along z of NG grids for a block of rows; two neighbouring rows of one grid
//               share a complex line; the real rows land in shared memory and an epilogue
//               object consumes them cell by cell
//
// Thread mappings follow the memory layout: along contiguous lines (z rows of the real grid,
// y lines of S) consecutive threads take consecutive positions; across strided lines (x and
// kz) consecutive threads take consecutive lines, so every global access is a run of
// consecutive elements.
#pragma once

#include "rg_fft.cuh"

namespace rg {

constexpr int MAXG = 8;  // grids per launch

struct GridPtrs {
  const void* p[MAXG];
};
struct GridPtrsW {
  void* p[MAXG];
};

// largest power of two <= cap that divides n (at least 1)
__host__ __device__ constexpr int pow2_div(int n, int cap) {
  int b = 1;
  while (b * 2 <= cap && n % (b * 2) == 0) b *= 2;
  return b;
}

template <int N>
struct Cfg {
  static constexpr int T = Plan<N>::T;
  static constexpr int NZ = N / 2 + 1;
  static constexpr int PADW = 2 * (N / 2 + 1);
  // x pass: BX contiguous y columns per block (>= 8 for 64-byte runs)
  static constexpr int BX = pow2_div(N, (256 / T) >= 8 ? 256 / T : 8);
  // y pass: BY lines per block
  static constexpr int BY = pow2_div(N, (256 / T) >= 1 ? 256 / T : 1);
  // forward z: QF row pairs per block
  static constexpr int QF = pow2_div(N / 2, (256 / T) >= 1 ? 256 / T : 1);
  // inverse z: QZ row pairs per block (2 QZ rows)
  static constexpr int QZ = pow2_div(N / 2, (256 / T) >= 4 ? 256 / T : 4);
  static constexpr int PITCH_Y = N + (T < 16 ? T : 0);   // line pitch of the y exchange buffer
  static constexpr int PITCH_F = N + (T < 16 ? T : 0);
  static constexpr int RT_PITCH = N + 1;                  // real row pitch (floats) in k_inv_z
};

// ---------------------------------------------------------------------------

template <int N>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::QF) k_fwd_z(GridPtrs srcs, GridPtrsW dsts, const cf* __restrict__ g_tw) {
  constexpr int T = Cfg<N>::T, Q = Cfg<N>::QF, NZ = Cfg<N>::NZ, PADW = Cfg<N>::PADW, PI = Cfg<N>::PITCH_F;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  cf* zbuf = xbuf + Q * PI;
  const float* src = static_cast<const float*>(srcs.p[blockIdx.z]);
  cf* dst = static_cast<cf*>(dsts.p[blockIdx.z]);
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * 2 * Q;
  const int t = threadIdx.x % T, q = threadIdx.x / T;
  load_twiddles<N>(s_tw, g_tw);
  __syncthreads();
  const float* r0 = src + ((size_t)x * N + y0 + 2 * q) * PADW;
  line_fft<N, false>(
      t, xbuf, s_tw, [&](int p) { return cf{__ldg(r0 + p), __ldg(r0 + PADW + p)}; },
      [&](int p) { return q * PI + p; }, [&](int p, cf v) { zbuf[q * PI + p] = v; });
  __syncthreads();
  // split Z = X(y) + i X(y+1) and store S[k][x][y0 .. y0 + 2Q)
  for (int i = threadIdx.x; i < NZ * 2 * Q; i += T * Q) {
    const int yy = i % (2 * Q), k = i / (2 * Q);
    const int qq = yy >> 1;
    const cf zk = zbuf[qq * PI + k];
    const cf zn = zbuf[qq * PI + (N - k) % N];
    cf out;
    if ((yy & 1) == 0) {
      out = cf{0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y)};  // (Z[k] + conj Z[N-k]) / 2
    } else {
      out = cf{0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x)};  // (Z[k] - conj Z[N-k]) / 2i
    }
    dst[((size_t)k * N + x) * N + y0 + yy] = out;
  }
}

template <int N, bool INV>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::BY) k_pass_y(GridPtrsW bufs, const cf* __restrict__ g_tw) {
  constexpr int T = Cfg<N>::T, B = Cfg<N>::BY, PI = Cfg<N>::PITCH_Y;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  cf* g = static_cast<cf*>(bufs.p[blockIdx.z]);
  const int kz = blockIdx.y;
  const int x0 = blockIdx.x * B;
  const int t = threadIdx.x % T, b = threadIdx.x / T;
  load_twiddles<N>(s_tw, g_tw);
  __syncthreads();
  cf* line = g + ((size_t)kz * N + x0 + b) * N;
  line_fft<N, INV>(
      t, xbuf, s_tw, [&](int p) { return line[p]; }, [&](int p) { return b * PI + p; },
      [&](int p, cf v) { line[p] = v; });
}

// x pass.  Load hook LD(line_ptr_offset, p, y, kz) -> cf supplies the input (plain copy,
// window, combination of spectra); the result is scaled by `scale` and stored to dst.
template <int N, bool INV, class LD>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::BX) k_pass_x(LD ld, GridPtrsW dsts, const cf* __restrict__ g_tw, float scale) {
  constexpr int T = Cfg<N>::T, B = Cfg<N>::BX;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  const int g = blockIdx.z;
  cf* dst = static_cast<cf*>(dsts.p[g]);
  const int kz = blockIdx.y;
  const int y0 = blockIdx.x * B;
  const int b = threadIdx.x % B, t = threadIdx.x / B;
  const int y = y0 + b;
  load_twiddles<N>(s_tw, g_tw);
  __syncthreads();
  const size_t col = (size_t)kz * N * N + y;   // element (kz, p, y) at col + p * N
  line_fft<N, INV>(
      t, xbuf, s_tw, [&](int p) { return ld(g, col + (size_t)p * N, p, y, kz); },
      [&](int p) { return p * B + b; },
      [&](int p, cf v) {
        v.x *= scale;
        v.y *= scale;
        dst[col + (size_t)p * N] = v;
      });
}

// plain x-pass input: src[g][idx]
struct LoadPlain {
  GridPtrs src;
  __device__ __forceinline__ cf operator()(int g, size_t idx, int, int, int) const {
    return static_cast<const cf*>(src.p[g])[idx];
  }
};

// x-pass input multiplied by a window that depends on |k|^2 = nx^2 + ny^2 + nz^2
template <int N>
struct LoadWindow {
  GridPtrs src;
  const float* wrow;   // W[n2], null = no window
  __device__ __forceinline__ cf operator()(int g, size_t idx, int p, int y, int kz) const {
    cf v = static_cast<const cf*>(src.p[g])[idx];
    if (wrow != nullptr) {
      const int nx = p > N / 2 ? p - N : p;
      const int ny = y > N / 2 ? y - N : y;
      const float w = __ldg(wrow + nx * nx + ny * ny + kz * kz);
      v.x *= w;
      v.y *= w;
    }
    return v;
  }
};

// ---------------------------------------------------------------------------
// inverse z: c2r of NG grids for rows [y0, y0 + 2 QZ) of plane x.  Real row r of grid g lands
// at rt[(g * 2 QZ + r) * RT_PITCH + z]; then epi(rt, x, y0) consumes the block's cells.

template <int N>
__device__ __forceinline__ cf build_c2r_input(const cf* __restrict__ g, size_t colpair, int p) {
  // Z[p] = A[p] + i B[p] for the full-length Hermitian extensions of rows A = y, B = y + 1,
  // whose halves sit at g[colpair + k N^2] (A) and +1 (B), k in [0, N/2]
  const int k = p <= N / 2 ? p : N - p;
  const float4 ab = __ldg(reinterpret_cast<const float4*>(g + colpair + (size_t)k * N * N));
  if (p == 0 || p == N / 2) return cf{ab.x, ab.z};
  if (p < N / 2) return cf{ab.x - ab.w, ab.y + ab.z};
  return cf{ab.x + ab.w, ab.z - ab.y};
}

template <int N, int NG, class EPI>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::QZ) k_inv_z(GridPtrs works, const cf* __restrict__ g_tw, EPI epi) {
  constexpr int T = Cfg<N>::T, Q = Cfg<N>::QZ, RP = Cfg<N>::RT_PITCH;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  float* rt = reinterpret_cast<float*>(xbuf + N * Q);
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * 2 * Q;
  const int q = threadIdx.x % Q, t = threadIdx.x / Q;
  load_twiddles<N>(s_tw, g_tw);
  __syncthreads();
  const size_t colpair = (size_t)x * N + y0 + 2 * q;
#pragma unroll
  for (int g = 0; g < NG; ++g) {
    const cf* src = static_cast<const cf*>(works.p[g]);
    float* r0 = rt + (size_t)(g * 2 * Q + 2 * q) * RP;
    line_fft<N, true>(
        t, xbuf, s_tw, [&](int p) { return build_c2r_input<N>(src, colpair, p); },
        [&](int p) { return p * Q + q; },
        [&](int p, cf v) {
          r0[p] = v.x;
          r0[RP + p] = v.y;
        });
  }
  __syncthreads();
  epi.template run<N, 2 * Q, T * Q>(rt, x, y0);
}

// epilogue: write the real rows to a padded grid
struct EpiPadded {
  float* out;
  template <int N, int ROWS, int NTH>
  __device__ __forceinline__ void run(const float* rt, int x, int y0) const {
    constexpr int PADW = 2 * (N / 2 + 1);
    for (int i = threadIdx.x; i < ROWS * N; i += NTH) {
      const int z = i % N, r = i / N;
      out[((size_t)x * N + y0 + r) * PADW + z] = rt[r * (N + 1) + z];
    }
  }
};

}  // namespace rg
