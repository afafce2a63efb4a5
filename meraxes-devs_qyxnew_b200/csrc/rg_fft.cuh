// Shared-memory Stockham FFT building blocks for sm_100a.
//
// A tile in shared memory holds B independent complex lines of length L.  Element
// (pos p, line b) lives at buf[p * PS + b] with PS = B + 1: lines are the fast
// axis, so a warp's accesses during a butterfly stage touch consecutive words, and
// the odd pitch keeps column-wise fills (threads walking p) at 2-way bank sharing.
//
// The transform is the self-sorting Stockham formulation: log_R(L) stages, each
// reading R elements spaced L/R apart, twiddling, doing a radix-R DFT in registers
// and writing them to their sorted positions.  Reads of a stage complete (barrier)
// before its writes, so one buffer suffices.  L must be 2^a 3^b; radices 8, 4, 2
// and 3 are used, largest first.  Twiddles exp(-2 pi i k / L) come from a table in
// shared memory that was rounded once from double precision on the host.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rg {

struct cf {  // complex float, 8 bytes
  float x, y;
};

__device__ __forceinline__ cf cmk(float a, float b) { return cf{a, b}; }
__device__ __forceinline__ cf cadd(cf a, cf b) { return cf{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cf csub(cf a, cf b) { return cf{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cf cmul(cf a, cf b) {
  return cf{fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x)};
}
__device__ __forceinline__ cf cconj(cf a) { return cf{a.x, -a.y}; }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ cf mul_mi(cf a) {
  return INV ? cf{-a.y, a.x} : cf{a.y, -a.x};
}

// ---------------------------------------------------------------------------
// radix-R DFTs in registers; forward uses exp(-2 pi i / R), inverse exp(+2 pi i / R)

template <bool INV>
__device__ __forceinline__ void dft2(cf* v) {
  cf a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(cf* v) {
  cf t0 = cadd(v[0], v[2]);
  cf t1 = csub(v[0], v[2]);
  cf t2 = cadd(v[1], v[3]);
  cf t3 = mul_mi<INV>(csub(v[1], v[3]));
  v[0] = cadd(t0, t2);
  v[1] = cadd(t1, t3);
  v[2] = csub(t0, t2);
  v[3] = csub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void dft8(cf* v) {
  const float h = 0.70710678118654752440f;
  cf e[4] = {v[0], v[2], v[4], v[6]};
  cf o[4] = {v[1], v[3], v[5], v[7]};
  dft4<INV>(e);
  dft4<INV>(o);
  // o[k] *= W8^k
  o[1] = INV ? cf{h * (o[1].x - o[1].y), h * (o[1].x + o[1].y)}
             : cf{h * (o[1].x + o[1].y), h * (o[1].y - o[1].x)};
  o[2] = mul_mi<INV>(o[2]);
  o[3] = INV ? cf{-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y)}
             : cf{h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y)};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = cadd(e[k], o[k]);
    v[k + 4] = csub(e[k], o[k]);
  }
}

template <bool INV>
__device__ __forceinline__ void dft3(cf* v) {
  const float s = 0.86602540378443864676f;  // sqrt(3)/2
  cf t = cadd(v[1], v[2]);
  cf d = csub(v[1], v[2]);
  cf m = cf{v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y};
  // forward: y1 = m - i s d, y2 = m + i s d ; inverse swaps the signs
  cf isd = cf{-s * d.y, s * d.x};  // i * s * d
  v[0] = cadd(v[0], t);
  if (INV) {
    v[1] = cadd(m, isd);
    v[2] = csub(m, isd);
  } else {
    v[1] = csub(m, isd);
    v[2] = cadd(m, isd);
  }
}

template <int R, bool INV>
__device__ __forceinline__ void dft_small(cf* v) {
  if constexpr (R == 2) dft2<INV>(v);
  else if constexpr (R == 4) dft4<INV>(v);
  else if constexpr (R == 8) dft8<INV>(v);
  else if constexpr (R == 3) dft3<INV>(v);
}

template <int REM>
struct PickRadix {
  static constexpr int value = (REM % 8 == 0) ? 8 : (REM % 4 == 0) ? 4 : (REM % 2 == 0) ? 2 : 3;
  static_assert(REM % value == 0, "transform length must be 2^a 3^b");
};

// One Stockham stage over all B lines of the tile, executed by NT threads.
template <int L, int R, int NS, bool INV, int B, int NT>
__device__ __forceinline__ void stockham_stage(cf* buf, const cf* tw) {
  constexpr int PS = B + 1;
  constexpr int NBF = (L / R) * B;
  constexpr int K = (NBF + NT - 1) / NT;
  cf v[K][R];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = threadIdx.x + k * NT;
    if (NBF % NT == 0 || t < NBF) {
      const int b = t % B;
      const int j = t / B;
#pragma unroll
      for (int r = 0; r < R; ++r) v[k][r] = buf[(j + r * (L / R)) * PS + b];
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int t = threadIdx.x + k * NT;
    if (NBF % NT == 0 || t < NBF) {
      const int b = t % B;
      const int j = t / B;
      const int jm = j % NS;
      if constexpr (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          cf w = tw[(r * jm * (L / (NS * R))) % L];
          if (INV) w.y = -w.y;
          v[k][r] = cmul(v[k][r], w);
        }
      }
      dft_small<R, INV>(v[k]);
      const int idxD = (j / NS) * NS * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[(idxD + r * NS) * PS + b] = v[k][r];
    }
  }
  __syncthreads();
}

template <int L, int NS, bool INV, int B, int NT>
__device__ __forceinline__ void fft_stages(cf* buf, const cf* tw) {
  if constexpr (NS < L) {
    constexpr int R = PickRadix<L / NS>::value;
    stockham_stage<L, R, NS, INV, B, NT>(buf, tw);
    fft_stages<L, NS * R, INV, B, NT>(buf, tw);
  }
}

// In-place FFT of all B lines of a [L][B+1] tile.  Starts and ends with a barrier-clean state.
template <int L, bool INV, int B, int NT>
__device__ __forceinline__ void tile_fft(cf* buf, const cf* tw) {
  fft_stages<L, 1, INV, B, NT>(buf, tw);
}

// Copy the L-entry twiddle table into shared memory (caller syncs).
template <int L, int NT>
__device__ __forceinline__ void load_twiddles(cf* s_tw, const cf* __restrict__ g_tw) {
  for (int i = threadIdx.x; i < L; i += NT) s_tw[i] = g_tw[i];
}

}  // namespace rg
