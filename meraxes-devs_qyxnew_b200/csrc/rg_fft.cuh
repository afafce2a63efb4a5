// Register-resident Stockham FFT building blocks for sm_100a.
//
// A line of length N is transformed by T threads.  The transform is the self-sorting
// Stockham factorisation N = R_0 R_1 ... R_{S-1}: at stage s, butterfly j (0 <= j < N/R_s)
// reads x[j + r N/R_s] (r < R_s), multiplies by exp(-+2 pi i r (j mod NS) / (NS R_s)) with
// NS = R_0 ... R_{s-1}, does a radix-R_s DFT in registers and writes its R_s results to
// (j / NS) NS R_s + (j mod NS) + r NS.  Thread t owns butterflies j = t, t + T, ... at every
// stage, so it always holds V = N / T values in registers.  Stage 0 reads through a load
// functor (global memory, or a prologue that builds the input), the last stage writes through
// a store functor (global memory, or an epilogue); between stages the values cross shared
// memory once (write, barrier, read).  With the radix plans below that is one exchange for
// N = 64, 128, 256 and two for N = 96, 192, 512.
//
// Twiddles come from a table exp(-2 pi i k / N) in shared memory, rounded once from double.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rg {

struct __align__(8) cf {  // complex float
  float x, y;
};

__device__ __forceinline__ cf cadd(cf a, cf b) { return cf{a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cf csub(cf a, cf b) { return cf{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cf cmul(cf a, cf b) {
  return cf{fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x)};
}
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ cf mul_mi(cf a) {
  return INV ? cf{-a.y, a.x} : cf{a.y, -a.x};
}
// multiply by exp(-+ 2 pi i m / 16), m in [0, 16)
template <bool INV, int M>
__device__ __forceinline__ cf mul_w16(cf a) {
  constexpr int m = M % 16;
  if constexpr (m == 0) return a;
  constexpr float C[4] = {1.0f, 0.92387953251128675613f, 0.70710678118654752440f, 0.38268343236508977173f};
  // cos and sin of 2 pi m / 16 from the first-quadrant table
  constexpr int q = m / 4, rr = m % 4;
  constexpr float c0 = rr == 0 ? 1.0f : C[rr];
  constexpr float s0 = rr == 0 ? 0.0f : C[4 - rr];
  constexpr float c = q == 0 ? c0 : q == 1 ? -s0 : q == 2 ? -c0 : s0;
  constexpr float s = q == 0 ? s0 : q == 1 ? c0 : q == 2 ? -s0 : -c0;
  // forward: (c - i s), inverse: (c + i s)
  const float sg = INV ? s : -s;
  return cf{a.x * c - a.y * sg, a.x * sg + a.y * c};
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
  o[1] = INV ? cf{h * (o[1].x - o[1].y), h * (o[1].x + o[1].y)} : cf{h * (o[1].x + o[1].y), h * (o[1].y - o[1].x)};
  o[2] = mul_mi<INV>(o[2]);
  o[3] = INV ? cf{-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y)} : cf{h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y)};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = cadd(e[k], o[k]);
    v[k + 4] = csub(e[k], o[k]);
  }
}

// 16 = 4 x 4: DFT4 over n1 of x[4 n1 + n2], twiddle W16^(n2 k1), DFT4 over n2 -> X[k1 + 4 k2]
template <bool INV>
__device__ __forceinline__ void dft16(cf* v) {
  cf a[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) a[n2][n1] = v[4 * n1 + n2];
    dft4<INV>(a[n2]);
  }
  a[1][1] = mul_w16<INV, 1>(a[1][1]);
  a[1][2] = mul_w16<INV, 2>(a[1][2]);
  a[1][3] = mul_w16<INV, 3>(a[1][3]);
  a[2][1] = mul_w16<INV, 2>(a[2][1]);
  a[2][2] = mul_w16<INV, 4>(a[2][2]);
  a[2][3] = mul_w16<INV, 6>(a[2][3]);
  a[3][1] = mul_w16<INV, 3>(a[3][1]);
  a[3][2] = mul_w16<INV, 6>(a[3][2]);
  a[3][3] = mul_w16<INV, 9>(a[3][3]);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    cf b[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
    dft4<INV>(b);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = b[k2];
  }
}

template <bool INV>
__device__ __forceinline__ void dft3(cf* v) {
  const float s = 0.86602540378443864676f;  // sqrt(3)/2
  cf t = cadd(v[1], v[2]);
  cf d = csub(v[1], v[2]);
  cf m = cf{v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y};
  cf isd = cf{-s * d.y, s * d.x};  // i s d
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
  else if constexpr (R == 3) dft3<INV>(v);
  else if constexpr (R == 4) dft4<INV>(v);
  else if constexpr (R == 8) dft8<INV>(v);
  else if constexpr (R == 16) dft16<INV>(v);
}

// ---------------------------------------------------------------------------
// radix plans: length NN, stages R[0..S) and threads per line T (T divides every N / R[s])

#define RG_PLAN(name, n, t, ...)                      \
  template <>                                         \
  struct name<n> {                                    \
    static constexpr int NN = n;                      \
    static constexpr int T = t;                       \
    static constexpr int R[] = {__VA_ARGS__};         \
    static constexpr int S = sizeof(R) / sizeof(int); \
  };

// default plans: few stages (one shared-memory exchange where the radices allow)
template <int N>
struct Plan;
RG_PLAN(Plan, 8, 1, 8)
RG_PLAN(Plan, 16, 1, 16)
RG_PLAN(Plan, 24, 1, 8, 3)
RG_PLAN(Plan, 32, 4, 8, 4)
RG_PLAN(Plan, 48, 2, 8, 2, 3)
RG_PLAN(Plan, 64, 8, 8, 8)
RG_PLAN(Plan, 96, 4, 8, 4, 3)
RG_PLAN(Plan, 128, 8, 16, 8)
RG_PLAN(Plan, 192, 8, 8, 8, 3)
RG_PLAN(Plan, 256, 16, 16, 16)
RG_PLAN(Plan, 384, 16, 8, 8, 2, 3)
RG_PLAN(Plan, 512, 64, 8, 8, 8)

// eight values per thread (power-of-two N): leaves registers for per-cell accumulators
template <int N>
struct Plan8;
RG_PLAN(Plan8, 8, 1, 8)
RG_PLAN(Plan8, 16, 2, 8, 2)
RG_PLAN(Plan8, 32, 4, 8, 4)
RG_PLAN(Plan8, 64, 8, 8, 8)
RG_PLAN(Plan8, 128, 16, 8, 4, 4)
RG_PLAN(Plan8, 256, 32, 8, 8, 4)
RG_PLAN(Plan8, 512, 64, 8, 8, 8)
#undef RG_PLAN

template <class PL, int s>
struct StageNS {
  static constexpr int value = StageNS<PL, s - 1>::value * PL::R[s - 1];
};
template <class PL>
struct StageNS<PL, 0> {
  static constexpr int value = 1;
};

template <class PL>
constexpr int plan_product() {
  int p = 1;
  for (int i = 0; i < PL::S; ++i) p *= PL::R[i];
  return p;
}

// Twiddles are kept per stage: stage s >= 1 owns entries [tw_offset(s), tw_offset(s) + NS (R - 1))
// with entry jm (R - 1) + (r - 1) = e^{-2 pi i r jm / (NS R)}, so threads with consecutive jm
// read consecutive words (a table indexed by r jm N / (NS R) puts them on a few banks).  The
// stages together hold N - R_0 entries.
template <class PL>
__host__ __device__ constexpr int tw_offset(int s) {
  int off = 0, ns = PL::R[0];
  for (int i = 1; i < s; ++i) {
    off += ns * (PL::R[i] - 1);
    ns *= PL::R[i];
  }
  return off;
}

// Stage-0 input position of register slot `slot` (0 <= slot < N/T) of thread t.
template <class PL>
__device__ __forceinline__ int stage0_pos(int t, int slot) {
  constexpr int R = PL::R[0];
  constexpr int T = PL::T;
  constexpr int N = PL::NN;
  return t + (slot / R) * T + (slot % R) * (N / R);
}

// run stage s: fill v from `load(pos, slot)`, twiddle, DFT
template <class PL, int s, bool INV, class Load>
__device__ __forceinline__ void stage_compute(cf* v, int t, const cf* __restrict__ tw, Load&& load) {
  constexpr int N = PL::NN;
  constexpr int T = PL::T;
  constexpr int R = PL::R[s];
  constexpr int NS = StageNS<PL, s>::value;
  constexpr int K = (N / R) / T;
  static_assert((N / R) % T == 0, "T must divide N/R");
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int j = t + k * T;
#pragma unroll
    for (int r = 0; r < R; ++r) v[k * R + r] = load(j + r * (N / R), k * R + r);
    if constexpr (NS > 1) {
      const int jm = j % NS;
      constexpr int OFF = tw_offset<PL>(s);
#pragma unroll
      for (int r = 1; r < R; ++r) {
        cf w = tw[OFF + jm * (R - 1) + (r - 1)];
        if (INV) w.y = -w.y;
        v[k * R + r] = cmul(v[k * R + r], w);
      }
    }
    dft_small<R, INV>(v + k * R);
  }
}

// hand stage s's outputs to `put(pos, value, slot)`
template <class PL, int s, class Put>
__device__ __forceinline__ void stage_emit(const cf* v, int t, Put&& put) {
  constexpr int T = PL::T;
  constexpr int N = PL::NN;
  constexpr int R = PL::R[s];
  constexpr int NS = StageNS<PL, s>::value;
  constexpr int K = (N / R) / T;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int j = t + k * T;
    const int idxD = (j / NS) * NS * R + (j % NS);
#pragma unroll
    for (int r = 0; r < R; ++r) put(idxD + r * NS, v[k * R + r], k * R + r);
  }
}

// WS: every line's threads are lanes of one warp and its exchange buffer region is its own, so
// a warp barrier orders the exchange; otherwise a block barrier
template <bool WS>
__device__ __forceinline__ void exchange_sync() {
  if constexpr (WS) __syncwarp();
  else __syncthreads();
}

template <class PL, int s, bool INV, bool WS = false, class Addr, class Store>
__device__ __forceinline__ void stages_from(cf* v, int t, cf* xbuf, Addr&& addr, const cf* tw, Store&& store) {
  if constexpr (s + 1 < PL::S) {
    exchange_sync<WS>();  // every thread is done reading xbuf
    stage_emit<PL, s>(v, t, [&](int p, cf x, int) { xbuf[addr(p)] = x; });
    exchange_sync<WS>();
    stage_compute<PL, s + 1, INV>(v, t, tw, [&](int p, int) { return xbuf[addr(p)]; });
    stages_from<PL, s + 1, INV, WS>(v, t, xbuf, addr, tw, store);
  } else {
    stage_emit<PL, s>(v, t, store);
  }
}

// Last-stage output position of register slot `slot` of thread t (the order store() sees).
template <class PL>
__device__ __forceinline__ int last_pos(int t, int slot) {
  constexpr int s = PL::S - 1;
  constexpr int R = PL::R[s];
  constexpr int NS = StageNS<PL, s>::value;
  const int j = t + (slot / R) * PL::T;
  return (j / NS) * NS * R + (j % NS) + (slot % R) * NS;
}

// Full transform of one line by thread t (0 <= t < PL::T):
//   load(p, slot)       -> input element at position p, held in register slot `slot`
//                          (stage0_pos<PL>(t, slot) == p)
//   addr(p)             -> index into xbuf of position p of this thread's line (exchange buffer)
//   store(p, val, slot) <- output element at position p (last_pos<PL>(t, slot) == p)
// Every thread of the block must call it (it contains block barriers when S > 1, unless WS).
//   WS: the line's threads are lanes of one warp (T <= 32, consecutive lanes) and addr() maps
//   each line into a region of xbuf no other line uses: warp barriers instead of block barriers.
template <class PL, bool INV, bool WS = false, class Load, class Addr, class Store>
__device__ __forceinline__ void line_fft_p(int t, cf* xbuf, const cf* tw, Load&& load, Addr&& addr, Store&& store) {
  static_assert(plan_product<PL>() == PL::NN, "radix plan does not multiply to N");
  static_assert(!WS || (PL::T <= 32 && 32 % PL::T == 0), "warp barriers need a line within a warp");
  constexpr int V = PL::NN / PL::T;
  cf v[V];
  stage_compute<PL, 0, INV>(v, t, tw, load);
  stages_from<PL, 0, INV, WS>(v, t, xbuf, addr, tw, store);
}

// line_fft with the default plan; store(p, val) without the slot
template <int N, bool INV, class Load, class Addr, class Store>
__device__ __forceinline__ void line_fft(int t, cf* xbuf, const cf* tw, Load&& load, Addr&& addr, Store&& store) {
  line_fft_p<Plan<N>, INV>(t, xbuf, tw, load, addr, [&](int p, cf v, int) { store(p, v); });
}

template <int N>
__device__ __forceinline__ int stage0_pos(int t, int slot) {
  return stage0_pos<Plan<N>>(t, slot);
}

// Fill the per-stage twiddle tables of plan PL in shared memory from the N-entry table
// g_tw[k] = e^{-2 pi i k / N} (caller syncs).
template <class PL, int s>
__device__ __forceinline__ void load_twiddle_stages(cf* s_tw, const cf* __restrict__ g_tw) {
  if constexpr (s < PL::S) {
    constexpr int N = PL::NN;
    constexpr int R = PL::R[s];
    constexpr int NS = StageNS<PL, s>::value;
    constexpr int OFF = tw_offset<PL>(s);
    for (int i = threadIdx.x; i < NS * (R - 1); i += blockDim.x) {
      const int jm = i / (R - 1), r = i % (R - 1) + 1;
      s_tw[OFF + i] = g_tw[(r * jm * (N / (NS * R))) % N];
    }
    load_twiddle_stages<PL, s + 1>(s_tw, g_tw);
  }
}
template <class PL>
__device__ __forceinline__ void load_twiddles_p(cf* s_tw, const cf* __restrict__ g_tw) {
  load_twiddle_stages<PL, 1>(s_tw, g_tw);
}
// the default plan's tables (N entries of shared memory always suffice)
template <int N>
__device__ __forceinline__ void load_twiddles(cf* s_tw, const cf* __restrict__ g_tw) {
  load_twiddles_p<Plan<N>>(s_tw, g_tw);
}

}  // namespace rg
