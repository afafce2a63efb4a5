// The 3-D r2c / c2r FFT passes over the spectrum layout S[kz][x][y] (complex, kz in [0, N/2],
// x and y in [0, N)), built on line_fft:
//
//   k_fwd_z     : r2c along z of padded real grids, two neighbouring rows per complex line,
//                 split into the two Hermitian halves in shared memory, stored as S[kz][x][y]
//   k_pass_y    : c2c along y (contiguous lines), in place, over a run of equally spaced grids
//   k_pass_x_fwd: c2c along x (lines of stride N), in place, scaled on store
//   zfront      : c2r along z of NG grids for a block of rows; two neighbouring rows of one grid
//                 share a complex line; the real rows land in shared memory for an epilogue
//
// Thread mappings follow the memory layout: along contiguous lines (z rows of the real grid,
// y lines of S) consecutive threads take consecutive positions; across strided lines (x and
// kz) consecutive threads take consecutive lines, so every global access is a run of
// consecutive elements.  Exchange buffers are padded so the Stockham write pattern (stride R
// between threads) does not collide on shared-memory banks.
#pragma once

#include "rg_fft.cuh"

namespace rg {

constexpr int MAXG = 8;  // separately addressed grids per launch

// minimum resident blocks per SM for a block of n threads: enough for 512 threads, which caps
// the registers a pass kernel may take at 128 per thread
#define RG_MINB(n) ((n) >= 512 ? 1 : 512 / (n))

struct GridPtrs {
  const void* p[MAXG];
};
struct GridPtrsW {
  void* p[MAXG];
};

// pointer g of a pack without dynamic indexing into kernel parameters (which would put the
// pack in local memory)
__device__ __forceinline__ const void* pick(const GridPtrs& a, int g) {
  const void* r = a.p[0];
#pragma unroll
  for (int i = 1; i < MAXG; ++i)
    if (g == i) r = a.p[i];
  return r;
}

// largest power of two <= cap that divides n (at least 1)
__host__ __device__ constexpr int pow2_div(int n, int cap) {
  int b = 1;
  while (b * 2 <= cap && n % (b * 2) == 0) b *= 2;
  return b;
}
__host__ __device__ constexpr int round_up(int a, int m) { return (a + m - 1) / m * m; }
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <int N>
struct Cfg {
  static constexpr int T = Plan<N>::T;
  static constexpr int V = N / T;
  static constexpr int NZ = N / 2 + 1;
  static constexpr int PADW = 2 * (N / 2 + 1);
  // x pass: BX contiguous y columns per block (>= 8 for 64-byte runs)
  static constexpr int BX = pow2_div(N, cmax(256 / T, 8));
  // y pass: BY lines per block
  static constexpr int BY = pow2_div(N, cmax(256 / T, 1));
  // forward z: QF row pairs per block
  static constexpr int QF = pow2_div(N / 2, cmax(256 / T, 1));
  // inverse z: QZ row pairs per block (2 QZ rows), at least 4 pairs for 64-byte runs
  static constexpr int QZ = pow2_div(N / 2, cmax(128 / T, 4));
  // padded line pitch for position-major exchange buffers (see pos_addr)
  static constexpr int PITCH_P = round_up(N + N / 16, 16) + (T < 16 ? T : 0);
  static constexpr int RT_PITCH = N + 1;  // real row pitch (floats) in zfront
};

// Plans of at most 32 threads a line, for passes whose lines may then be warp-local: the default
// plans, except 512 = 8 x 16 x 4 over 32 threads (16 values a thread)
template <int N>
struct PlanW : Plan<N> {};
template <>
struct PlanW<512> {
  static constexpr int NN = 512;
  static constexpr int T = 32;
  static constexpr int R[] = {8, 16, 4};
  static constexpr int S = 3;
};

// minimum resident blocks of the windowed inverse x passes: with radix-8 plans two blocks of 512
// threads (at most 64 registers); otherwise the general cap
template <int N>
constexpr int x_pass_minb() {
  constexpr int nth = Cfg<N>::T * Cfg<N>::BX;
  return (Cfg<N>::V <= 8 && nth >= 512) ? 2 : RG_MINB(nth);
}

// exchange-buffer index of position p of line b when threads walk positions (one pad slot
// every 16 positions breaks the stride-R write pattern of the first stages)
// For 192, 384 and 512 points an XOR of position bits 3-6 into bits 0-3 (a bijection within
// each 16-position group) spreads every exchange of the plan over all banks; for the other sizes
// the pad slot does.
template <int N>
__device__ __forceinline__ int pos_addr(int b, int p) {
  if constexpr (N == 192 || N == 384 || N == 512) return b * Cfg<N>::PITCH_P + (p ^ ((p >> 3) & 15));
  return b * Cfg<N>::PITCH_P + p + (p >> 4);
}
// exchange-buffer index when threads walk lines (B consecutive lines per position).  With
// B < 16 a half-warp spans 16/B threads of the first stage, whose outputs sit R0 positions
// apart; B extra slots after every R0 positions shift them onto different banks.
template <int N, int B>
__device__ __forceinline__ int line_addr(int p, int b) {
  constexpr int R0 = Plan<N>::R[0];
  if constexpr (B < 16) return p * B + b + B * (p / R0);
  return p * B + b;
}
template <int N, int B>
__host__ __device__ constexpr int line_buf() {
  constexpr int R0 = Plan<N>::R[0];
  return N * B + (B < 16 ? B * (N / R0 + 1) : 0);
}
// the same for a plan whose first radix is R0
template <int R0, int B>
__device__ __forceinline__ int line_addr_r0(int p, int b) {
  if constexpr (B < 16) return p * B + b + B * (p / R0);
  return p * B + b;
}
template <int N, int R0, int B>
__host__ __device__ constexpr int line_buf_r0() {
  return N * B + (B < 16 ? B * (N / R0 + 1) : 0);
}

// ---------------------------------------------------------------------------

// the forward z pass's launch shape: QF row pairs per block, one line of T threads each (the
// default plans: at 512 the 32-thread plan measured slower here, 6.9 against 5.6 ms a snapshot)
template <int N>
struct ZFCfg {
  using PL = Plan<N>;
  static constexpr int T = PL::T;
  static constexpr int QF = pow2_div(N / 2, cmax(256 / T, 1));
  static constexpr int NTH = T * QF;
  // the split reads rows qq of the transformed pairs at KN kz values a warp: a row pitch of KN mod
  // 16 values puts the warp's (row, kz) reads on distinct banks
  static constexpr int KN = 2 * QF >= 32 ? 1 : 32 / (2 * QF);
  static constexpr int ZP = round_up(Cfg<N>::PITCH_P, 16) + KN;
  static constexpr size_t smem() { return sizeof(cf) * (N + (size_t)QF * (Cfg<N>::PITCH_P + ZP)); }
};

template <int N>
__global__ void __launch_bounds__(ZFCfg<N>::NTH, RG_MINB(ZFCfg<N>::NTH))
    k_fwd_z(GridPtrs srcs, cf* __restrict__ dst_base, size_t dst_stride, const cf* __restrict__ g_tw) {
  using PL = typename ZFCfg<N>::PL;
  constexpr int T = ZFCfg<N>::T, Q = ZFCfg<N>::QF, NZ = Cfg<N>::NZ, PADW = Cfg<N>::PADW, PI = Cfg<N>::PITCH_P;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  cf* zbuf = xbuf + Q * PI;
  const float* src = static_cast<const float*>(pick(srcs, blockIdx.z));
  cf* dst = dst_base + blockIdx.z * dst_stride;
  const int x = blockIdx.y;
  const int y0 = blockIdx.x * 2 * Q;
  const int t = threadIdx.x % T, q = threadIdx.x / T;
  load_twiddles_p<PL>(s_tw, g_tw);
  __syncthreads();
  const float* r0 = src + ((size_t)x * N + y0 + 2 * q) * PADW;
  constexpr int ZP = ZFCfg<N>::ZP;
  auto zpos = [&](int qq, int p) { return qq * ZP + pos_addr<N>(0, p); };
  line_fft_p<PL, false, (T <= 32)>(   // warp barriers when a line fits a warp (its rows are its own)
      t, xbuf, s_tw, [&](int p, int) { return cf{__ldg(r0 + p), __ldg(r0 + PADW + p)}; },
      [&](int p) { return pos_addr<N>(q, p); }, [&](int p, cf v, int) { zbuf[zpos(q, p)] = v; });
  __syncthreads();
  // split Z = X(y) + i X(y+1) and store S[k][x][y0 .. y0 + 2Q)
  for (int i = threadIdx.x; i < NZ * 2 * Q; i += T * Q) {
    const int yy = i % (2 * Q), k = i / (2 * Q);
    const int qq = yy >> 1;
    const cf zk = zbuf[zpos(qq, k)];
    const cf zn = zbuf[zpos(qq, (N - k) % N)];
    cf out;
    if ((yy & 1) == 0) {
      out = cf{0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y)};  // (Z[k] + conj Z[N-k]) / 2
    } else {
      out = cf{0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x)};  // (Z[k] - conj Z[N-k]) / 2i
    }
    dst[((size_t)k * N + x) * N + y0 + yy] = out;
  }
}

// the y pass's launch shape: BY lines of T threads per block
template <int N>
struct YCfg {
  using PL = PlanW<N>;
  static constexpr int T = PL::T;
  static constexpr int BY = pow2_div(N, cmax(256 / T, 1));
  static constexpr int NTH = T * BY;
  static constexpr size_t smem() { return sizeof(cf) * (N + (size_t)BY * Cfg<N>::PITCH_P); }
};

// y pass over grids base + z * stride (z = blockIdx.z), in place.  A line's T <= 32 threads are
// consecutive lanes of one warp and its exchange row is its own: warp barriers.
template <int N, bool INV>
__global__ void __launch_bounds__(YCfg<N>::NTH, RG_MINB(YCfg<N>::NTH))
    k_pass_y(cf* __restrict__ base, size_t stride, const cf* __restrict__ g_tw) {
  using Y = YCfg<N>;
  using PL = typename Y::PL;
  constexpr int T = Y::T, B = Y::BY;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  cf* g = base + blockIdx.z * stride;
  const int kz = blockIdx.y;
  const int x0 = blockIdx.x * B;
  const int t = threadIdx.x % T, b = threadIdx.x / T;
  load_twiddles_p<PL>(s_tw, g_tw);
  __syncthreads();
  cf* line = g + ((size_t)kz * N + x0 + b) * N;
  line_fft_p<PL, INV, true>(
      t, xbuf, s_tw, [&](int p, int) { return line[p]; }, [&](int p) { return pos_addr<N>(b, p); },
      [&](int p, cf v, int) { line[p] = v; });
}

// the y pass over ng grids at base + g * stride
template <int N, bool INV>
inline cudaError_t launch_pass_y(cf* base, size_t stride, int ng, const cf* tw, cudaStream_t st) {
  using Y = YCfg<N>;
  cudaError_t e = cudaFuncSetAttribute(k_pass_y<N, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Y::smem());
  if (e != cudaSuccess) return e;
  k_pass_y<N, INV><<<dim3(N / Y::BY, Cfg<N>::NZ, ng), Y::NTH, Y::smem(), st>>>(base, stride, tw);
  return cudaGetLastError();
}

// forward x pass over grids base + z * stride, in place, scaled on store
template <int N>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::BX, RG_MINB(Cfg<N>::T* Cfg<N>::BX))
    k_pass_x_fwd(cf* __restrict__ base, size_t stride, const cf* __restrict__ g_tw, float scale) {
  constexpr int T = Cfg<N>::T, B = Cfg<N>::BX;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  cf* g = base + blockIdx.z * stride;
  const int kz = blockIdx.y;
  const int b = threadIdx.x % B, t = threadIdx.x / B;
  const size_t col = (size_t)kz * N * N + blockIdx.x * B + b;
  load_twiddles<N>(s_tw, g_tw);
  __syncthreads();
  line_fft<N, false>(
      t, xbuf, s_tw, [&](int p, int) { return g[col + (size_t)p * N]; }, [&](int p) { return line_addr<N, B>(p, b); },
      [&](int p, cf v) { g[col + (size_t)p * N] = cf{v.x * scale, v.y * scale}; });
}

// ---------------------------------------------------------------------------
// zfront: c2r of NG grids (work + g * stride) for rows [y0, y0 + 2 QZ) of plane x.  Real row
// r of grid g lands at rt[(g * 2 QZ + r) * RT_PITCH + z].  Ends with a block barrier.

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

template <int N>
constexpr size_t zfront_smem_bytes(int ng) {
  return sizeof(cf) * (N + (size_t)line_buf<N, Cfg<N>::QZ>()) +
         sizeof(float) * (size_t)ng * 2 * Cfg<N>::QZ * (N + 1);
}

template <int N, int NG>
__device__ __forceinline__ void zfront(const cf* __restrict__ work, size_t stride, const cf* s_tw, cf* xbuf,
                                       float* rt, int x, int y0) {
  constexpr int T = Cfg<N>::T, Q = Cfg<N>::QZ, RP = Cfg<N>::RT_PITCH;
  const int q = threadIdx.x % Q, t = threadIdx.x / Q;
  const size_t colpair = (size_t)x * N + y0 + 2 * q;
#pragma unroll
  for (int g = 0; g < NG; ++g) {
    const cf* src = work + g * stride;
    float* r0 = rt + (size_t)(g * 2 * Q + 2 * q) * RP;
    line_fft<N, true>(
        t, xbuf, s_tw, [&](int p, int) { return build_c2r_input<N>(src, colpair, p); },
        [&](int p) { return line_addr<N, Q>(p, q); },
        [&](int p, cf v) {
          r0[p] = v.x;
          r0[RP + p] = v.y;
        });
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// asynchronous global -> shared copies (cp.async, 16 bytes per instruction); the copies of a
// commit group complete in order, wait<n> leaves at most n groups in flight

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int n>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(n) : "memory");
}

// the Hermitian halves of rows [y0, y0 + 2Q) of plane x of one grid as a shared tile
// tile[k][j] = g[k][x][y0 + j], k <= N/2, j < 2Q, copied by the whole block
template <int N, int Q>
__device__ __forceinline__ void ztile_issue(cf* tile, const cf* __restrict__ g, int x, int y0, int nth) {
  constexpr int NZ = N / 2 + 1;
  for (int c = threadIdx.x; c < NZ * Q; c += nth) {
    const int k = c / Q, j = 2 * (c % Q);
    cp_async16(tile + k * 2 * Q + j, g + ((size_t)k * N + x) * N + y0 + j);
  }
}

// build_c2r_input from a shared tile (row pair q)
template <int N, int Q>
__device__ __forceinline__ cf ztile_c2r_input(const cf* tile, int q, int p) {
  const int k = p <= N / 2 ? p : N - p;
  const float4 ab = *reinterpret_cast<const float4*>(tile + k * 2 * Q + 2 * q);
  if (p == 0 || p == N / 2) return cf{ab.x, ab.z};
  if (p < N / 2) return cf{ab.x - ab.w, ab.y + ab.z};
  return cf{ab.x + ab.w, ab.z - ab.y};
}

template <int N>
constexpr size_t ztile_elems() {
  return (size_t)(N / 2 + 1) * 2 * Cfg<N>::QZ;
}

// c2r of one spectrum into a padded real grid (tests)
template <int N>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::QZ, RG_MINB(Cfg<N>::T* Cfg<N>::QZ))
    k_inv_z_padded(const cf* __restrict__ work, const cf* __restrict__ g_tw, float* __restrict__ out) {
  constexpr int T = Cfg<N>::T, Q = Cfg<N>::QZ, PADW = Cfg<N>::PADW;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  float* rt = reinterpret_cast<float*>(xbuf + line_buf<N, Q>());
  const int x = blockIdx.y, y0 = blockIdx.x * 2 * Q;
  load_twiddles<N>(s_tw, g_tw);
  __syncthreads();
  zfront<N, 1>(work, 0, s_tw, xbuf, rt, x, y0);
  for (int i = threadIdx.x; i < 2 * Q * N; i += T * Q) {
    const int z = i % N, r = i / N;
    out[((size_t)x * N + y0 + r) * PADW + z] = rt[r * (N + 1) + z];
  }
}

}  // namespace rg
