// The inverse x and y passes of a batch of filtered grids as ONE persistent kernel whose
// intermediate plane stays in L2.
//
// A job is one kz plane of one radius (or shell) of the batch, over all of the batch's grids:
// the x pass of the job (window x spectrum, c2c along x) writes the plane into the work buffer,
// the y pass (c2c along y) transforms it there in place.  Run as two kernels over the whole
// batch, every plane crosses HBM three times (x store, y load, y store); here the y pass of a
// job is issued shortly after its x pass, so the y loads hit the x stores in L2 and the plane
// reaches HBM once.
//
// Work items are handed out by one atomic counter in a fixed sequence of segments of M items
// (M = N / B column groups or line groups):
//
//   X(0) .. X(L-1), X(L), Y(0), X(L+1), Y(1), ..., X(J-1), Y(J-L-1), Y(J-L) .. Y(J-1)
//
// (J jobs, lag L).  Jobs run kz-major, radius-minor, so a spectrum plane is read from HBM by the
// first radius and from L2 by the others.  A Y item waits (thread 0, acquire load, bounded) until
// all M X items of its job have signalled (release after a block barrier).  Every X item of a
// job precedes its Y items in the sequence and X items wait on nothing, so the smallest
// unfinished item can always finish: the kernel needs no co-resident grid and no cooperative
// launch.  A wait that runs out sets the error word and the item goes on (the host reports
// RG_ETIMEDOUT); no wait is unbounded.
//
// An X item's input, the spectrum tile (all x, its B columns) of each grid, arrives in shared
// memory by tensor loads (TMA, mbarrier completion) into two alternating buffers: the load of the
// next grid's tile, or of the next X item's first tile, is issued before the current tile is
// transformed, so the loads overlap the transforms.  A buffer is also the FFT exchange buffer
// of the tile it holds.
#pragma once

#include <algorithm>
#include <string>

#include "rg_internal.h"
#include "rg_pass.cuh"
#include "rg_tma.cuh"

namespace rg {

struct XYSched {
  int nr;            // radii (or shells) per kz plane
  int M;             // items per segment
  int J;             // jobs = (N/2 + 1) * nr
  int L;             // lag of the Y segments behind the X segments, 1 <= L <= J
  int total;         // 2 J M
  uint32_t* ctr;     // item counter (zero at launch)
  uint32_t* done;    // [J] finished X items per job (zero at launch)
  uint32_t* err;     // set to 1 when a wait runs out
  int max_polls;     // polls of a Y item's wait before it gives up
  int signal;        // X items signal their job (0 only in the forced-timeout test)
};

__device__ __forceinline__ void xy_decode(const XYSched& s, int seg, bool& is_y, int& job) {
  if (seg < s.L) {
    is_y = false;
    job = seg;
    return;
  }
  const int u = seg - s.L;
  const int mid = 2 * (s.J - s.L);
  if (u < mid) {
    is_y = (u & 1) != 0;
    job = is_y ? (u >> 1) : s.L + (u >> 1);
  } else {
    is_y = true;
    job = s.J - s.L + (u - mid);
  }
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// thread 0 only: wait until job's X items have all signalled (at most max_polls + 1 checks)
__device__ __forceinline__ void xy_wait(const XYSched& s, int job) {
  for (int i = 0;; ++i) {
    if (ld_acquire_u32(s.done + job) >= (uint32_t)s.M) return;
    if (i >= s.max_polls) break;
    __nanosleep(64);
  }
  atomicExch(s.err, 1u);
}

// The fused pass's plans (PlanW): at 512, 8 x 16 x 4 over 32 threads a line measured faster than
// 8 x 8 x 8 over 64 (77.2 against 81.3 ms for the 61 radii of a 512^3 snapshot; 16 x 16 x 2 took
// 78.5 ms, and 16 columns an item instead of 8 took 85-87 ms), and its Y lines are warp-local.
template <int N>
struct XYF {
  using PL = PlanW<N>;
  static constexpr int T = PL::T;
  static constexpr int V = N / T;
  static constexpr int B = Cfg<N>::BX;   // columns per X item, lines per Y item
  static constexpr int MINB = N != 512 ? x_pass_minb<N>() : 2;
  static constexpr int NTH = T * B;
  static constexpr int M = N / B;
  static constexpr int XROWS = N <= 256 ? N : N / 2;   // x rows per tensor box (box dimensions <= 256)
  static constexpr int NXB = N / XROWS;
  // a buffer: an X tile [x][B columns], then its exchange buffer; or a Y item's exchange buffer
  static constexpr int TB = round_up(cmax(cmax(line_buf_r0<N, PL::R[0], B>(), B * Cfg<N>::PITCH_P), N * B), 16);
  static constexpr int ZB = 2;
  static constexpr uint32_t TX = (uint32_t)(N * B * sizeof(cf));
  static constexpr size_t smem() { return 128 + sizeof(cf) * ((size_t)ZB * TB + N) + sizeof(uint64_t) * ZB; }
  static_assert((XROWS * B * sizeof(cf)) % 128 == 0, "second x box off a 128-byte boundary");
};

__device__ __forceinline__ cf ldcg_cf(const cf* p) {
  const float2 v = __ldcg(reinterpret_cast<const float2*>(p));
  return cf{v.x, v.y};
}

// release the finished X item: the block barrier before it orders the block's stores
__device__ __forceinline__ void xy_signal(uint32_t* p) {
  __threadfence();
  atomicAdd(p, 1u);
}

// Op (by value) describes the batch:
//   int grids() const                         grids per job
//   bool filtered(int r) const                radius r is windowed
//   const float* wrow(int r) const            its window row W[n2]
//   int cutoff(int r) const                   >= -1: the row is the step W = (n2 <= cutoff), read
//                                             without gathers (sharp-k); < -1: read the row
//   cf* out(int r, int g) const               output grid (plane kz at kz N^2)
// The X input of grid g is W(k) * spectrum_g(k); the spectra are the tensor `smap` (floats, y
// innermost, then x, then kz of grid g at g (N/2 + 1) + kz).
template <int N, class Op>
__global__ void __launch_bounds__(XYF<N>::NTH, XYF<N>::MINB)
    k_xy_fused(XYSched sch, Op op, const __grid_constant__ CUtensorMap smap, const cf* __restrict__ g_tw) {
  using F = XYF<N>;
  using PL = typename F::PL;
  constexpr int T = F::T, B = F::B, V = F::V, TB = F::TB, NZ = N / 2 + 1;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  cf* bufs = reinterpret_cast<cf*>(sm);
  cf* s_tw = bufs + F::ZB * TB;
  uint64_t* bars = reinterpret_cast<uint64_t*>(s_tw + N);
  __shared__ int s_item[2];
  __shared__ int s_pref[2];   // the next item's first tile is in flight
  if (threadIdx.x == 0) {
    for (int b = 0; b < F::ZB; ++b) mbar_init(&bars[b], 1);
    mbar_init_fence();
  }
  load_twiddles_p<PL>(s_tw, g_tw);
  if (threadIdx.x == 0) {
    s_item[0] = (int)atomicAdd(sch.ctr, 1u);
    s_pref[0] = 0;
  }
  __syncthreads();
  const int ng = op.grids();
  // thread 0: the tile of grid g for the X item `itm` into buffer b
  auto issue = [&](int itm, int g, int b) {
    const int seg = itm / sch.M, k = itm - seg * sch.M;
    bool is_y;
    int job;
    xy_decode(sch, seg, is_y, job);
    const int kz = job / sch.nr;
    mbar_arrive_expect_tx(&bars[b], F::TX);
#pragma unroll
    for (int xb = 0; xb < F::NXB; ++xb)
      tma_load_3d(bufs + b * TB + xb * F::XROWS * B, &smap, 2 * k * B, xb * F::XROWS, g * NZ + kz, &bars[b]);
  };
  auto is_x_item = [&](int itm) {
    if (itm >= sch.total) return false;
    bool is_y;
    int job;
    xy_decode(sch, itm / sch.M, is_y, job);
    return !is_y;
  };
  int it = 0;
  int item = s_item[0];
  uint32_t xu = 0;          // X units (item, grid) this block has started: unit u uses buffer u & 1
  bool waited = true;
  while (item < sch.total) {
    int nxt = 0;
    if (threadIdx.x == 0) nxt = (int)atomicAdd(sch.ctr, 1u);   // the next item, fetched early
    const bool pref = s_pref[it & 1] != 0;
    const int seg = item / sch.M, k = item - seg * sch.M;
    bool is_y;
    int job;
    xy_decode(sch, seg, is_y, job);
    const int kz = job / sch.nr, r = job - kz * sch.nr;
    const size_t plane = (size_t)kz * N * N;
    int next_pref = 0;
    if (!is_y) {
      const int bcol = threadIdx.x % B, t = threadIdx.x / B;
      const int y = k * B + bcol;
      const size_t col = plane + y;
      float wv[V];
#pragma unroll
      for (int sl = 0; sl < V; ++sl) wv[sl] = 1.f;
      if (op.filtered(r)) {
        const float* wr = op.wrow(r);
        const int cut = op.cutoff(r);
        const int ny = y > N / 2 ? y - N : y;
#pragma unroll
        for (int sl = 0; sl < V; ++sl) {
          const int p = stage0_pos<PL>(t, sl);
          const int nx = p > N / 2 ? p - N : p;
          const int n2 = nx * nx + ny * ny + kz * kz;
          wv[sl] = cut >= -1 ? (n2 <= cut ? 1.f : 0.f) : __ldg(wr + n2);
        }
      }
      for (int g = 0; g < ng; ++g, ++xu) {
        const int b = (int)(xu & 1u);
        if (threadIdx.x == 0) {
          if (g == 0 && !pref) issue(item, 0, b);
          // the next unit's tile into the other buffer (its previous unit has ended)
          if (g + 1 < ng) {
            issue(item, g + 1, b ^ 1);
          } else if (is_x_item(nxt)) {
            issue(nxt, 0, b ^ 1);
            next_pref = 1;
          }
        }
        if (!mbar_wait(&bars[b], (xu >> 1) & 1u, 1 << 22)) waited = false;
        cf* tile = bufs + b * TB;
        cf* dst = op.out(r, g);
        line_fft_p<PL, true>(
            t, tile, s_tw,
            [&](int p, int sl) {
              const cf v = tile[p * B + bcol];
              return cf{v.x * wv[sl], v.y * wv[sl]};
            },
            [&](int p) { return line_addr_r0<PL::R[0], B>(p, bcol); },
            [&](int p, cf v, int) { dst[col + (size_t)p * N] = v; });
        fence_proxy_async_smem();
        __syncthreads();   // every store of the unit is issued; its buffer may be refilled
      }
      if (threadIdx.x == 0 && sch.signal) xy_signal(sch.done + job);
    } else {
      if (threadIdx.x == 0) xy_wait(sch, job);
      __syncthreads();
      const int t = threadIdx.x % T, b = threadIdx.x / T;
      const size_t row = plane + (size_t)(k * B + b) * N;
      // a line's T <= 32 threads are consecutive lanes of one warp, its exchange rows its own
      for (int g = 0; g < ng; ++g) {
        cf* line = op.out(r, g) + row;
        line_fft_p<PL, true, (T <= 32)>(
            t, bufs, s_tw, [&](int p, int) { return ldcg_cf(line + p); }, [&](int p) { return pos_addr<N>(b, p); },
            [&](int p, cf v, int) { line[p] = v; });
      }
      fence_proxy_async_smem();   // the exchange buffer is a tile buffer of later X items
    }
    if (threadIdx.x == 0) {
      s_item[(it + 1) & 1] = nxt;
      s_pref[(it + 1) & 1] = next_pref;
    }
    __syncthreads();
    ++it;
    item = s_item[it & 1];
  }
  if (!waited && threadIdx.x % 32 == 0) atomicExch(sch.err, 1u);
}

// Launch the fused pass of one batch of nr radii (or shells); the control words must have been
// sized by xy_ctrl_reset for at least (N/2 + 1) nr jobs.
template <int N, class Op>
int launch_xy_fused(rg_context* ctx, const Op& op, const cf* spec, int nspec, int nr, const char* name,
                    double alg_bytes, cudaStream_t st) {
  using F = XYF<N>;
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  // the nspec spectra (S[kz][x][y], one after another) as a 3-D float tensor
  CUtensorMap smap;
  const uint64_t dims[3] = {2ull * N, (uint64_t)N, (uint64_t)Cfg<N>::NZ * nspec};
  const uint64_t strides[2] = {8ull * N, 8ull * N * N};
  const uint32_t box[3] = {2u * F::B, (uint32_t)F::XROWS, 1u};
  const int mrc = tma_map_3d(&smap, spec, dims, strides, box);
  if (mrc != 0) return set_error(ctx, RG_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(mrc) + ")");
  const int J = Cfg<N>::NZ * nr;
  if (nr < 1 || (size_t)J + 2 > ctx->xy_ctrl_elems) return set_error(ctx, RG_EINVAL, "fused x/y pass: batch too large");
  auto kern = k_xy_fused<N, Op>;
  RG_CUDA_TRY(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F::smem()));
  int per_sm = 0;
  RG_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, F::NTH, F::smem()));
  const int grid = std::max(per_sm, 1) * ctx->num_sms;
  XYSched s;
  s.nr = nr;
  s.M = F::M;
  s.J = J;
  // Y(j) is handed out (2L + 1) M items after X(j) starts; with `grid` blocks in flight that is
  // about when X(j) completes for L = grid / (2M), one more for slack
  s.L = std::min(J, (grid + 2 * F::M - 1) / (2 * F::M) + 1);
  s.total = 2 * J * F::M;
  s.err = ctx->xy_ctrl;
  s.max_polls = ctx->xy_poll_limit;
  s.signal = ctx->xy_signal;
  s.ctr = ctx->xy_ctrl + 1;
  s.done = ctx->xy_ctrl + 2;
  RG_CUDA_TRY(ctx, cudaMemsetAsync(s.ctr, 0, sizeof(uint32_t) * ((size_t)J + 1), st));
  prof_begin(ctx, name, st);
  kern<<<std::min(grid, s.total), F::NTH, F::smem(), st>>>(s, op, smap, tw);
  prof_end(ctx, alg_bytes, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

}  // namespace rg
