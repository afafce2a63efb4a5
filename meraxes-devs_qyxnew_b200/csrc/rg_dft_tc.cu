// The split-BF16 tensor-core form of a DFT pass, against the FP32 register form the step uses.
//
// One c2c pass along y (the contiguous axis of the spectra S[kz][x][y]) over whole spectra, for
// ReionGridDim 256, as the four-step factorisation 256 = 16 x 16 of each line:
//   Y[k1][n2]      = sum_n1 x[16 n1 + n2] w16^(n1 k1)      (radix-16 stage 1)
//   Y'[k1][n2]     = Y[k1][n2] w256^(n2 k1)                 (twiddle, FP32)
//   X[k1 + 16 k2]  = sum_n2 Y'[k1][n2] w16^(n2 k2)          (radix-16 stage 2)
// Each radix-16 stage of a tile of 8 lines is one matrix product D[128 x 32] = A[128 x 32] B^T,
// rows = (line, the other index), K = the 16 complex inputs as 32 reals, N = the 16 complex
// outputs: the 32 x 32 real form of the DFT-16 matrix.  A and B are each split into BF16 hi and
// lo parts (v = hi + lo to about 2^-17 relative) and D = Ahi Bhi + Alo Bhi + Ahi Blo is
// accumulated in FP32 in tensor memory by tcgen05.mma (kind::f16, M = 128, N = 32, K = 16 per
// instruction, both operands K-major in shared memory without swizzle).  The two-part operands
// (about 16 significant bits) leave about 4e-6 relative error per pass; the dropped Alo Blo term
// adds little.  One thread (TMEM lane) per matrix row reads its 32 accumulators back with
// tcgen05.ld.
//
// It replaces nothing of the reference's code by itself: the reference transforms with FFTW
// (find_HII_bubbles.c:351-370, ComputeTs.c:480-581), whose y stage both forms implement.  It is
// here to measure whether tensor cores help a pass of this path; the step keeps the FP32 form.
#include <cuda_bf16.h>

#include "rg_internal.h"
#include "rg_pass.cuh"
#include "rg_tma.cuh"

namespace rg {

namespace {

constexpr int TC_N = 256;        // line length
constexpr int TC_L = 8;          // lines per tile (8 lines x 16 = 128 matrix rows)
constexpr int TC_NT = 128;       // threads: one per matrix row and TMEM lane
constexpr int TC_COLS = 32;      // TMEM columns: 32 FP32 accumulators per row
constexpr uint32_t TC_LBO = 128; // operand layout: byte stride of 8 x 16-byte core matrices along K
constexpr uint32_t TC_SBO = 512; //   and along M/N (a row group of 8 holds K = 32 -> 4 core matrices)
constexpr int TC_YP = 17;        // pitch (complex) of the transposition buffer's rows
constexpr int TC_BLOCKS_PER_SM = 4;   // 4 x 32 TMEM columns of the SM's 512
constexpr int TC_WAIT_LIMIT = 1 << 22;

// shared memory (bytes from a 1024-byte aligned base)
constexpr uint32_t OFF_AHI = 0, OFF_ALO = 8192, OFF_BHI = 16384, OFF_BLO = 18432, OFF_W = 20480,
                   OFF_Y = 22528, OFF_BAR = OFF_Y + 128 * TC_YP * 8, OFF_SLOT = OFF_BAR + 8,
                   TC_SMEM = OFF_SLOT + 8 + 1024;

// instruction descriptor: D FP32, A and B BF16, both K-major, N = 32, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_COLS >> 3) << 17) |
                              ((uint32_t)(128 >> 4) << 24);

// byte offset of element (row, k) of a K-major operand with K = 32 (no swizzle)
__device__ __forceinline__ uint32_t op_off(int row, int k) {
  return (uint32_t)(row >> 3) * TC_SBO + (uint32_t)(k >> 3) * TC_LBO + (uint32_t)(row & 7) * 16u +
         (uint32_t)(k & 7) * 2u;
}

// shared-memory matrix descriptor (sm_100 form: version 1, no swizzle)
__device__ __forceinline__ uint64_t op_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((TC_LBO >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((TC_SBO >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(TC_IDESC), "r"(acc)
      : "memory");
}

// arrive on the barrier when every earlier tcgen05 operation of this thread has completed
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// this warp's 32 TMEM lanes, 32 columns from `taddr`, waited for in the same statement
__device__ __forceinline__ void tc_load32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 h) { return *reinterpret_cast<uint32_t*>(&h); }

// row `row` of the hi and lo operands from 16 complex values (k = 2 n + {0 re, 1 im})
__device__ __forceinline__ void put_row(unsigned char* a_hi, unsigned char* a_lo, int row, const cf (&v)[16]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const cf x = v[4 * c + i];
      const __nv_bfloat162 hi = __floats2bfloat162_rn(x.x, x.y);
      const float2 hf = __bfloat1622float2(hi);
      h[i] = bf2_bits(hi);
      l[i] = bf2_bits(__floats2bfloat162_rn(x.x - hf.x, x.y - hf.y));
    }
    const uint32_t o = op_off(row, 8 * c);
    *reinterpret_cast<uint4*>(a_hi + o) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(a_lo + o) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

// one radix-16 stage of the tile: D = Ahi Bhi + Alo Bhi + Ahi Blo (K = 32 as two K = 16 steps)
__device__ __forceinline__ void issue_stage(uint32_t tmem, uint32_t sbase, uint32_t bar) {
  const uint32_t as[3] = {sbase + OFF_AHI, sbase + OFF_ALO, sbase + OFF_AHI};
  const uint32_t bs[3] = {sbase + OFF_BHI, sbase + OFF_BHI, sbase + OFF_BLO};
#pragma unroll
  for (int t = 0; t < 3; ++t)
#pragma unroll
    for (int s = 0; s < 2; ++s)
      tc_mma(tmem, op_desc(as[t] + s * 2 * TC_LBO), op_desc(bs[t] + s * 2 * TC_LBO), (t | s) ? 1u : 0u);
  tc_commit(bar);
}

// tiles of TC_L consecutive lines of the grids base + g * stride (g < ngrids), persistent blocks
template <bool INV>
__global__ void __launch_bounds__(TC_NT, TC_BLOCKS_PER_SM)
    k_pass_y_tc(cf* __restrict__ base, size_t stride, int ngrids, uint32_t* err) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const uint32_t sbase = smem_u32(sm);
  unsigned char* a_hi = sm + OFF_AHI;
  unsigned char* a_lo = sm + OFF_ALO;
  cf* s_w = reinterpret_cast<cf*>(sm + OFF_W);
  cf* ybuf = reinterpret_cast<cf*>(sm + OFF_Y);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + OFF_BAR);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + OFF_SLOT);
  const int t = threadIdx.x, warp = t >> 5;
  const double sg = INV ? 1.0 : -1.0;

  if (t == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"((uint32_t)TC_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // the DFT-16 matrix in its 32 x 32 real form, hi and lo: row j = (kout, re/im), column
  // k = (n, re/im); and the 256 twiddles w256^j
  for (int i = t; i < 32 * 32; i += TC_NT) {
    const int j = i >> 5, k = i & 31;
    const int m = ((j >> 1) * (k >> 1)) & 15;
    double sn, cs;
    sincospi(m / 8.0, &sn, &cs);
    sn *= sg;
    const double v = (j & 1) ? ((k & 1) ? cs : sn) : ((k & 1) ? -sn : cs);
    const __nv_bfloat16 hi = __double2bfloat16(v);
    const __nv_bfloat16 lo = __double2bfloat16(v - (double)__bfloat162float(hi));
    *reinterpret_cast<__nv_bfloat16*>(sm + OFF_BHI + op_off(j, k)) = hi;
    *reinterpret_cast<__nv_bfloat16*>(sm + OFF_BLO + op_off(j, k)) = lo;
  }
  for (int j = t; j < TC_N; j += TC_NT) {
    double sn, cs;
    sincospi(j / 128.0, &sn, &cs);
    s_w[j] = cf{(float)cs, (float)(sg * sn)};
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot;
  const uint32_t tlane = tmem + ((uint32_t)(warp * 32) << 16);

  constexpr int NZ = TC_N / 2 + 1;
  const int tiles_per_grid = NZ * TC_N / TC_L;
  const int ntiles = ngrids * tiles_per_grid;
  const int l = t >> 4, n = t & 15;   // this thread's line of the tile and its 16-index
  uint32_t phase = 0;
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int g = tile / tiles_per_grid;
    cf* lines = base + (size_t)g * stride + (size_t)(tile - g * tiles_per_grid) * TC_L * TC_N;
    cf* line = lines + l * TC_N;
    cf v[16];
    // stage 1 operand: row (l, n2 = n), inputs x[16 n1 + n2]
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = line[16 * i + n];
    put_row(a_hi, a_lo, t, v);
    fence_proxy_async_smem();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      issue_stage(tmem, sbase, smem_u32(bar));
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, TC_WAIT_LIMIT));
    phase ^= 1u;
    if (!ok) break;
    tc_fence_after();
    float d[32];
    tc_load32(tlane, d);
    // twiddle, then the transposition to rows (l, k1) through shared memory
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) {
      const cf w = s_w[n * k1];
      ybuf[(l * 16 + k1) * TC_YP + n] = cf{d[2 * k1] * w.x - d[2 * k1 + 1] * w.y, d[2 * k1] * w.y + d[2 * k1 + 1] * w.x};
    }
    tc_fence_before();
    __syncthreads();
    // stage 2 operand: row (l, k1 = n), inputs Y'[k1][n2]
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = ybuf[t * TC_YP + i];
    put_row(a_hi, a_lo, t, v);
    fence_proxy_async_smem();
    __syncthreads();
    if (t == 0) {
      tc_fence_after();
      issue_stage(tmem, sbase, smem_u32(bar));
    }
    ok = __syncthreads_and(mbar_wait(bar, phase, TC_WAIT_LIMIT));
    phase ^= 1u;
    if (!ok) break;
    tc_fence_after();
    tc_load32(tlane, d);
    // output row (l, k1 = n): X[k1 + 16 k2]
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) line[n + 16 * k2] = cf{d[2 * k2], d[2 * k2 + 1]};
    tc_fence_before();
  }
  if (!ok) {
    if (t == 0) atomicExch(err, 1u);
    // the stage in flight: let it finish (bounded) before the tensor memory is released
    mbar_wait(bar, phase ^ 1u, TC_WAIT_LIMIT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TC_COLS)
                 : "memory");
  }
}

template <typename K>
cudaError_t set_smem(K kernel, size_t smem) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <bool INV>
int launch_tc(rg_context* ctx, cf* spec, size_t stride, int ng, cudaStream_t st) {
  auto kern = k_pass_y_tc<INV>;
  RG_CUDA_TRY(ctx, set_smem(kern, TC_SMEM));
  // persistent blocks: TC_BLOCKS_PER_SM per SM (shared memory allows five; tensor memory, 32 of
  // the SM's 512 columns a block, sixteen).  Blocks are independent, so any that do not fit at
  // once simply start later.
  static_assert(TC_BLOCKS_PER_SM * TC_COLS <= 512, "tensor memory columns per SM");
  const int ntiles = ng * ((TC_N / 2 + 1) * TC_N / TC_L);
  const int grid = std::min(ntiles, TC_BLOCKS_PER_SM * ctx->num_sms);
  int rc = xy_ctrl_reset(ctx, 0, st);
  if (rc) return rc;
  prof_begin(ctx, "dft_y_tc_bf16x3", st);
  kern<<<grid, TC_NT, TC_SMEM, st>>>(spec, stride, ng, ctx->xy_ctrl);
  prof_end(ctx, ng * 16.0 * (double)stride, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

template <bool INV>
int launch_fp32(rg_context* ctx, cf* spec, size_t stride, int ng, cudaStream_t st) {
  constexpr int N = TC_N;
  const cf* tw;
  int rc = twiddles_for(ctx, N, &tw);
  if (rc) return rc;
  prof_begin(ctx, "dft_y_fp32", st);
  RG_CUDA_TRY(ctx, (launch_pass_y<N, INV>(spec, stride, ng, tw, st)));
  prof_end(ctx, ng * 16.0 * (double)stride, st);
  return RG_OK;
}

}  // namespace

}  // namespace rg

using namespace rg;

extern "C" int rg_dft_y_pass(rg_context* ctx, void* spec, int n_grids, int inverse, int impl) {
  if (!ctx || !spec || n_grids < 0) return RG_EINVAL;
  if (impl != RG_DFT_FP32 && impl != RG_DFT_TC_BF16X3) return set_error(ctx, RG_EINVAL, "unknown DFT implementation");
  if (ctx->N != TC_N) return set_error(ctx, RG_EUNSUPPORTED, "rg_dft_y_pass: ReionGridDim 256 only");
  if (reinterpret_cast<uintptr_t>(spec) % 16) return set_error(ctx, RG_EINVAL, "rg_dft_y_pass: spec not 16-byte aligned");
  if (n_grids == 0) return RG_OK;
  RG_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t stride = (size_t)(TC_N / 2 + 1) * TC_N * TC_N;
  cf* s = reinterpret_cast<cf*>(spec);
  int rc;
  if (impl == RG_DFT_FP32)
    rc = inverse ? launch_fp32<true>(ctx, s, stride, n_grids, st) : launch_fp32<false>(ctx, s, stride, n_grids, st);
  else
    rc = inverse ? launch_tc<true>(ctx, s, stride, n_grids, st) : launch_tc<false>(ctx, s, stride, n_grids, st);
  if (rc) return rc;
  if (impl == RG_DFT_TC_BF16X3) {
    uint32_t err = 0;
    RG_CUDA_TRY(ctx, cudaMemcpyAsync(&err, ctx->xy_ctrl, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (err) return set_error(ctx, RG_ETIMEDOUT, "tensor-core y pass: a wait for a matrix product ran out");
  }
  return RG_OK;
}
