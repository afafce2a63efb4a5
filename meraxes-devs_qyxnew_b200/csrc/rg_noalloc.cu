// rg_filter_roundtrip_noalloc: the forward r2c + filter() + c2r round trip of
// rg_debug_filter_roundtrip, for callers that must not allocate device memory: a caller
// that has handed the device's memory to its own pool and sized it exactly, or a caller
// on a latency budget for which cudaMalloc's implicit device synchronisation is too
// costly.  The call makes no cudaMalloc / cudaFree and calls no allocating library; its
// working memory is one static __device__ array of RG_NOALLOC_SCRATCH_BYTES per device.
//
//   scratch layout (bytes, each region 256-byte aligned):
//     [0, S)        spectrum   S[kz][x][y], (N/2+1) N^2 complex, S = NC_MAX * 8
//     [S, 2S)       work       the filtered spectrum, same shape
//     [2S, 2S + 8M) twiddles   e^{-2 pi i k / N}, k < N  (M = RG_NOALLOC_MAX_GRID_DIM)
//   NC_MAX = (M/2 + 1) M^2.  Nothing in it has to start at zero: every element a call reads
//   was written earlier in the same call.
//
// Set-up: the first call on a device (with that device current) looks up the array's
// device address with cudaGetSymbolAddress and caches it together with the CUDA context it
// belongs to; later calls in the same context reuse it.  After cudaDeviceReset (or any
// other way the device's primary context is destroyed and made anew) the next call sees a
// different context and looks the address up again, so a stale address is never used.
// Make the first call on each device, and the first after a reset, before any stream
// capture begins.
//
// Two calls in flight at the same time on one device (different streams, or different
// host threads) share the scratch and race: the caller orders them, e.g. on one stream.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "rg_internal.h"
#include "rg_pass.cuh"

namespace rg {
namespace {

constexpr int NA_MAX = RG_NOALLOC_MAX_GRID_DIM;
constexpr size_t NA_NC_MAX = (size_t)(NA_MAX / 2 + 1) * NA_MAX * NA_MAX;
constexpr size_t NA_SPEC_OFF = 0;
constexpr size_t NA_WORK_OFF = NA_NC_MAX * sizeof(cf);
constexpr size_t NA_TW_OFF = 2 * NA_NC_MAX * sizeof(cf);
constexpr size_t NA_BYTES = NA_TW_OFF + (size_t)NA_MAX * sizeof(cf);
static_assert(NA_BYTES <= RG_NOALLOC_SCRATCH_BYTES, "scratch size constant too small");
static_assert(NA_WORK_OFF % 256 == 0 && NA_TW_OFF % 256 == 0, "scratch regions must stay 256-byte aligned");

__device__ __align__(256) unsigned char g_noalloc_scratch[RG_NOALLOC_SCRATCH_BYTES];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
void* g_na_base[NA_MAX_DEVICES] = {};
CUcontext g_na_ctx[NA_MAX_DEVICES] = {};

// the current driver context, through the runtime's driver entry point (no link-time
// dependency on libcuda); nullptr when it cannot be had, which forces a fresh look-up
CUcontext na_current_context() {
  using Fn = CUresult (*)(CUcontext*);
  static Fn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<Fn>(f);
  }();
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

// twiddles computed on the device in double, rounded to float (the host table of the
// context path is cos/sin in double rounded to float: the same values up to the last bit of
// the double results)
__global__ void k_na_twiddles(cf* tw, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double s, c;
  sincospi(-2.0 * (double)k / (double)n, &s, &c);
  tw[k] = cf{(float)c, (float)s};
}

// inverse x pass of one spectrum with the window of one radius evaluated in place (the
// closed forms of filter(), src/core/reionization.c:3404-3428, in double as the window
// table of the context path): the single-radius variant of the batched x pass
template <int N>
__global__ void __launch_bounds__(Cfg<N>::T* Cfg<N>::BX, RG_MINB(Cfg<N>::T* Cfg<N>::BX))
    k_na_inv_x(const cf* __restrict__ spec, cf* __restrict__ work, const cf* __restrict__ g_tw, double delta_k,
               double R, int ftype) {
  constexpr int T = Cfg<N>::T, B = Cfg<N>::BX, V = Cfg<N>::V;
  extern __shared__ cf smem[];
  cf* s_tw = smem;
  cf* xbuf = smem + N;
  const int kz = blockIdx.y;
  const int b = threadIdx.x % B, t = threadIdx.x / B;
  const int y = blockIdx.x * B + b;
  const size_t col = (size_t)kz * N * N + y;
  load_twiddles<N>(s_tw, g_tw);
  float wv[V];
  const int ny = y > N / 2 ? y - N : y;
#pragma unroll
  for (int sl = 0; sl < V; ++sl) {
    const int p = stage0_pos<N>(t, sl);
    const int nx = p > N / 2 ? p - N : p;
    const double kR = delta_k * sqrt((double)(nx * nx + ny * ny + kz * kz)) * R;
    double w = 1.0;
    if (ftype == 0) {
      if (kR > 1e-4) w = 3.0 * (sin(kR) / (kR * kR * kR) - cos(kR) / (kR * kR));
    } else if (ftype == 1) {
      if (kR * 0.413566994 > 1.0) w = 0.0;
    } else if (ftype == 2) {
      const double g = kR * 0.643;
      w = exp(-g * g / 2.0);
    }
    wv[sl] = (float)w;
  }
  __syncthreads();
  line_fft<N, true>(
      t, xbuf, s_tw,
      [&](int p, int sl) {
        const cf v = spec[col + (size_t)p * N];
        return cf{v.x * wv[sl], v.y * wv[sl]};
      },
      [&](int p) { return line_addr<N, B>(p, b); }, [&](int p, cf v) { work[col + (size_t)p * N] = v; });
}

template <int N>
constexpr size_t na_smem_fz() { return ZFCfg<N>::smem(); }
template <int N>
constexpr size_t na_smem_y() { return YCfg<N>::smem(); }
template <int N>
constexpr size_t na_smem_x() { return sizeof(cf) * (N + (size_t)line_buf<N, Cfg<N>::BX>()); }

template <int N>
cudaError_t na_roundtrip(unsigned char* base, const float* in, float* out, double box, double R, int ftype,
                         cudaStream_t st) {
  using C = Cfg<N>;
  // every launch fits the default 48 KB of dynamic shared memory, so no attribute is set
  static_assert(na_smem_fz<N>() <= 48 * 1024 && na_smem_y<N>() <= 48 * 1024 && na_smem_x<N>() <= 48 * 1024 &&
                    zfront_smem_bytes<N>(1) <= 48 * 1024,
                "no-alloc round trip expects default shared-memory limits");
  cf* spec = reinterpret_cast<cf*>(base + NA_SPEC_OFF);
  cf* work = reinterpret_cast<cf*>(base + NA_WORK_OFF);
  cf* tw = reinterpret_cast<cf*>(base + NA_TW_OFF);
  const size_t nc = (size_t)C::NZ * N * N;
  k_na_twiddles<<<1, N, 0, st>>>(tw, N);
  GridPtrs srcs{};
  srcs.p[0] = in;
  k_fwd_z<N><<<dim3(N / (2 * ZFCfg<N>::QF), N, 1), ZFCfg<N>::NTH, na_smem_fz<N>(), st>>>(srcs, spec, nc, tw);
  k_pass_y<N, false><<<dim3(N / YCfg<N>::BY, C::NZ, 1), YCfg<N>::NTH, na_smem_y<N>(), st>>>(spec, nc, tw);
  k_pass_x_fwd<N><<<dim3(N / C::BX, C::NZ, 1), C::T * C::BX, na_smem_x<N>(), st>>>(
      spec, nc, tw, (float)(1.0 / ((double)N * N * N)));
  // filter_type < 0: the window is 1 everywhere (no filter)
  k_na_inv_x<N><<<dim3(N / C::BX, C::NZ), C::T * C::BX, na_smem_x<N>(), st>>>(spec, work, tw, 2.0 * M_PI / box, R,
                                                                               ftype);
  k_pass_y<N, true><<<dim3(N / YCfg<N>::BY, C::NZ, 1), YCfg<N>::NTH, na_smem_y<N>(), st>>>(work, nc, tw);
  k_inv_z_padded<N><<<dim3(N / (2 * C::QZ), N), C::T * C::QZ, zfront_smem_bytes<N>(1), st>>>(work, tw, out);
  return cudaGetLastError();
}

int na_fail(char* errbuf, size_t errlen, int status, const char* msg) {
  if (errbuf && errlen) {
    std::strncpy(errbuf, msg, errlen - 1);
    errbuf[errlen - 1] = '\0';
  }
  return status;
}

}  // namespace
}  // namespace rg

extern "C" int rg_filter_roundtrip_noalloc(const rg_params* p, const float* d_in_padded, float* d_out_padded,
                                           double R, int filter_type, void* stream, char* errbuf, size_t errlen) {
  using namespace rg;
  if (errbuf && errlen) errbuf[0] = '\0';
  if (!p || !d_in_padded || !d_out_padded) return na_fail(errbuf, errlen, RG_EINVAL, "null argument");
  if (filter_type > 2) return na_fail(errbuf, errlen, RG_EINVAL, "filter_type must be <= 2 (< 0 = no filter)");
  if (!(p->BoxSize > 0)) return na_fail(errbuf, errlen, RG_EINVAL, "BoxSize must be positive");
  const int N = p->ReionGridDim;
  if (N > NA_MAX) {
    char msg[160];
    std::snprintf(msg, sizeof(msg),
                  "ReionGridDim %d exceeds RG_NOALLOC_MAX_GRID_DIM (%d), the largest grid the static scratch holds",
                  N, NA_MAX);
    return na_fail(errbuf, errlen, RG_EUNSUPPORTED, msg);
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES)
    return na_fail(errbuf, errlen, RG_ENODEV, "no usable current CUDA device");
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_na_mutex);
    const CUcontext cur = na_current_context();
    if (!g_na_base[dev] || !cur || cur != g_na_ctx[dev]) {
      g_na_base[dev] = nullptr;
      g_na_ctx[dev] = nullptr;
      void* addr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
      if (e != cudaSuccess) return na_fail(errbuf, errlen, RG_ECUDA, cudaGetErrorString(e));
      // cudaGetSymbolAddress makes the primary context current if none was: read it again
      g_na_ctx[dev] = na_current_context();
      g_na_base[dev] = addr;
    }
    base = g_na_base[dev];
  }
  unsigned char* b = static_cast<unsigned char*>(base);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  switch (N) {
    case 8: e = na_roundtrip<8>(b, d_in_padded, d_out_padded, p->BoxSize, R, filter_type, st); break;
    case 16: e = na_roundtrip<16>(b, d_in_padded, d_out_padded, p->BoxSize, R, filter_type, st); break;
    case 24: e = na_roundtrip<24>(b, d_in_padded, d_out_padded, p->BoxSize, R, filter_type, st); break;
    case 32: e = na_roundtrip<32>(b, d_in_padded, d_out_padded, p->BoxSize, R, filter_type, st); break;
    case 48: e = na_roundtrip<48>(b, d_in_padded, d_out_padded, p->BoxSize, R, filter_type, st); break;
    case 64: e = na_roundtrip<64>(b, d_in_padded, d_out_padded, p->BoxSize, R, filter_type, st); break;
    default:
      return na_fail(errbuf, errlen, RG_EUNSUPPORTED, "ReionGridDim must be one of 8, 16, 24, 32, 48, 64");
  }
  if (e != cudaSuccess) return na_fail(errbuf, errlen, RG_ECUDA, cudaGetErrorString(e));
  return RG_OK;
}
