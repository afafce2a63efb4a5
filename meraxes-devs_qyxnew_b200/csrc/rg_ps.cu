// The callers next to the step on the output and input sides, on the library's transforms:
//
//   * the 21-cm power spectrum, Compute_PS() (src/core/ComputePowerSpectrum.c:44-255), which
//     dracarys.c:393-394 runs on delta_T right after ComputeBrightnessTemperatureBox(); its bin
//     count is Initialise_PowerSpectrum() (ComputePowerSpectrum.c:18-42);
//   * smooth_grid() (src/core/read_grids.c:127-165): forward transform, / N^3, real-space
//     top-hat of radius BoxSize / ReionGridDim / 2, inverse transform, applied to a grid read at
//     a finer resolution before it is subsampled.
//
// Power spectrum on the device: one pass sums delta_T (FP64 per block), one pass writes the
// padded real field ((delta_T / ave - 1) V / N^3) ave, the r2c transform (unnormalised, as
// FFTW's), then one pass over the Hermitian modes bins k^3 |delta_k|^2 / (2 pi^2 V), k and the
// mode count into per-block FP64 partials that the host adds in block order.  The modes' |k| and
// the bin edges are formed in float exactly as the reference does (products and sums rounded
// separately, the square root in double), so every mode lands in the reference's bin.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "rg_internal.h"
#include "rg_pass.cuh"

namespace rg {

constexpr int PS_NT = 256;
constexpr int PS_MAXBINS = 64;

struct PsBins {
  float ceil[PS_MAXBINS];   // upper edge of bin i; its lower edge is ceil[i - 1] (0 for bin 0)
  int nb;
  float dk;                 // 2 pi / (BoxSize / h), float as in the reference
  double norm;              // 1 / (2 pi^2 V), V = powf(BoxSize / h, 3)
};

// the bin edges and count of Initialise_PowerSpectrum / Compute_PS (float arithmetic)
static PsBins ps_bins(const rg_params* p) {
  PsBins b;
  std::memset(&b, 0, sizeof(b));
  const double box_size = p->BoxSize / p->Hubble_h;  // Mpc
  const float k_factor = 1.35f;
  b.dk = (float)(2. * M_PI / box_size);
  const float k_max = b.dk * p->ReionGridDim;
  float k_ceil = b.dk;
  while (k_ceil < k_max && b.nb < PS_MAXBINS + 1) {
    if (b.nb < PS_MAXBINS) b.ceil[b.nb] = k_ceil;
    b.nb++;
    k_ceil *= k_factor;
  }
  const float volume = powf((float)box_size, 3);
  b.norm = 1.0 / (2.0 * M_PI * M_PI * (double)volume);
  return b;
}

__global__ void __launch_bounds__(PS_NT) k_ps_sum(const float* __restrict__ dT, size_t n3, double* partials) {
  double acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * PS_NT + threadIdx.x; i < n3; i += (size_t)gridDim.x * PS_NT) acc += dT[i];
  __shared__ double sh[PS_NT];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = PS_NT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

// deldel_ps (ComputePowerSpectrum.c:98-104) into a padded real grid; ave = sum / N^3 in double
__global__ void __launch_bounds__(PS_NT) k_ps_prepare(const float* __restrict__ dT, int n, const double* __restrict__ sum,
                                                      float volume, float* __restrict__ pad) {
  const double n3 = (double)n * n * n;
  const double ave = *sum / n3;
  const int padw = 2 * (n / 2 + 1);
  const size_t rows = (size_t)n * n;
  for (size_t row = blockIdx.x; row < rows; row += gridDim.x) {
    for (int z = threadIdx.x; z < n; z += PS_NT) {
      float v = (float)(((double)dT[row * n + z] / ave - 1) * (double)volume / (double)(float)n3);
      v = (float)((double)v * ave);
      pad[row * padw + z] = v;
    }
  }
}

// |k| of mode (nx, ny, nz) as Compute_PS forms it: float components, float squares and sums
// (no contraction), square root in double, rounded to float
__device__ __forceinline__ float ps_kmag(int nx, int ny, int nz, int n, float dk) {
  const int h = n / 2;
  const float kx = (float)(nx > h ? nx - n : nx) * dk;
  const float ky = (float)(ny > h ? ny - n : ny) * dk;
  const float kz = (float)nz * dk;
  const float s = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
  return (float)sqrt((double)s);
}

// per-block sums [3][nb]: k^3 |d|^2 norm, k, count over the Hermitian modes S[kz][x][y]
__global__ void __launch_bounds__(PS_NT) k_ps_bins(const cf* __restrict__ spec, int n, PsBins b,
                                                   double* __restrict__ partials) {
  __shared__ double sp[PS_MAXBINS], sk[PS_MAXBINS], sc[PS_MAXBINS];
  __shared__ float ceil_s[PS_MAXBINS];
  for (int i = threadIdx.x; i < PS_MAXBINS; i += PS_NT) {
    sp[i] = sk[i] = sc[i] = 0.0;
    ceil_s[i] = i < b.nb ? b.ceil[i] : 0.f;
  }
  __syncthreads();
  const int nb = b.nb;
  const size_t total = (size_t)(n / 2 + 1) * n * n;
  const unsigned lane = threadIdx.x & 31;
  // every lane of a warp runs the same number of iterations (total rounded up to the stride)
  const size_t stride = (size_t)gridDim.x * PS_NT;
  const size_t span = (total + stride - 1) / stride * stride;
  for (size_t i = (size_t)blockIdx.x * PS_NT + threadIdx.x; i < span; i += stride) {
    int bin = -1;
    double pw = 0.0, kk = 0.0;
    if (i < total) {
      const int y = (int)(i % n);
      const size_t r = i / n;
      const int x = (int)(r % n);
      const int kz = (int)(r / n);
      const float km = ps_kmag(x, y, kz, n, b.dk);
      // first bin whose upper edge exceeds |k| (bins are contiguous from 0)
      for (int c = 0; c < nb; ++c)
        if (km < ceil_s[c]) {
          bin = c;
          break;
        }
      if (bin >= 0) {
        const float2 v = __ldg(reinterpret_cast<const float2*>(spec + i));
        const double kd = (double)km;
        pw = kd * kd * kd * ((double)v.x * v.x + (double)v.y * v.y) * b.norm;
        kk = kd;
      }
    }
    // a warp whose lanes share one bin adds once; otherwise each lane adds its own mode
    const int b0 = __shfl_sync(0xffffffffu, bin, 0);
    if (__all_sync(0xffffffffu, bin == b0)) {
      double cnt = bin >= 0 ? 1.0 : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        pw += __shfl_down_sync(0xffffffffu, pw, o);
        kk += __shfl_down_sync(0xffffffffu, kk, o);
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
      }
      if (lane == 0 && b0 >= 0) {
        atomicAdd(sp + b0, pw);
        atomicAdd(sk + b0, kk);
        atomicAdd(sc + b0, cnt);
      }
    } else if (bin >= 0) {
      atomicAdd(sp + bin, pw);
      atomicAdd(sk + bin, kk);
      atomicAdd(sc + bin, 1.0);
    }
  }
  __syncthreads();
  double* out = partials + (size_t)blockIdx.x * 3 * PS_MAXBINS;
  for (int i = threadIdx.x; i < PS_MAXBINS; i += PS_NT) {
    out[i] = sp[i];
    out[PS_MAXBINS + i] = sk[i];
    out[2 * PS_MAXBINS + i] = sc[i];
  }
}

static int power_spectrum(rg_context* ctx, const rg_params* p, const float* d_dT, int max_bins, float* PS_k,
                          float* PS_data, float* PS_error, int* n_bins) {
  int rc = validate_common(ctx, p);
  if (rc) return rc;
  if (!(p->Hubble_h > 0)) return set_error(ctx, RG_EINVAL, "Hubble_h must be positive");
  const PsBins b = ps_bins(p);
  if (b.nb > PS_MAXBINS) return set_error(ctx, RG_EUNSUPPORTED, "more than 64 power-spectrum bins");
  *n_bins = b.nb;
  if (max_bins < b.nb) return set_error(ctx, RG_EINVAL, "max_bins is smaller than the number of bins");
  cudaStream_t st = ctx->stream;
  const int N = ctx->N;
  const size_t n3 = (size_t)N * N * N, nc = (size_t)(N / 2 + 1) * N * N, npad = 2 * nc;
  if ((rc = ensure_device(ctx, &ctx->spec, &ctx->spec_elems, nc))) return rc;
  if ((rc = ensure_device(ctx, &ctx->ps_pad, &ctx->ps_pad_elems, npad))) return rc;
  const int nblk = 4 * ctx->num_sms;
  double* partials = ensure_partials(ctx, (size_t)nblk * 3 * PS_MAXBINS);
  if (!partials) return set_error(ctx, RG_ENOMEM, "partials");
  const double box_size = p->BoxSize / p->Hubble_h;
  const float volume = powf((float)box_size, 3);

  prof_begin(ctx, "ps_sum", st);
  k_ps_sum<<<nblk, PS_NT, 0, st>>>(d_dT, n3, partials);
  prof_end(ctx, 4.0 * n3, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  if ((rc = reduce_partials(ctx, partials, nblk, 1, ctx->d_sums, st))) return rc;
  prof_begin(ctx, "ps_prepare", st);
  k_ps_prepare<<<nblk, PS_NT, 0, st>>>(d_dT, N, ctx->d_sums, volume, ctx->ps_pad);
  prof_end(ctx, 8.0 * n3, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  const float* src = ctx->ps_pad;
  if ((rc = fft_forward(ctx, N, &src, 1, ctx->spec, nc, 1.0, st))) return rc;
  prof_begin(ctx, "ps_bins", st);
  k_ps_bins<<<nblk, PS_NT, 0, st>>>(ctx->spec, N, b, partials);
  prof_end(ctx, 8.0 * nc, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  std::vector<double> h((size_t)nblk * 3 * PS_MAXBINS);
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), partials, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  prof_resolve(ctx);
  for (int i = 0; i < b.nb; ++i) {
    double pbox = 0.0, kave = 0.0, cnt = 0.0;
    for (int k = 0; k < nblk; ++k) {
      const double* q = h.data() + (size_t)k * 3 * PS_MAXBINS;
      pbox += q[i];
      kave += q[PS_MAXBINS + i];
      cnt += q[2 * PS_MAXBINS + i];
    }
    // ComputePowerSpectrum.c:233-235 (an empty bin gives 0/0, as there)
    PS_k[i] = (float)(kave / cnt);
    PS_data[i] = (float)(pbox / cnt);
    PS_error[i] = (float)((pbox / cnt) / sqrt(cnt));
  }
  return RG_OK;
}

}  // namespace rg

using namespace rg;

extern "C" {

int rg_power_spectrum_length(const rg_params* p, int* n_bins) {
  if (!p || !n_bins || p->ReionGridDim <= 0 || !(p->BoxSize > 0) || !(p->Hubble_h > 0)) return RG_EINVAL;
  *n_bins = ps_bins(p).nb;
  return RG_OK;
}

int rg_power_spectrum(rg_context* ctx, const rg_params* p, const float* d_delta_T, int max_bins, float* PS_k,
                      float* PS_data, float* PS_error, int* n_bins) {
  if (!ctx || !p || !d_delta_T || !PS_k || !PS_data || !PS_error || !n_bins) return RG_EINVAL;
  cudaSetDevice(ctx->device);
  return power_spectrum(ctx, p, d_delta_T, max_bins, PS_k, PS_data, PS_error, n_bins);
}

int rg_power_spectrum_host(rg_context* ctx, const rg_params* p, const float* h_delta_T, int max_bins, float* PS_k,
                           float* PS_data, float* PS_error, int* n_bins) {
  if (!ctx || !p || !h_delta_T || !PS_k || !PS_data || !PS_error || !n_bins) return RG_EINVAL;
  int rc = validate_common(ctx, p);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  const size_t n3 = (size_t)ctx->N * ctx->N * ctx->N;
  if ((rc = ensure_device(ctx, &ctx->ps_stage, &ctx->ps_stage_elems, n3))) return rc;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->ps_stage, h_delta_T, sizeof(float) * n3, cudaMemcpyHostToDevice, ctx->stream));
  return power_spectrum(ctx, p, ctx->ps_stage, max_bins, PS_k, PS_data, PS_error, n_bins);
}

int rg_smooth_grid(rg_context* ctx, double box_size, int reion_grid_dim, const float* d_in_padded,
                   float* d_out_padded) {
  if (!ctx || !d_in_padded || !d_out_padded || !(box_size > 0) || reion_grid_dim <= 0) return RG_EINVAL;
  cudaSetDevice(ctx->device);
  rg_params p;
  // the grid being smoothed is the context's (read_grids.c passes its n_cell)
  if (rg_params_default(&p, ctx->N, box_size) != RG_OK) return RG_EINVAL;
  // read_grids.c:151-155: float radius, real-space top-hat
  const double R = (double)(float)(box_size / (double)reion_grid_dim / 2.0);
  int rc = debug_roundtrip(ctx, &p, d_in_padded, d_out_padded, R, 0);
  if (rc) return rc;
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

}  // extern "C"
