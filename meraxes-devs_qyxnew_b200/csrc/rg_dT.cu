// 21-cm brightness temperature, ComputeBrightnessTemperatureBox()
// (src/core/BrightnessTemperature.c:24-124,512-548) without peculiar velocities: one pass
// over the cells, with the FP64 volume average reduced in the same kernel.
#include <cuda_runtime.h>

#include <cmath>

#include "rg_internal.h"

namespace rg {

constexpr int DT_NT = 256;

__global__ void __launch_bounds__(DT_NT) k_delta_T(const float* __restrict__ xH, const float* __restrict__ deltax,
                                                   const float* __restrict__ TS, float* __restrict__ dT, int n,
                                                   float const_factor, double t_rad, int spin, int pec_vel_gt1,
                                                   float redshift, double* __restrict__ partials) {
  const int padw = 2 * (n / 2 + 1);
  const size_t rows = (size_t)n * n;
  double acc = 0.0;
  for (size_t row = blockIdx.x; row < rows; row += gridDim.x) {
    for (int z = threadIdx.x; z < n; z += DT_NT) {
      const size_t ir = row * n + z;
      const double pixel_deltax = (double)deltax[row * padw + z];
      const double pixel_x_HI = (double)xH[ir];
      float v = (float)((double)const_factor * pixel_x_HI * (1.0 + pixel_deltax));
      if (spin) {
        if (pec_vel_gt1) {
          v = (float)((double)v * ((1. + (double)redshift) / (1000. * (double)TS[ir])));
        } else {
          const double fac = 1 - t_rad / (double)TS[ir];
          v = (float)((double)v * fac);
        }
      }
      dT[ir] = v;
      acc += (double)v;
    }
  }
  // block reduction in a fixed order
  __shared__ double sh[DT_NT];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = DT_NT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

int delta_T_launch(rg_context* ctx, int n, const float* xH, const float* deltax, const float* TS, float* dT,
                   float const_factor, double t_rad, int spin, int pec_gt1, float redshift, double* partials,
                   int nblocks, cudaStream_t st) {
  prof_begin(ctx, "delta_T", st);
  k_delta_T<<<nblocks, DT_NT, 0, st>>>(xH, deltax, TS, dT, n, const_factor, t_rad, spin, pec_gt1, redshift, partials);
  // xH, deltax (and TS) read, delta_T written
  prof_end(ctx, (double)n * n * n * (spin ? 16.0 : 12.0), st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

}  // namespace rg

using namespace rg;


extern "C" {

int rg_delta_T(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g, double* volume_ave_Tb) {
  if (!ctx || !p || !s || !g || !volume_ave_Tb || !s->ZZ) return RG_EINVAL;
  if (p->ReionGridDim != ctx->N) return set_error(ctx, RG_EINVAL, "ReionGridDim differs from the context's grid");
  if (s->snapshot < 0 || s->snapshot >= s->n_snapshots) return set_error(ctx, RG_EINVAL, "snapshot out of range");
  if (p->Flag_IncludeSpinTemp && p->Flag_IncludePecVelsFor21cm > 0 && p->Flag_IncludePecVelsFor21cm != 2)
    return set_error(ctx, RG_EUNSUPPORTED,
                     "Flag_IncludePecVelsFor21cm 1 and 3 (velocity gradient / LOS RSD) are not implemented");
  if (p->Flag_IncludeSpinTemp && p->Flag_IncludePecVelsFor21cm == 2)
    return set_error(ctx, RG_EUNSUPPORTED, "Flag_IncludePecVelsFor21cm=2 needs the velocity gradient, not implemented");
  if (!g->xH || !g->deltax || !g->delta_T || (p->Flag_IncludeSpinTemp && !g->TS_box))
    return set_error(ctx, RG_EINVAL, "missing grid pointer");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const int n = ctx->N;
  // BrightnessTemperature.c:49-54, 82: float parameters, double expression
  const float redshift = (float)s->ZZ[s->snapshot];
  const float Hubble_h = (float)p->Hubble_h;
  const float OmegaM = (float)p->OmegaM;
  const float OmegaB = (float)(OmegaM * p->BaryonFrac);
  const float const_factor = (float)(27.0 * ((double)(OmegaB * Hubble_h * Hubble_h) / 0.023) *
                                     std::sqrt((0.15 / (double)OmegaM / (double)Hubble_h / (double)Hubble_h) *
                                               (1.0 + (double)redshift) / 10.0));
  const double t_rad = TCMB * (1. + (double)redshift);
  const int nblocks = 148 * 8;
  if (!ensure_partials(ctx, (size_t)nblocks)) return set_error(ctx, RG_ENOMEM, "partials");
  int rc = delta_T_launch(ctx, n, g->xH, g->deltax, g->TS_box, g->delta_T, const_factor, t_rad,
                          p->Flag_IncludeSpinTemp, p->Flag_IncludePecVelsFor21cm > 1, redshift, ctx->partials,
                          nblocks, st);
  if (rc) return rc;
  if ((rc = reduce_partials(ctx, ctx->partials, nblocks, 1, ctx->d_sums, st))) return rc;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_sums, ctx->d_sums, sizeof(double), cudaMemcpyDeviceToHost, st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  // the reference divides by N^3 before its Allreduce (BrightnessTemperature.c:528); on one rank
  // that is the same division
  *volume_ave_Tb = ctx->h_sums[0] / std::pow((double)n, 3);
  return RG_OK;
}

int rg_delta_T_host(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* h,
                    double* volume_ave_Tb) {
  if (!ctx || !p || !s || !h || !volume_ave_Tb) return RG_EINVAL;
  if (p->ReionGridDim != ctx->N) return set_error(ctx, RG_EINVAL, "ReionGridDim differs from the context's grid");
  cudaSetDevice(ctx->device);
  if (!ctx->dev_grids_ready) {
    int rc = rg_alloc_grids(ctx, p, 0, &ctx->dev_grids);
    if (rc) return rc;
    ctx->dev_grids_ready = true;
  }
  const rg_grids& d = ctx->dev_grids;
  if (p->Flag_IncludeSpinTemp && !d.TS_box) return set_error(ctx, RG_EINVAL, "device grids lack TS_box");
  const size_t n = (size_t)ctx->N;
  const size_t bp = n * n * 2 * (n / 2 + 1) * sizeof(float), br = n * n * n * sizeof(float);
  cudaStream_t st = ctx->stream;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync((void*)d.deltax, h->deltax, bp, cudaMemcpyHostToDevice, st));
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(d.xH, h->xH, br, cudaMemcpyHostToDevice, st));
  if (p->Flag_IncludeSpinTemp) RG_CUDA_TRY(ctx, cudaMemcpyAsync(d.TS_box, h->TS_box, br, cudaMemcpyHostToDevice, st));
  int rc = rg_delta_T(ctx, p, s, &d, volume_ave_Tb);
  if (rc) return rc;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(h->delta_T, d.delta_T, br, cudaMemcpyDeviceToHost, st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return RG_OK;
}

}  // extern "C"
