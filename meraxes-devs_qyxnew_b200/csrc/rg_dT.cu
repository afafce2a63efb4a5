// 21-cm brightness temperature, ComputeBrightnessTemperatureBox()
// (src/core/BrightnessTemperature.c:24-124,512-548) without peculiar velocities: one pass
// over the cells, with the FP64 volume average reduced in the same kernel.
#include <cuda_runtime.h>

#include <cmath>

#include "rg_internal.h"
#include "rg_pass.cuh"
#include "rg_xray.h"

namespace rg {

constexpr int DT_NT = 256;
constexpr int N_RSD_STEPS = 50;      // reionization.h:34
constexpr float MAX_DVDR = 0.2f;     // reionization.h:45

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

// ---------------------------------------------------------------------------
// peculiar velocities (BrightnessTemperature.c:150-509): with the spin temperature,
// Flag_IncludePecVelsFor21cm 1 caps the velocity gradient (the 21cmFAST treatment), 2 uses the
// optical-depth form with the uncapped gradient, 3 adds the line-of-sight re-binning of 50
// sub-cells per cell (Greig & Mesinger 2018).  Every float/double step is the reference's.

// velocity in the tree code's units -> comoving velocity (BrightnessTemperature.c:173-196);
// the padding of each row is not touched (the r2c transform ignores it)
__global__ void __launch_bounds__(DT_NT) k_vel_convert(const float* __restrict__ vel, float* __restrict__ vc, int n,
                                                       int trees, float redshift) {
  const int padw = 2 * (n / 2 + 1);
  const size_t rows = (size_t)n * n;
  for (size_t row = blockIdx.x; row < rows; row += gridDim.x) {
    for (int z = threadIdx.x; z < n; z += DT_NT) {
      const size_t ip = row * padw + z;
      float v = vel[ip];
      if (trees == 1) v = (float)(sqrt(1. / (1. + (double)redshift)) * (double)v / 1000.);
      else if (trees == 0 || trees == 2) v = (float)((1. + (double)redshift) * (double)v);
      v = (float)((double)v * (1000. * 100. / MPC));
      v = (float)((double)v / (1. / (1. + (double)redshift)));
      vc[ip] = v;
    }
  }
}

// the spectrum of the velocity: / N^3, * Hubble_h (BrightnessTemperature.c:206-213), then * i k_z
// (velocity_gradient, reionization.c:3435-3450); S[kz][x][y]
__global__ void __launch_bounds__(DT_NT) k_vel_grad_spec(cf* __restrict__ spec, int n, double n3, double h, float dk) {
  const size_t total = (size_t)(n / 2 + 1) * n * n;
  for (size_t i = (size_t)blockIdx.x * DT_NT + threadIdx.x; i < total; i += (size_t)gridDim.x * DT_NT) {
    const int kz = (int)(i / ((size_t)n * n));
    const cf v = spec[i];
    float re = (float)((double)v.x / n3), im = (float)((double)v.y / n3);
    re = (float)((double)re * h);
    im = (float)((double)im * h);
    const float k = (float)kz * dk;
    // (re + i im) (0 + i k)
    spec[i] = cf{__fsub_rn(__fmul_rn(re, 0.f), __fmul_rn(im, k)), __fadd_rn(__fmul_rn(re, k), __fmul_rn(im, 0.f))};
  }
}

// the gradient correction of delta_T (BrightnessTemperature.c:215-305, spin temperature on)
__global__ void __launch_bounds__(DT_NT) k_vel_correct(float* __restrict__ dT, const float* __restrict__ grad,
                                                       const float* __restrict__ TS, int n, int flag, float H_z,
                                                       double t_rad, float redshift) {
  const int padw = 2 * (n / 2 + 1);
  const size_t rows = (size_t)n * n;
  const double max_v_deriv = fabs((double)(MAX_DVDR * H_z));
  for (size_t row = blockIdx.x; row < rows; row += gridDim.x) {
    for (int z = threadIdx.x; z < n; z += DT_NT) {
      const size_t ir = row * n + z;
      const double g = (double)grad[row * padw + z];
      float d = dT[ir];
      if (flag == 1) {
        double dvdx = g;
        if (fabs(dvdx) > max_v_deriv) dvdx = dvdx < 0 ? -max_v_deriv : max_v_deriv;
        d = (float)((double)d / (dvdx / (double)H_z + 1.0));
      } else {
        const double gc = fabs(g / (double)H_z + 1.0);
        const double ts = (double)TS[ir];
        if (gc < FRACT_FLOAT_ERR)
          d = (float)(1000. * (ts - t_rad) / (1. + (double)redshift));
        else
          d = (float)((1. - exp(-(double)d / gc)) * 1000. * (ts - t_rad) / (1. + (double)redshift));
      }
      dT[ir] = d;
    }
  }
}

struct RsdConst {
  float x_pos[N_RSD_STEPS];          // sub-cell centres in cell widths
  float x_pos_offset[N_RSD_STEPS];   // ... in Mpc
  double cell;                       // BoxSize / (float)ReionGridDim, Mpc
  double sub_w;                      // sub-cell width, Mpc
  float H_z;
};

// line-of-sight re-binning (BrightnessTemperature.c:307-509): one block per (x, y) line; every
// contributing cell moves its 50 sub-cells by the interpolated displacement v / H(z) and adds
// each (or its two parts) to the cells it lands in, periodically along z.  The line's sums live
// in shared memory; the adds of different cells meet there in any order.
__global__ void __launch_bounds__(DT_NT) k_rsd(float* __restrict__ dT, const float* __restrict__ xH,
                                               const float* __restrict__ vc, int n, RsdConst c) {
  extern __shared__ float acc[];
  const int padw = 2 * (n / 2 + 1);
  const size_t row = blockIdx.x;
  for (int k = threadIdx.x; k < n; k += DT_NT) acc[k] = 0.f;
  __syncthreads();
  const float* v = vc + row * padw;
  auto wrap = [n](int k) { return ((k % n) + n) % n; };   // the reference's periodic index
  const double w_sub = c.sub_w / c.cell;
  const double half = (c.sub_w / 2.) / c.cell;
  // the reference divides by the cell and sub-cell widths in every sub-cell; multiplying by the
  // reciprocals instead moves positions and shares by at most an ulp of double
  const double inv_cell = 1.0 / c.cell, inv_w_sub = 1.0 / w_sub;
  for (int kk = threadIdx.x; kk < n; kk += DT_NT) {
    const float d = dT[row * n + kk];
    if (!(fabs((double)d) >= FRACT_FLOAT_ERR && (double)xH[row * n + kk] >= FRACT_FLOAT_ERR)) continue;
    const double d1_low = (double)(v[kk == 0 ? n - 1 : kk - 1] / c.H_z);
    const double d2_low = (double)(v[kk] / c.H_z);
    const double d1_high = (double)(v[kk] / c.H_z);
    const double d2_high = (double)(v[kk == n - 1 ? 0 : kk + 1] / c.H_z);
    const float val = d / (float)N_RSD_STEPS;
    const double dd = (double)d / (double)N_RSD_STEPS;
    auto put = [&](int k, double frac) { atomicAdd(acc + wrap(k), (float)(frac * dd)); };
    for (int s = 0; s < N_RSD_STEPS; ++s) {
      const double xp = (double)c.x_pos[s];
      const double disp = xp <= 0.5 ? d1_low + ((xp + 0.5) - 0.) * (d2_low - d1_low) / (1. - 0.)
                                    : d1_high + ((xp - 0.5) - 0.) * (d2_high - d1_high) / (1. - 0.);
      const double pos = ((double)c.x_pos_offset[s] + disp) * inv_cell;
      const double lo = pos - half, hi = pos + half;
      if (lo >= 0.0 && hi < 1.0) {
        atomicAdd(acc + kk, val);
      } else if (lo < 0.0 && hi < 0.0) {
        const double cd = ceil(fabs(lo)) - 1.;
        const int ic = (int)cd;
        if (fabs(hi) > cd) {
          atomicAdd(acc + wrap(kk - (ic + 1)), val);
        } else {
          const double fo = (fabs(lo) - cd) * inv_w_sub, fw = 1. - fo;
          put(kk - ic, fw);
          put(kk - (ic + 1), fo);
        }
      } else if (lo < 0.0 && (hi > 0.0 && hi < 1.0)) {
        const double fw = hi * inv_w_sub, fo = 1. - fw;
        put(kk - 1, fo);
        put(kk, fw);
      } else if ((lo >= 0.0 && lo < 1.0) && (hi >= 1.0)) {
        const double fo = (hi - 1.) * inv_w_sub, fw = 1. - fo;
        put(kk, fw);
        put(kk + 1, fo);
      } else {
        const double cd = floor(fabs(hi));
        const int ic = (int)cd;
        if (lo >= cd) {
          atomicAdd(acc + wrap(kk + ic), val);
        } else {
          const double fo = (hi - cd) * inv_w_sub, fw = 1. - fo;
          put(kk + ic - 1, fw);
          put(kk + ic, fo);
        }
      }
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += DT_NT) dT[row * n + k] = acc[k];
}

__global__ void __launch_bounds__(DT_NT) k_dT_sum(const float* __restrict__ dT, size_t n3, double* partials) {
  double a = 0.0;
  for (size_t i = (size_t)blockIdx.x * DT_NT + threadIdx.x; i < n3; i += (size_t)gridDim.x * DT_NT) a += dT[i];
  __shared__ double sh[DT_NT];
  sh[threadIdx.x] = a;
  __syncthreads();
  for (int w = DT_NT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

// the velocity stages after k_delta_T; leaves the FP64 sum of the final delta_T in partials
static int velocity_modes(rg_context* ctx, const rg_params* p, const rg_grids* g, float redshift, double t_rad,
                          int nblocks, cudaStream_t st) {
  const int n = ctx->N;
  const int flag = p->Flag_IncludePecVelsFor21cm;
  const size_t nc = (size_t)(n / 2 + 1) * n * n, npad = 2 * nc, n3 = (size_t)n * n * n;
  int rc;
  if ((rc = ensure_device(ctx, &ctx->vel_work, &ctx->vel_work_elems, 2 * npad))) return rc;
  if ((rc = ensure_device(ctx, &ctx->spec, &ctx->spec_elems, nc))) return rc;
  float* vc = ctx->vel_work;
  float* grad = ctx->vel_work + npad;
  const Cosmo cm(p);
  const float H_z = (float)cm.hubble(redshift);
  prof_begin(ctx, "vel_convert", st);
  k_vel_convert<<<nblocks, DT_NT, 0, st>>>(g->vel, vc, n, p->TreesID, redshift);
  prof_end(ctx, 8.0 * n3, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  const float* src = vc;
  if ((rc = fft_forward(ctx, n, &src, 1, ctx->spec, nc, 1.0, st))) return rc;
  const float dk = (float)(2.0 * M_PI / (float)p->BoxSize);
  prof_begin(ctx, "vel_gradient", st);
  k_vel_grad_spec<<<nblocks, DT_NT, 0, st>>>(ctx->spec, n, std::pow((double)n, 3), p->Hubble_h, dk);
  prof_end(ctx, 16.0 * nc, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  if ((rc = xy_ctrl_reset(ctx, (size_t)(n / 2 + 1), st))) return rc;
  if ((rc = spectrum_to_padded(ctx, grad, st))) return rc;
  prof_begin(ctx, "vel_correct", st);
  k_vel_correct<<<nblocks, DT_NT, 0, st>>>(g->delta_T, grad, g->TS_box, n, flag, H_z, t_rad, redshift);
  prof_end(ctx, 16.0 * n3, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  if (flag == 3) {
    RsdConst c;
    const double box = p->BoxSize / p->Hubble_h;   // Mpc
    c.sub_w = (box / ((double)n)) / (double)N_RSD_STEPS;
    c.cell = box / (float)n;
    for (int i = 0; i < N_RSD_STEPS; ++i) {
      c.x_pos_offset[i] = (float)(c.sub_w * (float)i + c.sub_w / 2.);
      c.x_pos[i] = (float)(c.x_pos_offset[i] / (box / (float)n));
    }
    c.H_z = H_z;
    prof_begin(ctx, "rsd_los", st);
    k_rsd<<<(unsigned)((size_t)n * n), DT_NT, sizeof(float) * n, st>>>(g->delta_T, g->xH, vc, n, c);
    prof_end(ctx, 16.0 * n3, st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  k_dT_sum<<<nblocks, DT_NT, 0, st>>>(g->delta_T, n3, ctx->partials);
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
  if (p->Flag_IncludePecVelsFor21cm < 0 || p->Flag_IncludePecVelsFor21cm > 3)
    return set_error(ctx, RG_EINVAL, "Flag_IncludePecVelsFor21cm must be 0, 1, 2 or 3");
  if (p->UseMiniHalos)
    return set_error(ctx, RG_EUNSUPPORTED, "UseMiniHalos: the Pop II brightness temperature delta_TII is not built");
  const bool vel_modes = p->Flag_IncludeSpinTemp && p->Flag_IncludePecVelsFor21cm > 0;
  if (!g->xH || !g->deltax || !g->delta_T || (p->Flag_IncludeSpinTemp && !g->TS_box) || (vel_modes && !g->vel))
    return set_error(ctx, RG_EINVAL, "missing grid pointer");
  if (vel_modes && (p->TreesID < 0 || p->TreesID > 2)) return set_error(ctx, RG_EINVAL, "TreesID must be 0, 1 or 2");
  if (vel_modes && !(p->Hubble_h > 0)) return set_error(ctx, RG_EINVAL, "Hubble_h must be positive");
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
  if (vel_modes && (rc = velocity_modes(ctx, p, g, redshift, t_rad, nblocks, st))) return rc;
  if ((rc = reduce_partials(ctx, ctx->partials, nblocks, 1, ctx->d_sums, st))) return rc;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_sums, ctx->d_sums, sizeof(double), cudaMemcpyDeviceToHost, st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (vel_modes && (rc = xy_ctrl_check(ctx, st))) return rc;
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
  rg_grids dv = d;
  if (p->Flag_IncludeSpinTemp && p->Flag_IncludePecVelsFor21cm > 0) {
    if (!h->vel) return set_error(ctx, RG_EINVAL, "missing grid pointer");
    int rv = ensure_device(ctx, &ctx->vel_stage, &ctx->vel_stage_elems, bp / sizeof(float));
    if (rv) return rv;
    RG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->vel_stage, h->vel, bp, cudaMemcpyHostToDevice, st));
    dv.vel = ctx->vel_stage;
  }
  int rc = rg_delta_T(ctx, p, s, &dv, volume_ave_Tb);
  if (rc) return rc;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(h->delta_T, d.delta_T, br, cudaMemcpyDeviceToHost, st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return RG_OK;
}

}  // extern "C"
