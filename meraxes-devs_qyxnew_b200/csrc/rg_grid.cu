// The source grids from the galaxies, on the device: the nearest-grid-point deposit of
// construct_baryon_grids() (src/core/reionization.c:2025-2592) for one rank that holds the whole
// grid.  Every galaxy's values are added to the cell pos_to_ngp() (src/core/misc_tools.c:207-217)
// gives for its position; each grid is then clamped at zero (CLAMP_NEGATIVE, misc_tools.h:7),
// optionally divided (the sfr grid by the SFR timescale, reionization.c:2500-2510) and stored in
// the padded layout the steps read.  Which galaxy property feeds which grid, the black-hole mass
// limit and the shift of the history slots stay with the caller (the galaxy model).
//
// The reference adds a rank's galaxies to a float buffer in galaxy order; here the adds of the
// galaxies of one cell meet in any order (float atomics), which changes the cell sums by float
// rounding only.
#include <cuda_runtime.h>

#include <string>

#include "rg_internal.h"
#include "rg_pass.cuh"

namespace rg {

constexpr int NGP_NT = 256;

// grid p of a pack without dynamic indexing into kernel parameters
__device__ __forceinline__ float* grid_of(const GridPtrsW& a, int p) {
  void* r = a.p[0];
#pragma unroll
  for (int i = 1; i < MAXG; ++i)
    if (p == i) r = a.p[i];
  return static_cast<float*>(r);
}

// pos_to_ngp: nearest grid point, the top edge wrapped to 0; -1 for a position below the box
__device__ __forceinline__ int ngp(float x, double side, int nx) {
  int ind = (int)rint((double)x / side * (double)nx);
  if (ind > nx - 1) ind = 0;
  return ind;
}

__global__ void __launch_bounds__(NGP_NT) k_ngp_deposit(int n_gal, const float* __restrict__ pos, int n_prop,
                                                        const float* __restrict__ vals, GridPtrsW grids, double box,
                                                        int n, int* __restrict__ bad) {
  const int padw = 2 * (n / 2 + 1);
  for (int g = blockIdx.x * NGP_NT + threadIdx.x; g < n_gal; g += gridDim.x * NGP_NT) {
    const int ix = ngp(pos[3 * (size_t)g], box, n), iy = ngp(pos[3 * (size_t)g + 1], box, n),
              iz = ngp(pos[3 * (size_t)g + 2], box, n);
    if (ix < 0 || iy < 0 || iz < 0) {
      atomicAdd(bad, 1);
      continue;
    }
    const size_t ip = ((size_t)ix * n + iy) * padw + iz;
    for (int p = 0; p < n_prop; ++p) atomicAdd(grid_of(grids, p) + ip, vals[(size_t)p * n_gal + g]);
  }
}

struct NgpDiv {
  double d[MAXG];
};

// clamp at zero and divide, every real cell of every grid (ComputeTs/find_HII read only those)
__global__ void __launch_bounds__(NGP_NT) k_ngp_finish(GridPtrsW grids, int n_prop, int n, NgpDiv div) {
  const int padw = 2 * (n / 2 + 1);
  const size_t rows = (size_t)n * n;
  for (int p = 0; p < n_prop; ++p) {
    float* gp = grid_of(grids, p);
    double dv = div.d[0];
#pragma unroll
    for (int i = 1; i < MAXG; ++i)
      if (p == i) dv = div.d[i];
    for (size_t row = blockIdx.x; row < rows; row += gridDim.x)
      for (int z = threadIdx.x; z < n; z += NGP_NT) {
        double v = (double)gp[row * padw + z];
        if (v < 0) v = 0;
        if (dv != 1.0) v /= dv;
        gp[row * padw + z] = (float)v;
      }
  }
}

}  // namespace rg

using namespace rg;

extern "C" {

int rg_deposit_ngp(rg_context* ctx, double box_size, int n_gal, const float* d_pos, int n_prop,
                   const float* d_values, const double* divisors, float* const* d_grids) {
  if (!ctx || !(box_size > 0) || n_gal < 0 || n_prop < 1 || !d_grids || (n_gal > 0 && (!d_pos || !d_values)))
    return RG_EINVAL;
  if (n_prop > MAXG) return set_error(ctx, RG_EINVAL, "at most 8 grids per deposit");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const int n = ctx->N;
  const size_t npad = (size_t)n * n * 2 * (n / 2 + 1);
  GridPtrsW gp{};
  NgpDiv dv;
  for (int p = 0; p < MAXG; ++p) dv.d[p] = 1.0;
  for (int p = 0; p < n_prop; ++p) {
    if (!d_grids[p]) return set_error(ctx, RG_EINVAL, "missing grid pointer");
    gp.p[p] = d_grids[p];
    if (divisors) {
      if (!(divisors[p] > 0)) return set_error(ctx, RG_EINVAL, "divisors must be positive");
      dv.d[p] = divisors[p];
    }
    RG_CUDA_TRY(ctx, cudaMemsetAsync(d_grids[p], 0, sizeof(float) * npad, st));
  }
  int rc = ensure_device(ctx, &ctx->ngp_bad, &ctx->ngp_bad_elems, 1);
  if (rc) return rc;
  RG_CUDA_TRY(ctx, cudaMemsetAsync(ctx->ngp_bad, 0, sizeof(int), st));
  const int nblk = 4 * ctx->num_sms;
  if (n_gal > 0) {
    prof_begin(ctx, "ngp_deposit", st);
    k_ngp_deposit<<<nblk, NGP_NT, 0, st>>>(n_gal, d_pos, n_prop, d_values, gp, box_size, n, ctx->ngp_bad);
    prof_end(ctx, (double)n_gal * (12.0 + 8.0 * n_prop), st);
    RG_CUDA_TRY(ctx, cudaGetLastError());
  }
  prof_begin(ctx, "ngp_finish", st);
  k_ngp_finish<<<nblk, NGP_NT, 0, st>>>(gp, n_prop, n, dv);
  prof_end(ctx, 8.0 * n_prop * (double)n * n * n, st);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  int bad = 0;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(&bad, ctx->ngp_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  if (bad) return set_error(ctx, RG_EINVAL, "galaxy positions below the box (pos_to_ngp asserts on them)");
  return RG_OK;
}

int rg_push_histories(rg_context* ctx, const rg_params* p, const rg_grids* g) {
  if (!ctx || !p || !g) return RG_EINVAL;
  if (!p->Flag_IncludeSpinTemp) return RG_OK;   // the reference keeps histories for ComputeTs only
  if (g->n_hist < 1) return set_error(ctx, RG_EINVAL, "n_hist must be at least 1");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const int n = ctx->N;
  const size_t npad = (size_t)n * n * 2 * (n / 2 + 1);
  const int agn = p->Flag_IncludeAGNXray;
  struct Kind {
    const float* cur;
    float* hist;
    bool on;
    const char* name;
  } kinds[4] = {  // the histories are inputs of the step (const in rg_grids); this call updates them
      {g->sfr, const_cast<float*>(g->sfr_histories), true, "sfr"},
      {g->xray_luminosity, const_cast<float*>(g->xray_luminosity_histories), true, "xray_luminosity"},
      {g->bh_xray_soft, const_cast<float*>(g->bh_xray_histories_soft), agn == 1 || agn == 3, "bh_xray_soft"},
      {g->bh_xray_hard, const_cast<float*>(g->bh_xray_histories_hard), agn == 1 || agn == 2, "bh_xray_hard"}};
  for (const Kind& k : kinds) {
    if (!k.on) continue;
    if (!k.cur || !k.hist) return set_error(ctx, RG_EINVAL, std::string("missing grid or histories of ") + k.name);
  }
  prof_begin(ctx, "push_histories", st);
  double bytes = 0.0;
  for (const Kind& k : kinds) {
    if (!k.on) continue;
    // slot h + 1 <- slot h from the top, then slot 0 <- this snapshot's grid
    for (int h = g->n_hist - 2; h >= 0; --h)
      RG_CUDA_TRY(ctx, cudaMemcpyAsync(k.hist + (size_t)(h + 1) * npad, k.hist + (size_t)h * npad,
                                       sizeof(float) * npad, cudaMemcpyDeviceToDevice, st));
    RG_CUDA_TRY(ctx, cudaMemcpyAsync(k.hist, k.cur, sizeof(float) * npad, cudaMemcpyDeviceToDevice, st));
    bytes += 8.0 * npad * g->n_hist;
  }
  prof_end(ctx, bytes, st);
  return RG_OK;
}

}  // extern "C"
