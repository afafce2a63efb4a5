// The C ABI: context lifetime, parameter validation and the host orchestration of the
// grid step (find_HII_bubbles, ComputeTs, delta_T).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rg_fft.cuh"
#include "rg_internal.h"
#include "rg_xray.h"

namespace rg {

int set_error(rg_context* ctx, int status, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return status;
}

Units make_units(const rg_params* p) {
  Units u;
  u.UnitTime_in_s = p->UnitLength_in_cm / p->UnitVelocity_in_cm_per_s;
  u.G = GRAVITY / std::pow(p->UnitLength_in_cm, 3) * p->UnitMass_in_g * std::pow(u.UnitTime_in_s, 2);
  u.Hubble = HUBBLE * u.UnitTime_in_s;
  u.RhoCrit = 3 * u.Hubble * u.Hubble / (8 * M_PI * u.G);
  return u;
}

double hubble_time_at(const rg_params* p, double z) {
  // hubble_time() = 1 / (Hubble E(z)), src/core/virial_properties.c:6-20,79-96
  const Units u = make_units(p);
  const double opz = 1. + z;
  const double ez = std::sqrt(p->OmegaM * opz * opz * opz + p->OmegaK * opz * opz + p->OmegaLambda);
  return 1.0 / (u.Hubble * ez);
}

double dtdz(const rg_params* p, float zf) {
  // src/core/XRayHeatingFunctions.c:426-440
  const double opz = (double)(1.0f + zf);  // 1 + z is a float sum in the C
  const double oml = p->OmegaLambda, omm = p->OmegaM;
  const double x = std::sqrt(oml / omm) * std::pow(opz, -3.0 / 2.0);
  const double dxdz = std::sqrt(oml / omm) * std::pow(opz, -5.0 / 2.0) * (-3.0 / 2.0);
  const double const1 = 2 * std::sqrt(1 + omm / oml) / (3.0 * HUBBLE * p->Hubble_h);
  const double numer = dxdz * (1 + x * std::pow(std::pow(x, 2) + 1, -0.5));
  const double denom = x + std::sqrt(std::pow(x, 2) + 1);
  return const1 * numer / denom;
}

double rtom(const rg_params* p, double R) {
  // RtoM(), src/core/find_HII_bubbles.c:27-46
  const Units u = make_units(p);
  if (p->ReionRtoMFilterType == 0) return (4.0 / 3.0) * M_PI * std::pow(R, 3) * (p->OmegaM * u.RhoCrit);
  return std::pow(2 * M_PI, 1.5) * p->OmegaM * u.RhoCrit * std::pow(R, 3);
}

float cT_approx(float z) { return (float)(0.58 - 0.006 * ((double)z - 10.0)); }

std::vector<std::pair<double, bool>> radius_schedule(const rg_params* p, double z) {
  // find_HII_bubbles.c:147-148,256-285,546
  const double box = p->BoxSize;
  const int n = p->ReionGridDim;
  double cell_len_factor = L_FACTOR;
  if ((box / (double)n) < 1.0) cell_len_factor = 1.0;
  double rmax;
  if (p->Flag_EvolvingReionRBubbleMax)
    rmax = z > 6. ? 25.483241248322766 : 112. * std::pow((1. + z) / 5., -4.4);
  else
    rmax = p->Flag_IncludeRecombinations ? p->ReionRBubbleMaxRecomb : p->ReionRBubbleMax;
  double R = std::fmin(rmax, L_FACTOR * box);
  std::vector<std::pair<double, bool>> out;
  bool last = false;
  while (!last) {
    if (((R / p->ReionDeltaRFactor) <= (cell_len_factor * box / (double)n)) ||
        ((R / p->ReionDeltaRFactor) <= p->ReionRBubbleMin)) {
      last = true;
      R = cell_len_factor * box / (double)n;
    }
    out.emplace_back(R, last);
    R /= p->ReionDeltaRFactor;
    if (out.size() > 100000) break;  // guards a ReionDeltaRFactor <= 1 that validation missed
  }
  return out;
}

int twiddles_for(rg_context* ctx, int n, const cf** out) {
  for (auto& e : ctx->twiddles)
    if (e.first == n) {
      *out = e.second;
      return RG_OK;
    }
  std::vector<cf> h(n);
  for (int k = 0; k < n; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)n;
    h[k] = cf{(float)std::cos(a), (float)std::sin(a)};
  }
  cf* d = nullptr;
  RG_CUDA_TRY(ctx, cudaMalloc((void**)&d, sizeof(cf) * n));
  RG_CUDA_TRY(ctx, cudaMemcpy(d, h.data(), sizeof(cf) * n, cudaMemcpyHostToDevice));
  ctx->twiddles.emplace_back(n, d);
  *out = d;
  return RG_OK;
}

void prof_begin(rg_context* ctx, const char* name, cudaStream_t st) {
  if (!ctx->prof_on) return;
  auto take = [&]() {
    cudaEvent_t e;
    if (!ctx->prof_pool.empty()) {
      e = ctx->prof_pool.back();
      ctx->prof_pool.pop_back();
    } else {
      cudaEventCreate(&e);
    }
    return e;
  };
  rg_context::ProfRec r;
  r.name = name;
  r.e0 = take();
  r.e1 = take();
  r.bytes = 0;
  cudaEventRecord(r.e0, st);
  ctx->prof_pending.push_back(r);
}

void prof_end(rg_context* ctx, double alg_bytes, cudaStream_t st) {
  if (!ctx->prof_on || ctx->prof_pending.empty()) return;
  auto& r = ctx->prof_pending.back();
  r.bytes = alg_bytes;
  cudaEventRecord(r.e1, st);
}

void prof_resolve(rg_context* ctx) {
  for (auto& r : ctx->prof_pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(r.e1) == cudaSuccess) cudaEventElapsedTime(&ms, r.e0, r.e1);
    rg_kernel_stat* st = nullptr;
    for (auto& k : ctx->prof_stats)
      if (r.name == k.name) st = &k;
    if (!st) {
      rg_kernel_stat k{};
      std::snprintf(k.name, sizeof(k.name), "%s", r.name.c_str());
      ctx->prof_stats.push_back(k);
      st = &ctx->prof_stats.back();
    }
    st->launches += 1;
    st->ms_total += ms;
    st->alg_bytes_total += r.bytes;
    ctx->prof_pool.push_back(r.e0);
    ctx->prof_pool.push_back(r.e1);
  }
  ctx->prof_pending.clear();
}

bool supported_n(int n) {
  static const int ok[] = {8, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512};
  for (int v : ok)
    if (v == n) return true;
  return false;
}

int ensure_tables(rg_context* ctx, const rg_params* p) {
  const std::string dir = p->TablesForXHeatingDir ? p->TablesForXHeatingDir : "";
  if (ctx->tables.loaded && ctx->tables.dir == dir) return RG_OK;
  if (dir.empty()) return set_error(ctx, RG_ETABLE, "TablesForXHeatingDir is not set");
  const std::string e = load_tables(dir, p->ReionNionPhotPerBary, &ctx->tables);
  if (!e.empty()) return set_error(ctx, RG_ETABLE, e);
  return RG_OK;
}

double* ensure_partials(rg_context* ctx, size_t n) {
  if (ctx->partials && ctx->partials_elems >= n) return ctx->partials;
  if (ctx->partials) cudaFree(ctx->partials);
  ctx->partials = nullptr;
  ctx->partials_elems = 0;
  if (cudaMalloc((void**)&ctx->partials, sizeof(double) * n) != cudaSuccess) return nullptr;
  ctx->partials_elems = n;
  return ctx->partials;
}

int validate_common(rg_context* ctx, const rg_params* p) {
  if (!ctx || !p) return RG_EINVAL;
  if (p->ReionGridDim != ctx->N) return set_error(ctx, RG_EINVAL, "ReionGridDim differs from the context's grid");
  if (!(p->BoxSize > 0)) return set_error(ctx, RG_EINVAL, "BoxSize must be positive");
  if (!(p->UnitLength_in_cm > 0) || !(p->UnitMass_in_g > 0) || !(p->UnitVelocity_in_cm_per_s > 0))
    return set_error(ctx, RG_EINVAL, "units must be positive");
  return RG_OK;
}

__global__ void k_fill(float* p, size_t n, float v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

static int fill(rg_context* ctx, float* p, size_t n, float v) {
  if (!p) return RG_OK;
  if (v == 0.f) {
    RG_CUDA_TRY(ctx, cudaMemsetAsync(p, 0, n * sizeof(float), ctx->stream));
    return RG_OK;
  }
  k_fill<<<1184, 256, 0, ctx->stream>>>(p, n, v);
  RG_CUDA_TRY(ctx, cudaGetLastError());
  return RG_OK;
}

}  // namespace rg

using namespace rg;

// ---------------------------------------------------------------------------

extern "C" {

const char* rg_status_string(int s) {
  switch (s) {
    case RG_OK: return "ok";
    case RG_EINVAL: return "invalid argument";
    case RG_ENOMEM: return "out of memory";
    case RG_ECUDA: return "CUDA error";
    case RG_EUNSUPPORTED: return "unsupported feature";
    case RG_ETABLE: return "table file error";
    case RG_ENODEV: return "no CUDA device";
    case RG_ETIMEDOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

const char* rg_last_error(const rg_context* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int rg_params_default(rg_params* p, int grid_dim, double box_size) {
  if (!p) return RG_EINVAL;
  std::memset(p, 0, sizeof(*p));
  p->ReionGridDim = grid_dim;
  p->BoxSize = box_size;
  // Genesis cosmology and units (input/params/simulations/Genesis_L10_N512.par:17-31)
  p->OmegaM = 0.3121;
  p->OmegaK = 0.0;
  p->OmegaLambda = 0.6879;
  p->OmegaR = 0.0;
  p->BaryonFrac = 0.15714;
  p->Hubble_h = 0.6751;
  p->wLambda = -1.0;
  p->UnitLength_in_cm = 3.08568e+24;
  p->UnitMass_in_g = 1.989e+43;
  p->UnitVelocity_in_cm_per_s = 100000;
  // input/params/defaults.par:233-282
  p->ReionDeltaRFactor = 1.1;
  p->ReionRBubbleMax = 20.34;
  p->ReionRBubbleMaxRecomb = 33.9;
  p->ReionRBubbleMin = 0.4068;
  p->Flag_EvolvingReionRBubbleMax = 1;
  p->ReionFilterType = 0;
  p->ReionRtoMFilterType = 0;
  p->ReionUVBFlag = 1;
  p->ReionNionPhotPerBary = 4000;
  p->Y_He = 0.24;
  // set_ReionEfficiency(), src/core/reionization.c:299-328
  p->ReionEfficiency = 1.0 / p->BaryonFrac * p->ReionNionPhotPerBary / (1.0 - 0.75 * p->Y_He);
  p->ReionGammaHaloBias = 2.0;
  p->ReionAlphaUV = 2.0;
  p->ReionAlphaUVBH = 2.0;
  p->ReionSfrTimescale = 0.5;
  p->TsHeatingFilterType = 1;
  p->TsNumFilterSteps = 40;
  p->ReionMaxHeatingRedshift = 30.;
  p->NuXrayThreshold = 500.;
  p->NuXraySoftCut = 2000.;
  p->NuXrayMax = 10000.;
  p->SpecIndexXrayGal = 1.;
  p->Flag_TemperatureDependentRec = 1;   // input/params/defaults.par:19
  p->SpecIndexXrayAGNSoft = 2.2;          // input/params/defaults.par:67-68
  p->SpecIndexXrayAGNHard = 1.7;
  // Pop III (UseMiniHalos): the caller's IMF sets the photons per baryon; the efficiency follows
  // set_ReionEfficiency (reionization.c:311-314)
  p->UseMiniHalos = 0;
  p->ReionNionPhotPerBaryIII = p->ReionNionPhotPerBary;
  p->ReionEfficiencyIII = 1.0 / p->BaryonFrac * p->ReionNionPhotPerBaryIII / (1.0 - 0.75 * p->Y_He);
  return RG_OK;
}

int rg_create(int device, int grid_dim, rg_context** out) {
  if (!out) return RG_EINVAL;
  *out = nullptr;
  if (!supported_n(grid_dim)) return RG_EUNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return RG_ENODEV;
  if (device < 0 || device >= ndev) return RG_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return RG_ECUDA;
  rg_context* ctx = new rg_context();
  ctx->device = device;
  ctx->N = grid_dim;
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return RG_ECUDA;
  }
  ctx->stream = ctx->own_stream;
  if (cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->copy_stream_out, cudaStreamNonBlocking) != cudaSuccess) {
    rg_destroy(ctx);
    return RG_ECUDA;
  }
  if (cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      ctx->num_sms < 1) {
    rg_destroy(ctx);
    return RG_ECUDA;
  }
  if (cudaMallocHost((void**)&ctx->h_sums, sizeof(double) * 64) != cudaSuccess ||
      cudaMalloc((void**)&ctx->d_sums, sizeof(double) * 64) != cudaSuccess) {
    rg_destroy(ctx);
    return RG_ENOMEM;
  }
  *out = ctx;
  return RG_OK;
}

int rg_destroy(rg_context* ctx) {
  if (!ctx) return RG_EINVAL;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& e : ctx->twiddles) cudaFree(e.second);
  if (ctx->spec) cudaFree(ctx->spec);
  if (ctx->work) cudaFree(ctx->work);
  if (ctx->bits) cudaFree(ctx->bits);
  if (ctx->wtab) cudaFree(ctx->wtab);
  if (ctx->wcut) cudaFree(ctx->wcut);
  if (ctx->ps_pad) cudaFree(ctx->ps_pad);
  if (ctx->ps_stage) cudaFree(ctx->ps_stage);
  if (ctx->vel_work) cudaFree(ctx->vel_work);
  if (ctx->vel_stage) cudaFree(ctx->vel_stage);
  if (ctx->ngp_bad) cudaFree(ctx->ngp_bad);
  if (ctx->ts_agn) cudaFree(ctx->ts_agn);
  if (ctx->rec_knots) cudaFree(ctx->rec_knots);
  if (ctx->rec_y) cudaFree(ctx->rec_y);
  if (ctx->rec_c) cudaFree(ctx->rec_c);
  if (ctx->partials) cudaFree(ctx->partials);
  if (ctx->d_sums) cudaFree(ctx->d_sums);
  if (ctx->h_sums) cudaFreeHost(ctx->h_sums);
  if (ctx->batch_sums) cudaFree(ctx->batch_sums);
  if (ctx->h_batch_sums) cudaFreeHost(ctx->h_batch_sums);
  if (ctx->d_radii) cudaFree(ctx->d_radii);
  if (ctx->ts_stage) cudaFree(ctx->ts_stage);
  if (ctx->ts_const) cudaFree(ctx->ts_const);
  if (ctx->ts_sums) cudaFree(ctx->ts_sums);
  if (ctx->xy_ctrl) cudaFree(ctx->xy_ctrl);
  for (void* p : ctx->owned) cudaFree(p);
  prof_resolve(ctx);
  for (cudaEvent_t e : ctx->prof_pool) cudaEventDestroy(e);
  if (ctx->copy_stream) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  if (ctx->copy_stream_out) {
    cudaStreamSynchronize(ctx->copy_stream_out);
    cudaStreamDestroy(ctx->copy_stream_out);
  }
  for (cudaEvent_t e : ctx->stage_events) cudaEventDestroy(e);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return RG_OK;
}

int rg_set_mode(rg_context* ctx, int mode) {
  if (!ctx || (mode != RG_MODE_FUSED && mode != RG_MODE_PLAIN)) return RG_EINVAL;
  ctx->mode = mode;
  return RG_OK;
}

int rg_set_radius_batch(rg_context* ctx, int k) {
  if (!ctx || k < 0 || k > 64) return RG_EINVAL;
  ctx->radius_batch = k;
  return RG_OK;
}

int rg_debug_set_wait_limits(rg_context* ctx, int xy_poll_limit, int xy_signal, int ts_iteration_limit) {
  if (!ctx) return RG_EINVAL;
  ctx->xy_poll_limit = xy_poll_limit < 0 ? RG_XY_POLL_LIMIT : std::min(xy_poll_limit, RG_XY_POLL_LIMIT);
  ctx->xy_signal = xy_signal != 0;
  ctx->ts_iter_limit = ts_iteration_limit < 1 ? RG_TS_ITER_LIMIT : std::min(ts_iteration_limit, RG_TS_ITER_LIMIT);
  return RG_OK;
}

int rg_set_stream(rg_context* ctx, void* stream) {
  if (!ctx) return RG_EINVAL;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return RG_OK;
}

int rg_radius_schedule(const rg_params* p, double redshift, double* radii, int max_r, int* n) {
  if (!p || !n || p->ReionGridDim <= 0 || !(p->BoxSize > 0) || !(p->ReionDeltaRFactor > 1.0)) return RG_EINVAL;
  auto s = radius_schedule(p, redshift);
  *n = (int)s.size();
  for (int i = 0; i < (int)s.size() && i < max_r && radii; ++i) radii[i] = s[i].first;
  return RG_OK;
}

int rg_alloc_grids(rg_context* ctx, const rg_params* p, int n_hist, rg_grids* out) {
  if (!ctx || !p || !out) return RG_EINVAL;
  int rc = validate_common(ctx, p);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  const size_t n = (size_t)ctx->N;
  const size_t npad = n * n * 2 * (n / 2 + 1), nreal = n * n * n;
  std::memset(out, 0, sizeof(*out));
  auto A = [&](size_t elems, float** dst) -> int {
    void* q = nullptr;
    if (cudaMalloc(&q, elems * sizeof(float)) != cudaSuccess)
      return set_error(ctx, RG_ENOMEM, "cudaMalloc failed in rg_alloc_grids");
    ctx->owned.push_back(q);
    *dst = (float*)q;
    return RG_OK;
  };
  float* t = nullptr;
#define RG_ALLOC(field, elems)            \
  do {                                    \
    if ((rc = A((elems), &t))) return rc; \
    out->field = t;                       \
  } while (0)
  RG_ALLOC(deltax, npad);
  RG_ALLOC(stars, npad);
  RG_ALLOC(weighted_sfr, npad);
  if (p->Flag_BHFeedback) {
    RG_ALLOC(effective_bhm, npad);
    RG_ALLOC(effective_bhar, npad);
  }
  RG_ALLOC(xH, nreal);
  RG_ALLOC(r_bubble, nreal);
  RG_ALLOC(z_at_ionization, nreal);
  RG_ALLOC(J_21_at_ionization, nreal);
  RG_ALLOC(temp_kinetic_all_gas, nreal);
  RG_ALLOC(delta_T, nreal);
  if (p->Flag_IncludeSpinTemp && p->Flag_IncludePecVelsFor21cm > 0) RG_ALLOC(vel, npad);
  if (p->UseMiniHalos) {
    RG_ALLOC(starsIII, npad);
    RG_ALLOC(weighted_sfrIII, npad);
  }
  if (p->Flag_IncludeRecombinations) {
    RG_ALLOC(Gamma12, nreal);
    RG_ALLOC(N_rec, npad);
    RG_ALLOC(residual_xH, nreal);
    RG_ALLOC(clumping_factor, nreal);
    RG_ALLOC(t_resp, nreal);
  }
  if (p->Flag_IncludeSpinTemp) {
    RG_ALLOC(x_e_box_prev, npad);
    RG_ALLOC(x_e_box, npad);
    RG_ALLOC(Tk_box, nreal);
    RG_ALLOC(TS_box, nreal);
    RG_ALLOC(sfr, npad);
    RG_ALLOC(xray_luminosity, npad);
    if (n_hist > 0) {
      RG_ALLOC(sfr_histories, npad * (size_t)n_hist);
      RG_ALLOC(xray_luminosity_histories, npad * (size_t)n_hist);
    }
    out->n_hist = n_hist;
  }
#undef RG_ALLOC
  return RG_OK;
}

int rg_init_reion_grids(rg_context* ctx, const rg_params* p, const rg_grids* g) {
  if (!ctx || !p || !g) return RG_EINVAL;
  int rc = validate_common(ctx, p);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  const size_t n = (size_t)ctx->N;
  const size_t npad = n * n * 2 * (n / 2 + 1), nreal = n * n * n;
  // src/core/reionization.c:557-595
  if ((rc = fill(ctx, g->xH, nreal, 1.f))) return rc;
  if ((rc = fill(ctx, g->z_at_ionization, nreal, -1.f))) return rc;
  if ((rc = fill(ctx, g->r_bubble, nreal, 0.f))) return rc;
  if ((rc = fill(ctx, g->temp_kinetic_all_gas, nreal, 0.f))) return rc;
  if ((rc = fill(ctx, g->J_21_at_ionization, nreal, 0.f))) return rc;
  if ((rc = fill(ctx, g->delta_T, nreal, 0.f))) return rc;
  if ((rc = fill(ctx, g->Tk_box, nreal, 0.f))) return rc;
  if ((rc = fill(ctx, g->TS_box, nreal, 0.f))) return rc;
  if ((rc = fill(ctx, g->x_e_box_prev, npad, 0.f))) return rc;
  if ((rc = fill(ctx, g->x_e_box, npad, 0.f))) return rc;
  // reionization.c:576-582,698
  if ((rc = fill(ctx, g->Gamma12, nreal, 0.f))) return rc;
  if ((rc = fill(ctx, g->residual_xH, nreal, 0.f))) return rc;
  if ((rc = fill(ctx, g->clumping_factor, nreal, 0.f))) return rc;
  if ((rc = fill(ctx, g->t_resp, nreal, 1e30f))) return rc;
  if ((rc = fill(ctx, g->N_rec, npad, 0.f))) return rc;
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

}  // extern "C"

static int find_hii(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g,
                    rg_hii_scalars* out, const Staging* stg) {
  int rc = validate_common(ctx, p);
  if (rc) return rc;
  if (s->snapshot < 0 || s->snapshot >= s->n_snapshots) return set_error(ctx, RG_EINVAL, "snapshot out of range");
  if (p->Flag_IncludeRecombinations) {
    if (!ctx->rec_y || ctx->rec_nz < 1 || ctx->rec_nt < 1 || ctx->rec_ng < 3)
      return set_error(ctx, RG_EINVAL, "Flag_IncludeRecombinations needs rg_set_recombination_tables first");
    if (!g->Gamma12 || !g->N_rec || !g->residual_xH || !g->clumping_factor || !g->t_resp)
      return set_error(ctx, RG_EINVAL, "recombinations need Gamma12, N_rec, residual_xH, clumping_factor, t_resp");
  }
  if (p->ReionFilterType < 0 || p->ReionFilterType > 2)
    return set_error(ctx, RG_EINVAL, "ReionFilterType must be 0, 1 or 2");
  if (p->ReionRtoMFilterType < 0 || p->ReionRtoMFilterType > 1)
    return set_error(ctx, RG_EINVAL, "ReionRtoMFilterType must be 0 or 1");
  if (!(p->ReionDeltaRFactor > 1.0)) return set_error(ctx, RG_EINVAL, "ReionDeltaRFactor must exceed 1");
  if (!g->deltax || !g->stars || !g->weighted_sfr || !g->xH || !g->r_bubble || !g->z_at_ionization ||
      !g->J_21_at_ionization || !g->temp_kinetic_all_gas)
    return set_error(ctx, RG_EINVAL, "missing grid pointer");
  if (p->Flag_IncludeSpinTemp && (!g->x_e_box || !g->Tk_box))
    return set_error(ctx, RG_EINVAL, "spin temperature needs x_e_box and Tk_box");
  if (p->Flag_BHFeedback && (!g->effective_bhm || !g->effective_bhar))
    return set_error(ctx, RG_EINVAL, "BH feedback needs effective_bhm and effective_bhar");
  if (p->UseMiniHalos && (!g->starsIII || !g->weighted_sfrIII))
    return set_error(ctx, RG_EINVAL, "UseMiniHalos needs starsIII and weighted_sfrIII");
  if ((rc = ensure_tables(ctx, p))) return rc;
  cudaSetDevice(ctx->device);
  return hii_snapshot(ctx, p, s, g, out, stg);
}

// event i of the context's staging pool (created on first use)
static cudaEvent_t stage_event(rg_context* ctx, size_t i) {
  while (ctx->stage_events.size() <= i) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    ctx->stage_events.push_back(e);
  }
  return ctx->stage_events[i];
}

int rg::stage_wait(rg_context* ctx, cudaEvent_t ev, cudaStream_t st) {
  if (ev) RG_CUDA_TRY(ctx, cudaStreamWaitEvent(st, ev, 0));
  return RG_OK;
}

int rg::stage_record(rg_context* ctx, size_t i, cudaStream_t st, cudaEvent_t* out) {
  cudaEvent_t e = stage_event(ctx, i);
  if (!e) return set_error(ctx, RG_ECUDA, "cudaEventCreate failed");
  RG_CUDA_TRY(ctx, cudaEventRecord(e, st));
  *out = e;
  return RG_OK;
}

// the copy stream starts after the work already queued on the context's stream (which may
// still read the device grids the copies overwrite)
static int copy_stream_after_prior(rg_context* ctx) {
  cudaEvent_t e;
  int rc = stage_record(ctx, 0, ctx->stream, &e);
  if (rc) return rc;
  RG_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->copy_stream, e, 0));
  return RG_OK;
}

extern "C" {

int rg_set_recombination_tables(rg_context* ctx, const double* lnGamma, int n_z, int n_t, int n_gamma,
                                const double* RR, const double* CF, const double* RNH) {
  if (!ctx || !lnGamma || !RR || !CF || !RNH || n_z < 1 || n_t < 1 || n_gamma < 3) return RG_EINVAL;
  for (int i = 0; i + 1 < n_gamma; ++i)
    if (!(lnGamma[i + 1] > lnGamma[i])) return set_error(ctx, RG_EINVAL, "lnGamma knots must increase");
  cudaSetDevice(ctx->device);
  const size_t rows = (size_t)n_z * n_t, per = rows * (size_t)n_gamma;
  // natural cubic spline of every (table, z, T) row in ln Gamma12 (init_MHR's gsl_interp_cspline
  // splines, recombinations.c:347-363)
  std::vector<double> c(3 * per);
  const std::vector<double> x(lnGamma, lnGamma + n_gamma);
  const double* tabs[3] = {RR, CF, RNH};
  CubicSpline sp;
  for (int k = 0; k < 3; ++k)
    for (size_t r = 0; r < rows; ++r) {
      const double* y = tabs[k] + r * n_gamma;
      if (!sp.init(x, std::vector<double>(y, y + n_gamma)))
        return set_error(ctx, RG_EINVAL, "recombination spline setup failed");
      const std::vector<double>& h = sp.half_curvature();
      std::copy(h.begin(), h.end(), c.begin() + ((size_t)k * rows + r) * n_gamma);
    }
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->rec_knots) cudaFree(ctx->rec_knots);
  if (ctx->rec_y) cudaFree(ctx->rec_y);
  if (ctx->rec_c) cudaFree(ctx->rec_c);
  ctx->rec_knots = ctx->rec_y = ctx->rec_c = nullptr;
  ctx->rec_nz = ctx->rec_nt = ctx->rec_ng = 0;
  if (cudaMalloc((void**)&ctx->rec_knots, sizeof(double) * n_gamma) != cudaSuccess ||
      cudaMalloc((void**)&ctx->rec_y, sizeof(double) * 3 * per) != cudaSuccess ||
      cudaMalloc((void**)&ctx->rec_c, sizeof(double) * 3 * per) != cudaSuccess) {
    if (ctx->rec_knots) cudaFree(ctx->rec_knots);
    if (ctx->rec_y) cudaFree(ctx->rec_y);
    ctx->rec_knots = ctx->rec_y = ctx->rec_c = nullptr;
    return set_error(ctx, RG_ENOMEM, "cudaMalloc of the recombination tables failed");
  }
  cudaError_t e = cudaMemcpy(ctx->rec_knots, lnGamma, sizeof(double) * n_gamma, cudaMemcpyHostToDevice);
  for (int k = 0; k < 3 && e == cudaSuccess; ++k)
    e = cudaMemcpy(ctx->rec_y + (size_t)k * per, tabs[k], sizeof(double) * per, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(ctx->rec_c, c.data(), sizeof(double) * 3 * per, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    // no half-filled tables stay behind: find_HII_bubbles then asks for the tables again
    cudaFree(ctx->rec_knots);
    cudaFree(ctx->rec_y);
    cudaFree(ctx->rec_c);
    ctx->rec_knots = ctx->rec_y = ctx->rec_c = nullptr;
    return set_error(ctx, RG_ECUDA, std::string("copying the recombination tables: ") + cudaGetErrorString(e));
  }
  ctx->rec_nz = n_z;
  ctx->rec_nt = n_t;
  ctx->rec_ng = n_gamma;
  return RG_OK;
}

int rg_find_HII_bubbles(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g,
                        rg_hii_scalars* out) {
  if (!ctx || !p || !s || !g || !out || !s->ZZ) return RG_EINVAL;
  return find_hii(ctx, p, s, g, out, nullptr);
}

int rg_find_HII_bubbles_batch(rg_context* ctx, int n_units, const rg_params* p, const rg_snapshot* s,
                              const rg_grids* g, rg_hii_scalars* out) {
  if (!ctx || n_units < 0 || (n_units > 0 && (!p || !s || !g || !out))) return RG_EINVAL;
  if (n_units == 0) return RG_OK;
  for (int u = 0; u < n_units; ++u) {
    if (!s[u].ZZ) return set_error(ctx, RG_EINVAL, "snapshot without redshifts");
    if (p[u].ReionGridDim != p[0].ReionGridDim || p[u].BoxSize != p[0].BoxSize ||
        p[u].ReionFilterType != p[0].ReionFilterType || p[u].Flag_IncludeSpinTemp != p[0].Flag_IncludeSpinTemp ||
        p[u].Flag_BHFeedback != p[0].Flag_BHFeedback ||
        p[u].Flag_IncludeRecombinations != p[0].Flag_IncludeRecombinations ||
        p[u].UseMiniHalos != p[0].UseMiniHalos)
      return set_error(ctx, RG_EINVAL, "batch units differ in grid size, box, filter or feature flags");
  }
  // recombinations, Pop III sources and the plain mode: one snapshot at a time
  if (n_units == 1 || ctx->mode != RG_MODE_FUSED || p[0].Flag_IncludeRecombinations || p[0].UseMiniHalos) {
    for (int u = 0; u < n_units; ++u) {
      const int rc = find_hii(ctx, &p[u], &s[u], &g[u], &out[u], nullptr);
      if (rc) return rc;
    }
    return RG_OK;
  }
  for (int u = 0; u < n_units; ++u) {
    int rc = validate_common(ctx, &p[u]);
    if (rc) return rc;
    const rg_grids* gu = &g[u];
    if (s[u].snapshot < 0 || s[u].snapshot >= s[u].n_snapshots)
      return set_error(ctx, RG_EINVAL, "snapshot out of range");
    if (p[u].ReionRtoMFilterType < 0 || p[u].ReionRtoMFilterType > 1 || p[u].ReionFilterType < 0 ||
        p[u].ReionFilterType > 2 || !(p[u].ReionDeltaRFactor > 1.0))
      return set_error(ctx, RG_EINVAL, "filter or radius parameters out of range");
    if (!gu->deltax || !gu->stars || !gu->weighted_sfr || !gu->xH || !gu->r_bubble || !gu->z_at_ionization ||
        !gu->J_21_at_ionization || !gu->temp_kinetic_all_gas)
      return set_error(ctx, RG_EINVAL, "missing grid pointer");
    if (p[u].Flag_IncludeSpinTemp && (!gu->x_e_box || !gu->Tk_box))
      return set_error(ctx, RG_EINVAL, "spin temperature needs x_e_box and Tk_box");
    if (p[u].Flag_BHFeedback && (!gu->effective_bhm || !gu->effective_bhar))
      return set_error(ctx, RG_EINVAL, "BH feedback needs effective_bhm and effective_bhar");
  }
  int rc = ensure_tables(ctx, &p[0]);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  return hii_batch(ctx, n_units, p, s, g, out);
}

static int copy_grid(rg_context* ctx, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind,
                     cudaStream_t st = nullptr) {
  if (!dst || !src) return RG_OK;
  RG_CUDA_TRY(ctx, cudaMemcpyAsync(dst, src, bytes, kind, st ? st : ctx->stream));
  return RG_OK;
}

static int ensure_dev_grids(rg_context* ctx, const rg_params* p, int n_hist) {
  const bool need_spin = p->Flag_IncludeSpinTemp != 0;
  const bool need_bh = p->Flag_BHFeedback != 0;
  const bool need_rec = p->Flag_IncludeRecombinations != 0;
  const bool need_mini = p->UseMiniHalos != 0;
  if (ctx->dev_grids_ready) {
    const bool has_spin = ctx->dev_grids.Tk_box != nullptr;
    const bool has_bh = ctx->dev_grids.effective_bhm != nullptr;
    const bool has_rec = ctx->dev_grids.Gamma12 != nullptr;
    const bool has_mini = ctx->dev_grids.starsIII != nullptr;
    if ((!need_spin || has_spin) && (!need_bh || has_bh) && (!need_rec || has_rec) && (!need_mini || has_mini) &&
        ctx->dev_grids_nhist >= n_hist)
      return RG_OK;
    for (void* q : ctx->owned) cudaFree(q);
    ctx->owned.clear();
    ctx->dev_grids_ready = false;
  }
  int rc = rg_alloc_grids(ctx, p, n_hist, &ctx->dev_grids);
  if (rc) return rc;
  ctx->dev_grids_ready = true;
  ctx->dev_grids_nhist = n_hist;
  return RG_OK;
}

// The Pop III and recombination grids of the host forms: starsIII and weighted_sfrIII (Pop III),
// and with recombinations N_rec and effective_bhar, go with the first group of uploads (they are
// transformed, or with weighted_sfrIII only summed); r_bubble and the recombination grids come
// back after the step.
static int hii_extra_inputs(rg_context* ctx, const rg_params* p, const rg_grids* h, cudaStream_t cs) {
  const rg_grids& d = ctx->dev_grids;
  const size_t n = (size_t)ctx->N;
  const size_t bp = n * n * 2 * (n / 2 + 1) * sizeof(float);
  if (p->UseMiniHalos) {
    // Pop III grids: both transformed with recombinations, weighted_sfrIII otherwise only summed
    if (!h->starsIII || !h->weighted_sfrIII) return set_error(ctx, RG_EINVAL, "UseMiniHalos needs starsIII and weighted_sfrIII");
    int r = copy_grid(ctx, (void*)d.starsIII, h->starsIII, bp, cudaMemcpyHostToDevice, cs);
    if (!r) r = copy_grid(ctx, (void*)d.weighted_sfrIII, h->weighted_sfrIII, bp, cudaMemcpyHostToDevice, cs);
    if (r) return r;
  }
  if (!p->Flag_IncludeRecombinations) return RG_OK;
  if (!h->N_rec || !h->Gamma12 || !h->residual_xH || !h->clumping_factor || !h->t_resp)
    return set_error(ctx, RG_EINVAL, "recombinations need Gamma12, N_rec, residual_xH, clumping_factor, t_resp");
  int rc = copy_grid(ctx, d.N_rec, h->N_rec, bp, cudaMemcpyHostToDevice, cs);
  if (!rc && p->Flag_BHFeedback)
    rc = copy_grid(ctx, (void*)d.effective_bhar, h->effective_bhar, bp, cudaMemcpyHostToDevice, cs);
  return rc;
}

static int hii_extra_outputs(rg_context* ctx, const rg_params* p, const rg_grids* h, cudaStream_t st) {
  if (!p->Flag_IncludeRecombinations) return RG_OK;
  const rg_grids& d = ctx->dev_grids;
  const size_t n = (size_t)ctx->N;
  const size_t bp = n * n * 2 * (n / 2 + 1) * sizeof(float), br = n * n * n * sizeof(float);
  const auto D2H = cudaMemcpyDeviceToHost;
  int rc;
  if ((rc = copy_grid(ctx, h->r_bubble, d.r_bubble, br, D2H, st))) return rc;
  if ((rc = copy_grid(ctx, h->Gamma12, d.Gamma12, br, D2H, st))) return rc;
  if ((rc = copy_grid(ctx, h->N_rec, d.N_rec, bp, D2H, st))) return rc;
  if ((rc = copy_grid(ctx, h->residual_xH, d.residual_xH, br, D2H, st))) return rc;
  if ((rc = copy_grid(ctx, h->clumping_factor, d.clumping_factor, br, D2H, st))) return rc;
  return copy_grid(ctx, h->t_resp, d.t_resp, br, D2H, st);
}

int rg_find_HII_bubbles_host(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* h,
                             rg_hii_scalars* out) {
  if (!ctx || !p || !s || !h || !out || !s->ZZ) return RG_EINVAL;
  int rc = validate_common(ctx, p);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  if ((rc = ensure_dev_grids(ctx, p, 0))) return rc;
  const rg_grids& d = ctx->dev_grids;
  const size_t n = (size_t)ctx->N;
  const size_t bp = n * n * 2 * (n / 2 + 1) * sizeof(float), br = n * n * n * sizeof(float);
  const auto H2D = cudaMemcpyHostToDevice;
  cudaStream_t cs = ctx->copy_stream;
  const bool plain = ctx->mode == RG_MODE_PLAIN;
  // uploads in the order the snapshot reads them: the transformed grids, the ionisation state
  // (first z pass), the closing-pass grids; each group's event gates its first reader
  Staging stg;
  if ((rc = copy_stream_after_prior(ctx))) return rc;
  if ((rc = copy_grid(ctx, (void*)d.deltax, h->deltax, bp, H2D, cs))) return rc;
  if ((rc = copy_grid(ctx, (void*)d.stars, h->stars, bp, H2D, cs))) return rc;
  if (p->Flag_IncludeSpinTemp && (rc = copy_grid(ctx, (void*)d.x_e_box, h->x_e_box, bp, H2D, cs))) return rc;
  const bool rec = p->Flag_IncludeRecombinations != 0;
  if (p->Flag_BHFeedback && (rc = copy_grid(ctx, (void*)d.effective_bhm, h->effective_bhm, bp, H2D, cs))) return rc;
  if ((rc = hii_extra_inputs(ctx, p, h, cs))) return rc;
  if ((plain || rec) && (rc = copy_grid(ctx, (void*)d.weighted_sfr, h->weighted_sfr, bp, H2D, cs))) return rc;
  if ((rc = stage_record(ctx, 1, cs, &stg.inputs))) return rc;
  if ((rc = copy_grid(ctx, d.z_at_ionization, h->z_at_ionization, br, H2D, cs))) return rc;
  if ((rc = copy_grid(ctx, d.J_21_at_ionization, h->J_21_at_ionization, br, H2D, cs))) return rc;
  if (rec && (rc = copy_grid(ctx, d.Gamma12, h->Gamma12, br, H2D, cs))) return rc;
  if ((rc = stage_record(ctx, 2, cs, &stg.state))) return rc;
  if ((rc = copy_grid(ctx, d.temp_kinetic_all_gas, h->temp_kinetic_all_gas, br, H2D, cs))) return rc;
  if (p->Flag_IncludeSpinTemp && (rc = copy_grid(ctx, (void*)d.Tk_box, h->Tk_box, br, H2D, cs))) return rc;
  if (!plain && !rec && (rc = copy_grid(ctx, (void*)d.weighted_sfr, h->weighted_sfr, bp, H2D, cs))) return rc;
  if (p->Flag_BHFeedback && !rec &&
      (rc = copy_grid(ctx, (void*)d.effective_bhar, h->effective_bhar, bp, H2D, cs)))
    return rc;
  if ((rc = stage_record(ctx, 3, cs, &stg.closing))) return rc;
  stg.host_r_bubble = h->r_bubble;
  rc = find_hii(ctx, p, s, &d, out, &stg);
  if (rc) {
    cudaStreamSynchronize(cs);   // no copy of the caller's arrays outlives the call
    return rc;
  }
  const auto D2H = cudaMemcpyDeviceToHost;
  if ((rc = copy_grid(ctx, h->xH, d.xH, br, D2H))) return rc;
  if ((rc = copy_grid(ctx, h->z_at_ionization, d.z_at_ionization, br, D2H))) return rc;
  if ((rc = copy_grid(ctx, h->J_21_at_ionization, d.J_21_at_ionization, br, D2H))) return rc;
  if ((rc = copy_grid(ctx, h->temp_kinetic_all_gas, d.temp_kinetic_all_gas, br, D2H))) return rc;
  if ((rc = hii_extra_outputs(ctx, p, h, ctx->stream))) return rc;
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(cs));
  return RG_OK;
}

int rg_debug_filter_roundtrip(rg_context* ctx, const rg_params* p, const float* d_in, float* d_out, double R,
                              int filter_type) {
  if (!ctx || !p || !d_in || !d_out) return RG_EINVAL;
  int rc = validate_common(ctx, p);
  if (rc) return rc;
  if (filter_type > 2) return set_error(ctx, RG_EINVAL, "filter_type must be <= 2");
  cudaSetDevice(ctx->device);
  if ((rc = debug_roundtrip(ctx, p, d_in, d_out, R, filter_type))) return rc;
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

int rg_debug_ts_tables(const rg_params* p, const rg_snapshot* s, int n_hist, double x_e_ave,
                       double collapse_fraction, int max_shells, double* shells, double* freq, float* coef) {
  if (!p || !s || !s->ZZ || !shells || !coef || n_hist < 0) return RG_EINVAL;
  if (s->snapshot < 0 || s->snapshot >= s->n_snapshots) return RG_EINVAL;
  const int nS = p->TsNumFilterSteps;
  if (nS < 1 || nS > max_shells) return RG_EINVAL;
  TsShells sh = ts_shells(p, s->ZZ, s->n_snapshots, s->snapshot, n_hist);
  if (sh.error) return RG_EINVAL;
  TsTables tb;
  if (freq) {
    if (!s->stored_fcoll && s->snapshot > 0) return RG_EINVAL;
    Tables t;
    if (!p->TablesForXHeatingDir) return RG_ETABLE;
    if (!load_tables(p->TablesForXHeatingDir, p->ReionNionPhotPerBary, &t).empty()) return RG_ETABLE;
    std::string msg;
    int rc = ts_tables(p, t, sh, s->ZZ[s->snapshot], x_e_ave, collapse_fraction, s->ZZ, s->stored_fcoll,
                       s->snapshot, &tb, &msg);
    if (rc) return rc;
    for (int k = 0; k < 3; ++k) {
      const std::vector<double>& v = k == 0 ? tb.heat : k == 1 ? tb.ion : tb.lya;
      for (int m = 0; m < x_int_NXHII; ++m)
        for (int r = 0; r < nS; ++r) freq[((size_t)k * x_int_NXHII + m) * nS + r] = v[(size_t)m * nS + r];
    }
  }
  for (int r = 0; r < nS; ++r) {
    shells[r] = sh.R[r];
    shells[nS + r] = sh.zpp_edge[r];
    shells[2 * nS + r] = sh.zpp[r];
    shells[3 * nS + r] = sh.dzpp[r];
    shells[4 * nS + r] = sh.dt_dzpp[r];
    shells[5 * nS + r] = freq ? tb.sum_lyn[r] : 0.0;
    for (int k = 0; k < sh.nsrc; ++k) coef[(size_t)r * sh.nsrc + k] = sh.coef[(size_t)r * sh.nsrc + k];
  }
  return RG_OK;
}

int rg_debug_ts_agn_tables(const rg_params* p, const rg_snapshot* s, int n_hist, double x_e_ave,
                           double collapse_fraction, int max_shells, double* agn, double* const_zp) {
  if (!p || !s || !s->ZZ || !agn || !const_zp || n_hist < 0) return RG_EINVAL;
  if (s->snapshot < 0 || s->snapshot >= s->n_snapshots) return RG_EINVAL;
  if (p->Flag_IncludeAGNXray < 0 || p->Flag_IncludeAGNXray > 3) return RG_EINVAL;
  const int nS = p->TsNumFilterSteps;
  if (nS < 1 || nS > max_shells) return RG_EINVAL;
  if (!s->stored_fcoll && s->snapshot > 0) return RG_EINVAL;
  TsShells sh = ts_shells(p, s->ZZ, s->n_snapshots, s->snapshot, n_hist);
  if (sh.error) return RG_EINVAL;
  Tables t;
  if (!p->TablesForXHeatingDir) return RG_ETABLE;
  if (!load_tables(p->TablesForXHeatingDir, p->ReionNionPhotPerBary, &t).empty()) return RG_ETABLE;
  TsTables tb;
  std::string msg;
  int rc = ts_tables(p, t, sh, s->ZZ[s->snapshot], x_e_ave, collapse_fraction, s->ZZ, s->stored_fcoll, s->snapshot,
                     &tb, &msg);
  if (rc) return rc;
  for (int b = 0; b < 2; ++b)
    for (int k = 0; k < 3; ++k)
      for (int m = 0; m < x_int_NXHII; ++m)
        for (int r = 0; r < nS; ++r)
          agn[(((size_t)b * 3 + k) * x_int_NXHII + m) * nS + r] =
              tb.agn[b][k].empty() ? 0.0 : tb.agn[b][k][(size_t)m * nS + r];
  const TsPrefactors pf = ts_prefactors(p, s->ZZ[s->snapshot]);
  const_zp[0] = pf.const_zp_prefactor_GAL;
  const_zp[1] = pf.const_zp_prefactor_AGN[0];
  const_zp[2] = pf.const_zp_prefactor_AGN[1];
  return RG_OK;
}

int rg_profile_enable(rg_context* ctx, int on) {
  if (!ctx) return RG_EINVAL;
  prof_resolve(ctx);
  ctx->prof_on = on != 0;
  ctx->prof_stats.clear();
  return RG_OK;
}

int rg_profile_read(rg_context* ctx, rg_kernel_stat* out, int max, int* n) {
  if (!ctx || !n) return RG_EINVAL;
  cudaStreamSynchronize(ctx->stream);
  prof_resolve(ctx);
  *n = (int)ctx->prof_stats.size();
  for (int i = 0; i < *n && i < max && out; ++i) out[i] = ctx->prof_stats[i];
  return RG_OK;
}

static int compute_ts(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g,
                      const rg_grids* src_host, rg_ts_scalars* out, const Staging* stg = nullptr) {
  int rc = validate_common(ctx, p);
  if (rc) return rc;
  if (!s->ZZ) return set_error(ctx, RG_EINVAL, "ZZ is required");
  if (s->snapshot < 0 || s->snapshot >= s->n_snapshots) return set_error(ctx, RG_EINVAL, "snapshot out of range");
  const int N = ctx->N;
  if (N < 8 || (N & (N - 1)) != 0)
    return set_error(ctx, RG_EUNSUPPORTED, "ComputeTs needs a power-of-two ReionGridDim");
  if (p->Flag_IncludeAGNXray < 0 || p->Flag_IncludeAGNXray > 3)
    return set_error(ctx, RG_EINVAL, "Flag_IncludeAGNXray must be 0, 1, 2 or 3");
  if (p->UseMiniHalos)
    return set_error(ctx, RG_EUNSUPPORTED, "UseMiniHalos: the Pop III channels of ComputeTs are not built");
  if (p->TsHeatingFilterType < 0 || p->TsHeatingFilterType > 2)
    return set_error(ctx, RG_EINVAL, "TsHeatingFilterType must be 0, 1 or 2");
  if (p->TsNumFilterSteps < 1 || p->TsNumFilterSteps > 1024)
    return set_error(ctx, RG_EINVAL, "TsNumFilterSteps must be in [1, 1024]");
  if (!g->deltax || !g->stars || !g->x_e_box_prev || !g->x_e_box || !g->Tk_box || !g->TS_box)
    return set_error(ctx, RG_EINVAL, "missing grid pointer");
  const rg_grids* sg = src_host ? src_host : g;
  if (sg->n_hist < 0 || (sg->n_hist > 0 && (!sg->sfr_histories || !sg->xray_luminosity_histories)))
    return set_error(ctx, RG_EINVAL, "n_hist > 0 needs sfr_histories and xray_luminosity_histories");
  const bool homog = (s->ZZ[s->snapshot] - p->ReionMaxHeatingRedshift) >= -0.0001;
  if (!homog && (!sg->sfr || !sg->xray_luminosity))
    return set_error(ctx, RG_EINVAL, "ComputeTs needs the sfr and xray_luminosity grids");
  const bool agn_soft = p->Flag_IncludeAGNXray == 1 || p->Flag_IncludeAGNXray == 3;
  const bool agn_hard = p->Flag_IncludeAGNXray == 1 || p->Flag_IncludeAGNXray == 2;
  if (!homog && ((agn_soft && (!sg->bh_xray_soft || (sg->n_hist > 0 && !sg->bh_xray_histories_soft))) ||
                 (agn_hard && (!sg->bh_xray_hard || (sg->n_hist > 0 && !sg->bh_xray_histories_hard)))))
    return set_error(ctx, RG_EINVAL, "Flag_IncludeAGNXray needs bh_xray_soft/_hard and their histories");
  if ((rc = ensure_tables(ctx, p))) return rc;
  cudaSetDevice(ctx->device);
  rc = ts_snapshot(ctx, p, s, g, out, src_host, stg);
  if (rc == RG_OK && s->stored_fcoll) s->stored_fcoll[s->snapshot] = out->collapse_fraction;
  return rc;
}

int rg_compute_Ts(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g, rg_ts_scalars* out) {
  if (!ctx || !p || !s || !g || !out) return RG_EINVAL;
  return compute_ts(ctx, p, s, g, nullptr, out);
}

int rg_compute_Ts_host(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* h,
                       rg_ts_scalars* out) {
  if (!ctx || !p || !s || !h || !out) return RG_EINVAL;
  int rc = validate_common(ctx, p);
  if (rc) return rc;
  if (!p->Flag_IncludeSpinTemp) return set_error(ctx, RG_EINVAL, "rg_compute_Ts_host needs Flag_IncludeSpinTemp=1");
  cudaSetDevice(ctx->device);
  if ((rc = ensure_dev_grids(ctx, p, 0))) return rc;
  const rg_grids& d = ctx->dev_grids;
  const size_t n = (size_t)ctx->N;
  const size_t bp = n * n * 2 * (n / 2 + 1) * sizeof(float), br = n * n * n * sizeof(float);
  const auto H2D = cudaMemcpyHostToDevice;
  cudaStream_t cs = ctx->copy_stream;
  // deltax, stars and x_e_box_prev feed the first reduction; Tk_box only the evolution step.
  // The source grids are staged from h inside the step (only the history slots in use).
  Staging stg;
  if ((rc = copy_stream_after_prior(ctx))) return rc;
  if ((rc = copy_grid(ctx, (void*)d.deltax, h->deltax, bp, H2D, cs))) return rc;
  if ((rc = copy_grid(ctx, (void*)d.stars, h->stars, bp, H2D, cs))) return rc;
  if ((rc = copy_grid(ctx, d.x_e_box_prev, h->x_e_box_prev, bp, H2D, cs))) return rc;
  if ((rc = stage_record(ctx, 1, cs, &stg.inputs))) return rc;
  if ((rc = copy_grid(ctx, d.Tk_box, h->Tk_box, br, H2D, cs))) return rc;
  if ((rc = stage_record(ctx, 3, cs, &stg.closing))) return rc;
  if ((rc = compute_ts(ctx, p, s, &d, h, out, &stg))) {
    cudaStreamSynchronize(cs);   // no copy of the caller's arrays outlives the call
    return rc;
  }
  const auto D2H = cudaMemcpyDeviceToHost;
  if ((rc = copy_grid(ctx, h->x_e_box_prev, d.x_e_box_prev, bp, D2H))) return rc;
  if ((rc = copy_grid(ctx, h->x_e_box, d.x_e_box, bp, D2H))) return rc;
  if ((rc = copy_grid(ctx, h->Tk_box, d.Tk_box, br, D2H))) return rc;
  if ((rc = copy_grid(ctx, h->TS_box, d.TS_box, br, D2H))) return rc;
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(cs));
  return RG_OK;
}

// The snapshot's reionization block (dracarys.c:383-391): ComputeTs (with the spin temperature),
// find_HII_bubbles and, when host->delta_T is given, ComputeBrightnessTemperatureBox, on the
// HOST arrays.  Each input crosses PCIe once and in the order the steps read it (ComputeTs'
// inputs, its history sources, then find_HII's state and closing-pass grids behind them on the
// same copy stream); the grids the step hands from ComputeTs to find_HII_bubbles and to delta_T
// (x_e_box, Tk_box, TS_box, deltax, xH) stay on the device; ComputeTs' outputs go back on a
// second copy stream while find_HII_bubbles runs.
int rg_reion_step_host(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* h,
                       rg_ts_scalars* ts_out, rg_hii_scalars* hii_out, double* volume_ave_Tb) {
  if (!ctx || !p || !s || !h || !hii_out || !s->ZZ) return RG_EINVAL;
  const bool spin = p->Flag_IncludeSpinTemp != 0;
  if (spin && !ts_out) return RG_EINVAL;
  if (h->delta_T && !volume_ave_Tb) return RG_EINVAL;
  int rc = validate_common(ctx, p);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  if ((rc = ensure_dev_grids(ctx, p, 0))) return rc;
  const rg_grids& d = ctx->dev_grids;
  const size_t n = (size_t)ctx->N;
  const size_t bp = n * n * 2 * (n / 2 + 1) * sizeof(float), br = n * n * n * sizeof(float);
  const auto H2D = cudaMemcpyHostToDevice;
  const auto D2H = cudaMemcpyDeviceToHost;
  cudaStream_t cs = ctx->copy_stream, co = ctx->copy_stream_out, st = ctx->stream;
  const bool plain = ctx->mode == RG_MODE_PLAIN;
  const bool rec = p->Flag_IncludeRecombinations != 0;
  auto fail = [&](int code) {
    cudaStreamSynchronize(cs);   // no copy of the caller's arrays outlives the call
    cudaStreamSynchronize(co);
    return code;
  };
  // the velocity grid of delta_T's velocity modes goes to its own device buffer
  const bool vel = h->delta_T && spin && p->Flag_IncludePecVelsFor21cm > 0;
  if (vel && !h->vel) return set_error(ctx, RG_EINVAL, "missing grid pointer");
  if (vel && (rc = ensure_device(ctx, &ctx->vel_stage, &ctx->vel_stage_elems, bp / sizeof(float)))) return rc;
  if ((rc = copy_stream_after_prior(ctx))) return rc;
  RG_CUDA_TRY(ctx, cudaStreamWaitEvent(co, ctx->stage_events[0], 0));
  Staging hs;   // find_HII's copies
  // find_HII's own grids: the state for its first z pass, the closing-pass grids
  auto hii_uploads = [&]() -> int {
    int r;
    if ((plain || rec) && (r = copy_grid(ctx, (void*)d.weighted_sfr, h->weighted_sfr, bp, H2D, cs))) return r;
    if (p->Flag_BHFeedback && (r = copy_grid(ctx, (void*)d.effective_bhm, h->effective_bhm, bp, H2D, cs))) return r;
    if ((r = hii_extra_inputs(ctx, p, h, cs))) return r;
    if ((r = stage_record(ctx, 5, cs, &hs.inputs))) return r;
    if ((r = copy_grid(ctx, d.z_at_ionization, h->z_at_ionization, br, H2D, cs))) return r;
    if ((r = copy_grid(ctx, d.J_21_at_ionization, h->J_21_at_ionization, br, H2D, cs))) return r;
    if (rec && (r = copy_grid(ctx, d.Gamma12, h->Gamma12, br, H2D, cs))) return r;
    if ((r = stage_record(ctx, 6, cs, &hs.state))) return r;
    if ((r = copy_grid(ctx, d.temp_kinetic_all_gas, h->temp_kinetic_all_gas, br, H2D, cs))) return r;
    if (!plain && !rec && (r = copy_grid(ctx, (void*)d.weighted_sfr, h->weighted_sfr, bp, H2D, cs))) return r;
    if (p->Flag_BHFeedback && !rec &&
        (r = copy_grid(ctx, (void*)d.effective_bhar, h->effective_bhar, bp, H2D, cs)))
      return r;
    if (vel && (r = copy_grid(ctx, ctx->vel_stage, h->vel, bp, H2D, cs))) return r;   // delta_T, after find_HII
    return stage_record(ctx, 7, cs, &hs.closing);
  };
  if ((rc = copy_grid(ctx, (void*)d.deltax, h->deltax, bp, H2D, cs))) return fail(rc);
  if ((rc = copy_grid(ctx, (void*)d.stars, h->stars, bp, H2D, cs))) return fail(rc);
  if (spin) {
    Staging ts;
    if ((rc = copy_grid(ctx, d.x_e_box_prev, h->x_e_box_prev, bp, H2D, cs))) return fail(rc);
    if ((rc = stage_record(ctx, 1, cs, &ts.inputs))) return fail(rc);
    if ((rc = copy_grid(ctx, d.Tk_box, h->Tk_box, br, H2D, cs))) return fail(rc);
    if ((rc = stage_record(ctx, 3, cs, &ts.closing))) return fail(rc);
    ts.after_sources = hii_uploads;
    if ((rc = compute_ts(ctx, p, s, &d, h, ts_out, &ts))) return fail(rc);
    // ComputeTs' outputs go back while find_HII_bubbles runs (they are final, st is idle here)
    if ((rc = copy_grid(ctx, h->x_e_box_prev, d.x_e_box_prev, bp, D2H, co))) return fail(rc);
    if ((rc = copy_grid(ctx, h->x_e_box, d.x_e_box, bp, D2H, co))) return fail(rc);
    if ((rc = copy_grid(ctx, h->Tk_box, d.Tk_box, br, D2H, co))) return fail(rc);
    if ((rc = copy_grid(ctx, h->TS_box, d.TS_box, br, D2H, co))) return fail(rc);
  } else {
    if ((rc = hii_uploads())) return fail(rc);
  }
  // deltax and stars (and x_e_box, Tk_box from ComputeTs) are on the device already
  hs.host_r_bubble = h->r_bubble;
  if ((rc = find_hii(ctx, p, s, &d, hii_out, &hs))) return fail(rc);
  if ((rc = copy_grid(ctx, h->xH, d.xH, br, D2H, co))) return fail(rc);
  if ((rc = copy_grid(ctx, h->z_at_ionization, d.z_at_ionization, br, D2H, co))) return fail(rc);
  if ((rc = copy_grid(ctx, h->J_21_at_ionization, d.J_21_at_ionization, br, D2H, co))) return fail(rc);
  if ((rc = copy_grid(ctx, h->temp_kinetic_all_gas, d.temp_kinetic_all_gas, br, D2H, co))) return fail(rc);
  if ((rc = hii_extra_outputs(ctx, p, h, co))) return fail(rc);
  if (h->delta_T) {
    rg_grids dd = d;
    if (vel) dd.vel = ctx->vel_stage;
    if ((rc = rg_delta_T(ctx, p, s, &dd, volume_ave_Tb))) return fail(rc);
    if ((rc = copy_grid(ctx, h->delta_T, d.delta_T, br, D2H))) return fail(rc);
  }
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(cs));
  RG_CUDA_TRY(ctx, cudaStreamSynchronize(co));
  return RG_OK;
}

}  // extern "C"
