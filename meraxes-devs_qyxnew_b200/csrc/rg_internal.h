// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

#include "../../include/rg_b200.h"
#include "rg_tables.h"

namespace rg {

// physical constants of the reference (src/meraxes.h:21-67, src/core/reionization.h:10-44)
constexpr double GRAVITY = 6.672e-8;
constexpr double SOLAR_MASS = 1.989e33;
constexpr double SOLAR_LUM = 3.826e33;
constexpr double BOLTZMANN = 1.3806e-16;
constexpr double SPEED_OF_LIGHT = 2.9979e10;
constexpr double PLANCK = 6.6262e-27;
constexpr double PROTONMASS = 1.6726e-24;
constexpr double HUBBLE = 3.2407789e-18;
constexpr double SEC_PER_MEGAYEAR = 3.155e13;
constexpr double SEC_PER_YEAR = 3.155e7;
constexpr double MPC = 3.086e24;
constexpr double XRAY_LUMINOSITY_UNIT = 1.0e40;
constexpr double TCMB = 2.728;
constexpr double NU_over_EV = 1.60217646e-12 / PLANCK;
constexpr double NUIONIZATION = 13.60 * NU_over_EV;
constexpr double HeI_NUIONIZATION = 24.59 * NU_over_EV;
constexpr double HeII_NUIONIZATION = NUIONIZATION * 4;
constexpr double NU_LA = 10.2 * NU_over_EV;
constexpr double T_RE = 1e4;
constexpr float REL_TOL = 1e-5f;
constexpr float ABS_TOL = 1e-8f;
constexpr double SIGMA_HI = 6.3e-18;
constexpr double TINY = 1e-30;
constexpr double L_FACTOR = 0.620350491;
constexpr float MAX_TK = 5e4f;
constexpr float MIN_TK = 0.1f;
constexpr double FRACT_FLOAT_ERR = 1e-7;
constexpr double CLUMPING_FACTOR = 2.0;
constexpr double T21 = 0.0628;
constexpr double A10_HYPERFINE = 2.85e-15;
constexpr double R_XLy_MAX = 500.0;
constexpr int x_int_NXHII = 14;
constexpr int x_int_NENERGY = 258;
constexpr int NSPEC_MAX = 23;
constexpr int RECFAST_NPTS = 501;
constexpr int KAPPA_10_NPTS = 27;
constexpr int KAPPA_10_elec_NPTS = 20;
constexpr int KAPPA_10_pH_NPTS = 17;
// default bounds of the device waits
#define RG_XY_POLL_LIMIT (1 << 22)
#define RG_TS_ITER_LIMIT 10000

struct cf;

// Derived unit quantities, set_units() (src/core/init.c:203-225).
struct Units {
  double UnitTime_in_s, Hubble, G, RhoCrit;
};
Units make_units(const rg_params* p);
double hubble_time_at(const rg_params* p, double z);
double dtdz(const rg_params* p, float z);
double rtom(const rg_params* p, double R);
float cT_approx(float z);

// Radius schedule of the excursion-set loop.
std::vector<std::pair<double, bool>> radius_schedule(const rg_params* p, double z);

// Status helpers
int set_error(rg_context* ctx, int status, const std::string& msg);
#define RG_CUDA_TRY(ctx, call)                                                        \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return ::rg::set_error((ctx), RG_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// A context buffer of at least `need` elements: kept when large enough, else freed and allocated
// again (the old contents are not kept).
template <typename T>
int ensure_device(rg_context* ctx, T** ptr, size_t* have, size_t need) {
  if (*ptr && *have >= need) return RG_OK;
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  *have = 0;
  const cudaError_t e = cudaMalloc((void**)ptr, sizeof(T) * (need ? need : 1));
  if (e != cudaSuccess) return set_error(ctx, RG_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  *have = need;
  return RG_OK;
}

// Per-snapshot constants of the barrier test.
struct HiiConst {
  float redshift, TK, cT_ad;
  int uvb, spin, bh, rec, mini;
};

// Recombination tables on the device (splined_recombination, recombinations.c:35-84).
struct RecTables {
  const double* knots;   // ln Gamma12 knots [ng]
  const double* y;       // [3][nz * nt][ng]: ln RR, CF, ln RNH
  const double* c;       // natural-spline coefficients, same layout
  int nz, nt, ng;
  double lng_lo, lng_hi; // knots[0] and the float-rounded upper bound of the table
};

constexpr int HII_NSUM = 10;  // closing-pass sums
constexpr int KB_MAX = 16;    // radii per batch

// Forward r2c of ng padded real grids into spectra spec_base + g * stride, scaled.
int fft_forward(rg_context* ctx, int n, const float* const* d_real, int ng, cf* spec_base, size_t stride,
                double scale, cudaStream_t st);
// W[r][n2] for the radii in d_radii (filter() closed forms, double precision); for the sharp-k
// filter also d_wcut[r] (when given), the last n2 of the step, so W[r][n2] == (n2 <= d_wcut[r])
int window_table(rg_context* ctx, double box, const double* d_radii, int nr, int ftype, float* d_wtab, int n2max,
                 cudaStream_t st, int* d_wcut = nullptr);
// Uploads still in flight on the context's copy stream when a snapshot is enqueued (the host
// entry points): each stage of the snapshot waits for the event of the grids it reads or
// overwrites, so the copies overlap the work that needs none of them.  Null events are ready.
struct Staging {
  cudaEvent_t inputs = nullptr;    // grids of the forward transforms (Ts: also of the first reduction)
  cudaEvent_t state = nullptr;     // find_HII: z_at_ionization, J_21_at_ionization (first z pass)
  cudaEvent_t closing = nullptr;   // find_HII: temperature, Tk_box, weighted_sfr, effective_bhar
                                   // (closing pass); Ts: Tk_box (the evolution step)
  float* host_r_bubble = nullptr;  // find_HII: copy r_bubble here on the copy stream once zeroed
  // ComputeTs: called once all of its own copies are queued and before the host first waits
  // for the device, so a caller can queue the next step's copies behind them
  std::function<int()> after_sources;
};
int stage_wait(rg_context* ctx, cudaEvent_t ev, cudaStream_t st);
// record event i of the context's staging pool on st (events 0-3 are used by the host entry
// points, 4 and up by the source groups of ComputeTs)
int stage_record(rg_context* ctx, size_t i, cudaStream_t st, cudaEvent_t* out);

// The excursion-set step on device grids (rg_hii.cu).
int hii_snapshot(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g, rg_hii_scalars* out,
                 const Staging* stg = nullptr);
// find_HII_bubbles for nu snapshots of this size with the same radii, device grids, fused mode:
// the forward transforms and every radius batch's x/y passes of all of them in shared launches,
// the z passes per snapshot, one host synchronisation.
int hii_batch(rg_context* ctx, int nu, const rg_params* p, const rg_snapshot* s, const rg_grids* g,
              rg_hii_scalars* out);
// The spin-temperature step on device grids (rg_ts.cu).  With src_host, the sfr /
// xray_luminosity grids and their histories are read from those HOST arrays instead of g, and
// only the history slots the shells use are copied to the device (on the copy stream, one
// event per group of forward transforms).
int ts_snapshot(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g, rg_ts_scalars* out,
                const rg_grids* src_host = nullptr, const Staging* stg = nullptr);
// Unnormalised c2r of the spectrum in ctx->spec into a padded real grid (the context's inverse
// passes, no window); the caller checks the fused pass's error word (xy_ctrl_check) after a sync.
int spectrum_to_padded(rg_context* ctx, float* d_out, cudaStream_t st);
// Forward + (windowed) inverse of one padded grid, for tests.
int debug_roundtrip(rg_context* ctx, const rg_params* p, const float* d_in, float* d_out, double R, int ftype);
int reduce_partials(rg_context* ctx, const double* partials, int nblocks, int nsum, double* d_out, cudaStream_t st);
double* ensure_partials(rg_context* ctx, size_t n);
int ensure_tables(rg_context* ctx, const rg_params* p);
int validate_common(rg_context* ctx, const rg_params* p);

int twiddles_for(rg_context* ctx, int n, const cf** out);

// Control words of the fused x/y passes: xy_ctrl_reset sizes them for up to max_jobs jobs per
// launch and clears the error word (once per snapshot); xy_ctrl_check copies the error word to
// the host after a stream sync and returns RG_ETIMEDOUT when a wait ran out.
int xy_ctrl_reset(rg_context* ctx, size_t max_jobs, cudaStream_t st);
int xy_ctrl_check(rg_context* ctx, cudaStream_t st);

// Per-kernel event timing (active when ctx->prof_on).  prof_begin records a start event on
// the stream; prof_end records the stop event and the launch's algorithmic bytes.
void prof_begin(rg_context* ctx, const char* name, cudaStream_t st);
void prof_end(rg_context* ctx, double alg_bytes, cudaStream_t st);
void prof_resolve(rg_context* ctx);   // after a stream sync: fold finished events into the stats

}  // namespace rg

// The opaque context.
struct rg_context {
  int device = 0;
  int N = 0;
  int mode = RG_MODE_FUSED;
  int radius_batch = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string last_error;
  // twiddle tables keyed by transform length
  std::vector<std::pair<int, rg::cf*>> twiddles;
  // unfiltered spectra [grid][N/2+1][N][N] and per-radius work buffers [radius][grid][...]
  rg::cf* spec = nullptr;
  size_t spec_elems = 0;
  rg::cf* work = nullptr;
  size_t work_elems = 0;
  uint32_t* bits = nullptr;      // per-cell state between radius batches, one byte per cell
  size_t bits_elems = 0;
  float* wtab = nullptr;         // window table [nR][n2max+1]
  size_t wtab_elems = 0;
  int* wcut = nullptr;           // sharp-k window: last n2 of each row's step
  size_t wcut_elems = 0;
  float* ps_pad = nullptr;       // power spectrum: padded real input of the transform
  size_t ps_pad_elems = 0;
  float* ps_stage = nullptr;     // power spectrum from host delta_T: its device copy
  size_t ps_stage_elems = 0;
  float* vel_work = nullptr;     // delta_T velocity modes: [converted velocity][its z gradient], padded
  size_t vel_work_elems = 0;
  float* vel_stage = nullptr;    // rg_delta_T_host: device copy of the caller's velocity grid
  size_t vel_stage_elems = 0;
  int* ngp_bad = nullptr;        // rg_deposit_ngp: count of galaxies below the box
  size_t ngp_bad_elems = 0;
  float2* ts_agn = nullptr;       // ComputeTs: per-cell AGN heating sums of the two AGN units
  size_t ts_agn_elems = 0;
  // recombination tables (rg_set_recombination_tables): knots, and per table and (z, T) row the
  // values and the natural-spline coefficients c (half the second derivative), [3][nz*nt][ng]
  double* rec_knots = nullptr;
  double* rec_y = nullptr;
  double* rec_c = nullptr;
  int rec_nz = 0, rec_nt = 0, rec_ng = 0;
  double* partials = nullptr;
  size_t partials_elems = 0;
  double* d_sums = nullptr;      // reduced sums
  double* h_sums = nullptr;      // pinned host copy
  double* batch_sums = nullptr;  // rg_find_HII_bubbles_batch: reduced sums per snapshot [unit][32]
  size_t batch_sums_elems = 0;
  double* h_batch_sums = nullptr;   // their pinned host copy (h_batch_sums_elems snapshots)
  size_t h_batch_sums_elems = 0;
  // device grids owned by the context (rg_alloc_grids / host entry points)
  std::vector<void*> owned;
  rg_grids dev_grids{};
  bool dev_grids_ready = false;
  int dev_grids_nhist = 0;
  // host coefficient engine tables, loaded on first use from TablesForXHeatingDir
  rg::Tables tables;
  double* d_radii = nullptr;     // device copy of the radius list
  size_t d_radii_elems = 0;
  float* ts_stage = nullptr;     // ComputeTs source grids staged from host memory [slot][2][padded]
  size_t ts_stage_elems = 0;
  float4* ts_sums = nullptr;     // ComputeTs per-cell shell sums (FP32, scaled) [N^3]
  size_t ts_sums_elems = 0;
  char* ts_const = nullptr;      // ComputeTs device constants and per-shell coefficients
  size_t ts_const_elems = 0;
  // fused x/y pass control words: [0] error word, [1] item counter, [2 ..) per-job counts
  uint32_t* xy_ctrl = nullptr;
  size_t xy_ctrl_elems = 0;
  // bounds of the device waits (rg_debug_set_wait_limits): polls of a fused-pass Y item for its
  // plane's X items, whether X items signal at all, and get_Ts fixed-point iterations per cell
  int xy_poll_limit = RG_XY_POLL_LIMIT;
  int xy_signal = 1;
  int ts_iter_limit = RG_TS_ITER_LIMIT;
  int num_sms = 0;
  // host entry points: uploads and early downloads run on copy_stream, ordered by these events
  cudaStream_t copy_stream = nullptr;
  cudaStream_t copy_stream_out = nullptr;   // device-to-host copies that overlap later work
  std::vector<cudaEvent_t> stage_events;
  // profiling
  bool prof_on = false;
  struct ProfRec {
    std::string name;
    cudaEvent_t e0, e1;
    double bytes;
  };
  std::vector<ProfRec> prof_pending;
  std::vector<cudaEvent_t> prof_pool;
  std::vector<rg_kernel_stat> prof_stats;
};
