/*
 * rg_b200.h -- C ABI of the B200 reionization grid step.
 *
 * This library replaces the three grid-step entry points of Meraxes:
 *
 *   void find_HII_bubbles(int snapshot, timer_info* timer_total);   src/core/find_HII_bubbles.h:13
 *   void ComputeTs(int snapshot, timer_info* timer_total);          src/core/ComputeTs.h:15
 *   void ComputeBrightnessTemperatureBox(int snapshot);             src/core/BrightnessTemperature.h:10
 *
 * and the legacy device hooks they dispatch to under USE_CUDA:
 *
 *   void _find_HII_bubbles_gpu(const int snapshot, const bool flag_write_validation_output);  src/meraxes_gpu.h:53
 *   void init_CUDA(void);                                                                        src/meraxes_gpu.h:54
 *
 * The reference functions read everything from the global run_globals; these
 * take it explicitly: an rg_params struct with the run_globals.params fields the
 * step reads, the snapshot's redshift list, and an rg_grids struct of pointers
 * with the reion_grids_t layouts (src/meraxes.h:448-681):
 *
 *   real inputs   float[N][N][2(N/2+1)]  INDEX_PADDED  (src/core/misc_tools.c:249)
 *   real outputs  float[N][N][N]         INDEX_REAL    (src/core/misc_tools.c:252)
 *
 * All entry points return an int status (RG_OK = 0); nothing aborts or throws
 * across the ABI (the reference calls ABORT / throws C++ exceptions instead).
 * Calls on one context are not thread-safe; different contexts are independent.
 */
#ifndef RG_B200_H
#define RG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define RG_OK 0
#define RG_EINVAL 1        /* bad argument or parameter (checked before any launch) */
#define RG_ENOMEM 2        /* device or host allocation failed */
#define RG_ECUDA 3         /* a CUDA runtime call failed (rg_last_error() has the text) */
#define RG_EUNSUPPORTED 4  /* a feature flag the library does not implement */
#define RG_ETABLE 5        /* a 21cmFAST table file could not be read */
#define RG_ENODEV 6        /* no usable CUDA device */
#define RG_ETIMEDOUT 7     /* a bounded device-side wait gave up */

/* ---- parameters: the run_globals.params / .physics / .units fields the step reads ---- */
typedef struct rg_params {
  int ReionGridDim;                 /* N */
  double BoxSize;                   /* Mpc/h */
  double Hubble_h, OmegaM, OmegaK, OmegaLambda, OmegaR, BaryonFrac, wLambda;
  double UnitLength_in_cm, UnitMass_in_g, UnitVelocity_in_cm_per_s;
  /* find_HII_bubbles (src/core/find_HII_bubbles.c:90-285) */
  double ReionDeltaRFactor, ReionRBubbleMax, ReionRBubbleMaxRecomb, ReionRBubbleMin;
  int Flag_EvolvingReionRBubbleMax;
  int ReionFilterType;              /* 0 real-space top-hat, 1 sharp-k, 2 gaussian */
  int ReionRtoMFilterType;          /* 0 top-hat, 1 gaussian */
  int ReionUVBFlag;                 /* 0, 1 or 2 */
  double ReionEfficiency, ReionNionPhotPerBary, ReionGammaHaloBias, ReionAlphaUV, ReionAlphaUVBH;
  double ReionSfrTimescale, Y_He;
  int Flag_IncludeSpinTemp, Flag_IncludeRecombinations, Flag_BHFeedback;
  /* ComputeTs (src/core/ComputeTs.c:85-1554) */
  int TsHeatingFilterType, TsNumFilterSteps, Flag_IncludeAGNXray;
  double ReionMaxHeatingRedshift;
  double NuXrayThreshold, NuXraySoftCut, NuXrayMax;       /* eV */
  double SpecIndexXrayGal;
  /* ComputeBrightnessTemperatureBox */
  int Flag_IncludePecVelsFor21cm;
  /* directory holding recfast_LCDM.dat, kappa_*_table.dat, stellar_spectra.dat, x_int_tables/ */
  const char* TablesForXHeatingDir;
  /* merger-tree code of the velocity grid (meraxes.h:253-258): 0 VELOCIraptor, 1 gbpTrees,
     2 VELOCIraptor (augmented); sets the units of rg_grids.vel */
  int TreesID;
  /* recombinations (Flag_IncludeRecombinations): 1 = the MHR rates at the cell's gas
     temperature, 0 = at 10^4 K (find_HII_bubbles.c:613-619) */
  int Flag_TemperatureDependentRec;
  /* AGN X-ray channels of ComputeTs (Flag_IncludeAGNXray 1 soft + hard, 2 hard, 3 soft):
     nu^-alpha indices of the soft (NuXrayThreshold..NuXraySoftCut) and hard
     (NuXraySoftCut..NuXrayMax) bands (meraxes.h:187-189) */
  double SpecIndexXrayAGNSoft, SpecIndexXrayAGNHard;
  /* Pop III sources in find_HII_bubbles, as a USE_MINI_HALOS build of the reference has them
     (find_HII_bubbles.c:104-117,190-202,443-450,460-545): 1 = starsIII and weighted_sfrIII enter
     the barrier, J_21 and Gamma12 with their own efficiency and photons per baryon (the caller
     sets ReionNionPhotPerBaryIII from its Pop III IMF, PopIII.c:94, and ReionEfficiencyIII as
     set_ReionEfficiency does).  The Pop III channels of ComputeTs and delta_T are not built:
     rg_compute_Ts and rg_delta_T return RG_EUNSUPPORTED with UseMiniHalos. */
  int UseMiniHalos;
  double ReionEfficiencyIII, ReionNionPhotPerBaryIII;
} rg_params;

/* Fill *p with the values of input/params/defaults.par and the Genesis cosmology/units. */
int rg_params_default(rg_params* p, int grid_dim, double box_size);

/* ---- grids: reion_grids_t fields (device pointers unless an entry point says "host") ---- */
typedef struct rg_grids {
  /* padded real inputs [N][N][2(N/2+1)] */
  const float* deltax;
  const float* stars;
  const float* weighted_sfr;
  const float* effective_bhm;       /* Flag_BHFeedback */
  const float* effective_bhar;      /* Flag_BHFeedback */
  /* real [N]^3 outputs of find_HII_bubbles; z_at_ionization, J_21_at_ionization and
     temp_kinetic_all_gas persist across snapshots (initialise with rg_init_reion_grids) */
  float* xH;
  float* r_bubble;
  float* z_at_ionization;
  float* J_21_at_ionization;
  float* temp_kinetic_all_gas;
  /* spin temperature state: x_e_box_prev and x_e_box padded, Tk_box and TS_box real */
  float* x_e_box_prev;
  float* x_e_box;
  float* Tk_box;
  float* TS_box;
  /* ComputeTs sources, padded: sfr and xray_luminosity of this snapshot, and the
     histories [n_hist][N][N][2(N/2+1)], slot 0 = this snapshot (reionization.c:2093-2140) */
  const float* sfr;
  const float* xray_luminosity;
  const float* sfr_histories;
  const float* xray_luminosity_histories;
  int n_hist;
  /* brightness temperature output, real [N]^3 */
  float* delta_T;
  /* line-of-sight (z) velocity, padded, in the tree code's units; read by the brightness
     temperature when Flag_IncludePecVelsFor21cm > 0.  The reference converts this grid in
     place (BrightnessTemperature.c:173-196); the library leaves it unchanged. */
  const float* vel;
  /* inhomogeneous recombinations (Flag_IncludeRecombinations), reionization.c:1266-1292:
     N_rec padded and persistent (the cumulative recombinations per baryon); Gamma12 real and
     persistent (the ionising background at the cell's first crossing, 1e-12 s^-1 h^-2);
     residual_xH, clumping_factor and t_resp (Myr) real outputs */
  float* Gamma12;
  float* N_rec;
  float* residual_xH;
  float* clumping_factor;
  float* t_resp;
  /* AGN X-ray emissivity (Flag_IncludeAGNXray), padded, in the reference's units (1e10 L_sun per
     cell): this snapshot's BHXrayEmissivity_soft / _hard and their histories
     [n_hist][N][N][2(N/2+1)] (bh_xray_histories_soft / _hard), re-weighted per shell like the
     sfr histories (load_reion_bh_grids, reionization.c) */
  const float* bh_xray_soft;
  const float* bh_xray_hard;
  const float* bh_xray_histories_soft;
  const float* bh_xray_histories_hard;
  /* Pop III stellar mass and escape-weighted SFR (UseMiniHalos), padded */
  const float* starsIII;
  const float* weighted_sfrIII;
} rg_grids;

/* The snapshot being processed: run_globals.ZZ[] and the snapshot index into it. */
typedef struct rg_snapshot {
  int snapshot;
  int n_snapshots;
  const double* ZZ;                 /* host array, ZZ[0..n_snapshots) descending redshifts */
  double* stored_fcoll;             /* host array [n_snapshots]; rg_compute_Ts reads [snapshot - 1]
                                       and writes [snapshot] (ComputeTs.c:662) */
} rg_snapshot;

/* Global averages the reference stores into reion_grids_t (src/meraxes.h:628-675). */
typedef struct rg_hii_scalars {
  double volume_weighted_global_xH;
  double volume_weighted_global_r_bubble;
  double volume_weighted_global_weighted_sfr;
  double volume_weighted_global_effective_bhar;
  double volume_weighted_global_temp_kinetic_all_gas;
  double mass_weighted_global_xH;
  double mass_weighted_global_r_bubble;
  double mass_weighted_global_temp_kinetic_all_gas;
  int n_radii;                      /* filter radii processed */
  /* Flag_IncludeRecombinations only (0 otherwise) */
  double volume_weighted_global_Gamma12, volume_weighted_global_N_rec;
  double volume_weighted_global_residual_xH, volume_weighted_global_clumping_factor;
  double mass_weighted_global_Gamma12, mass_weighted_global_N_rec;
  double mass_weighted_global_residual_xH, mass_weighted_global_clumping_factor;
  double volume_weighted_global_weighted_sfrIII;   /* UseMiniHalos only (0 otherwise) */
} rg_hii_scalars;

typedef struct rg_ts_scalars {
  double volume_ave_J_alpha, volume_ave_xalpha, volume_ave_Xheat, volume_ave_Xion;
  double volume_ave_TS, volume_ave_TK, volume_ave_xe;
  double collapse_fraction, x_e_ave;      /* the stored_fcoll[snapshot] and <x_e> of this step */
  int homogeneous;                        /* 1 when zp >= ReionMaxHeatingRedshift */
  double volume_ave_Xheat_AGN_soft, volume_ave_Xheat_AGN_hard;   /* Flag_IncludeAGNXray (0 otherwise) */
} rg_ts_scalars;

typedef struct rg_context rg_context;

/* Execution modes (rg_set_mode). RG_MODE_FUSED is the default. */
#define RG_MODE_FUSED 0   /* dead-grid elimination, radius batching, graph replay */
#define RG_MODE_PLAIN 1   /* one 3-D FFT chain per grid per radius, every reference grid */

/* ---- lifetime; replaces init_CUDA() (src/core/meraxes_gpu.cu:127-194) ---- */
int rg_create(int device, int grid_dim, rg_context** out);
int rg_destroy(rg_context* ctx);
int rg_set_mode(rg_context* ctx, int mode);
/* Radii per batch of the fused mode's x/y and z passes: 0 = the default, 8; larger values are
   cut to 16 (the tuner in autotune.py picks one per workload shape). */
int rg_set_radius_batch(rg_context* ctx, int radii_per_batch);
/* cudaStream_t to launch on (NULL = the context's own stream). */
int rg_set_stream(rg_context* ctx, void* stream);
const char* rg_last_error(const rg_context* ctx);
const char* rg_status_string(int status);

/* Allocate every device grid a step with these flags needs, owned by ctx. */
int rg_alloc_grids(rg_context* ctx, const rg_params* p, int n_hist, rg_grids* out);
/* init_reion_grids() (src/core/reionization.c:504-716) for the device grids. */
int rg_init_reion_grids(rg_context* ctx, const rg_params* p, const rg_grids* g);

/* The MHR00 recombination tables of init_MHR() (src/core/recombinations.c:208-373), which a
   run with Flag_IncludeRecombinations must hand over once before its first find_HII_bubbles:
   lnGamma[n_gamma] (the knots, ln Gamma12), and RR (ln of the recombination rate), CF (the
   clumping factor) and RNH (ln of the residual neutral fraction), each [n_z][n_t][n_gamma]
   as Meraxes holds RR_table / CF_table / RNH_table (recombinations.h:17-34: 200 redshifts
   0, 0.2, ...; 100 temperatures log10 T = 2, 2.03, ...; 150 values of ln Gamma12).  The
   natural cubic splines of splined_recombination() (recombinations.c:35-84) are set up here,
   in FP64, and kept on the device; the host arrays may be freed on return. */
int rg_set_recombination_tables(rg_context* ctx, const double* lnGamma, int n_z, int n_t, int n_gamma,
                                const double* RR, const double* CF, const double* RNH);

/* ---- the grid step (device pointers, asynchronous on the context stream; scalars
        are written before return, so these synchronise the stream once) ---- */

/* _find_HII_bubbles (src/core/find_HII_bubbles.c:86-710).  With Flag_IncludeRecombinations
   it also filters N_rec and weighted_sfr (and effective_bhar), tests the barrier against
   1 + N_rec, records Gamma12, r_bubble (and J_21 for ReionUVBFlag 2) at each cell's first
   crossing, and updates N_rec, residual_xH, clumping_factor and t_resp in the closing pass
   (:226-230,467-508,613-644); rg_set_recombination_tables must have been called. */
int rg_find_HII_bubbles(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g,
                        rg_hii_scalars* out);

/* find_HII_bubbles for n_units independent snapshots of one ReionGridDim on device grids, in one
   call (arrays p[n_units], s[n_units], g[n_units], out[n_units]): the forward transforms of all
   their grids and, for every batch of radii, the windowed inverse x/y passes of all of them run
   as shared launches; the z passes (the barrier test) run per snapshot; the host synchronises
   once.  Each unit gets exactly what rg_find_HII_bubbles gives it.  The units must share
   ReionGridDim (= the context's), BoxSize, ReionFilterType, the feature flags and the radius
   schedule (RG_EINVAL otherwise).  With recombinations, Pop III sources or RG_MODE_PLAIN the
   units run one after another.  Device memory grows with the units: n_units x (live grids) x
   (radius batch + 1) spectra of (N/2+1) N^2 complex values.  No counterpart in the reference,
   which runs one snapshot per call (find_HII_bubbles.c:713-747). */
int rg_find_HII_bubbles_batch(rg_context* ctx, int n_units, const rg_params* p, const rg_snapshot* s,
                              const rg_grids* g, rg_hii_scalars* out);
/* _ComputeTs (src/core/ComputeTs.c:85-1554). */
int rg_compute_Ts(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g,
                  rg_ts_scalars* out);
/* ComputeBrightnessTemperatureBox (src/core/BrightnessTemperature.c:24-549); writes *volume_ave_Tb.
   With Flag_IncludeSpinTemp and Flag_IncludePecVelsFor21cm 1-3 it also applies the velocity
   gradient (:198-305, reionization.c:3435-3450) and, for 3, the line-of-sight redshift-space
   re-binning (:307-509); g->vel is then required. */
int rg_delta_T(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* g,
               double* volume_ave_Tb);

/* Host-buffer forms: g holds HOST pointers (the reion_grids_t arrays as Meraxes keeps
   them); inputs are copied to the context's device grids, the step runs, outputs are
   copied back.  These are what the USE_B200 shims of find_HII_bubbles(), ComputeTs()
   and ComputeBrightnessTemperatureBox() call. */
int rg_find_HII_bubbles_host(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* host,
                             rg_hii_scalars* out);
int rg_compute_Ts_host(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* host,
                       rg_ts_scalars* out);
int rg_delta_T_host(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* host,
                    double* volume_ave_Tb);

/* The snapshot's reionization block (src/core/dracarys.c:383-391: call_ComputeTs when
   Flag_IncludeSpinTemp, call_find_HII_bubbles, ComputeBrightnessTemperatureBox when
   host->delta_T is non-null) in one call on HOST arrays, with the host grids of the three
   _host entry points.  Each input is copied in once, in the order the steps read it, and
   overlaps the work before its first reader; the grids passed from one step to the next stay on
   the device; outputs are copied back as soon as they are final.  Outputs and scalars are those
   of the three calls made one after another. */
int rg_reion_step_host(rg_context* ctx, const rg_params* p, const rg_snapshot* s, const rg_grids* host,
                       rg_ts_scalars* ts, rg_hii_scalars* hii, double* volume_ave_Tb);

/* ---- callers next to the step ---- */

/* Number of k bins of the 21-cm power spectrum (PS_Length): Initialise_PowerSpectrum
   (src/core/ComputePowerSpectrum.c:18-42).  Needs ReionGridDim, BoxSize and Hubble_h. */
int rg_power_spectrum_length(const rg_params* p, int* n_bins);
/* Compute_PS (src/core/ComputePowerSpectrum.c:44-255) of the device grid delta_T (REAL layout,
   N^3 floats): fills PS_k, PS_data and PS_error (HOST arrays of at least max_bins floats) and
   *n_bins; an empty bin gives NaN there as in the reference.  Mini-halo (delta_TII) channels
   are not built. */
int rg_power_spectrum(rg_context* ctx, const rg_params* p, const float* d_delta_T, int max_bins, float* PS_k,
                      float* PS_data, float* PS_error, int* n_bins);
/* The same from a HOST delta_T (the reion_grids_t array). */
int rg_power_spectrum_host(rg_context* ctx, const rg_params* p, const float* h_delta_T, int max_bins,
                           float* PS_k, float* PS_data, float* PS_error, int* n_bins);
/* smooth_grid (src/core/read_grids.c:127-165): a padded grid of the context's dimension (the
   finer grid read from file) is transformed, divided by N^3, filtered with the real-space
   top-hat of radius (float)(box_size / reion_grid_dim / 2) and transformed back (device
   pointers; in place allowed). */
int rg_smooth_grid(rg_context* ctx, double box_size, int reion_grid_dim, const float* d_in_padded,
                   float* d_out_padded);

/* The nearest-grid-point deposit of construct_baryon_grids (src/core/reionization.c:2025-2592)
   for one rank holding the whole grid: galaxy g at d_pos[3g .. 3g+2] (box units, [0, box_size))
   adds d_values[p * n_gal + g] to grid p at the cell pos_to_ngp (src/core/misc_tools.c:207-217)
   gives; each grid is then clamped at zero, divided by divisors[p] (a host array, or null for
   none; the sfr grid's SFR timescale) and left in the padded layout.  The grids are overwritten
   (device pointers, n_prop <= 8).  Which galaxy property goes to which grid, the black-hole mass
   limit and the history shift stay with the caller.  A position below the box returns RG_EINVAL
   (the reference asserts). */
int rg_deposit_ngp(rg_context* ctx, double box_size, int n_gal, const float* d_pos, int n_prop,
                   const float* d_values, const double* divisors, float* const* d_grids);

/* The history bookkeeping of construct_baryon_grids (src/core/reionization.c:2105-2140 shifts
   the slots, :2470-2500 writes the snapshot's grid into slot 0) for the grids ComputeTs reads:
   with Flag_IncludeSpinTemp, for sfr, xray_luminosity and the AGN bands Flag_IncludeAGNXray
   uses, slot h + 1 <- slot h for h = n_hist - 2 .. 0, then slot 0 <- the current grid (device
   pointers of g, n_hist slots of the padded size each).  Called after the snapshot's grids are
   deposited, it leaves the histories as the reference's deposit does.  Stream-ordered on the
   context's stream; returns without a sync. */
int rg_push_histories(rg_context* ctx, const rg_params* p, const rg_grids* g);

/* ---- per-kernel timing: CUDA events on the launching stream around every launch ---- */
typedef struct rg_kernel_stat {
  char name[48];
  int launches;
  double ms_total;          /* summed event time */
  double alg_bytes_total;   /* algorithmic HBM bytes (minimum reads + writes) of those launches */
} rg_kernel_stat;
int rg_profile_enable(rg_context* ctx, int on);                  /* clears the counters */
int rg_profile_read(rg_context* ctx, rg_kernel_stat* out, int max, int* n);

/* ---- building blocks exposed for tests ---- */

/* Forward r2c of one padded grid, normalised by 1/N^3, into an internal spectrum slot;
   then unnormalised c2r of the slot (optionally filtered at radius R) into a padded grid.
   filter_type < 0 = no filter.  These mirror one forward plan + filter() + reverse plan. */
int rg_debug_filter_roundtrip(rg_context* ctx, const rg_params* p, const float* d_in_padded,
                              float* d_out_padded, double R, int filter_type);

/* Bounds of the device waits, for tests of their time-out paths (no counterpart in the
   reference, whose CPU loops have no waits).  xy_poll_limit: checks a Y item of the fused x/y
   pass makes for its plane's X items before it gives up (default 2^22, sleeping 64 ns between
   checks); xy_signal = 0 stops X items from signalling, so every Y wait runs out; the pass then
   completes with unordered planes and the call returns RG_ETIMEDOUT.  ts_iteration_limit:
   get_Ts fixed-point iterations per cell (default 10000); a cell that reaches it makes
   rg_compute_Ts return RG_ETIMEDOUT.  A negative (poll) or non-positive (iteration) value
   restores the default; larger values are cut to the defaults. */
int rg_debug_set_wait_limits(rg_context* ctx, int xy_poll_limit, int xy_signal, int ts_iteration_limit);

/* One c2c pass along y (the contiguous axis of the library's internal spectrum layout
   S[kz][x][y], complex64) over n_grids whole Hermitian spectra of ReionGridDim 256, in place:
   every line (kz, x) of (N/2+1) * N is transformed, forward (exp(-2 pi i n k / N), inverse = 0)
   or inverse (exp(+...), no 1/N), by one of two implementations:
     RG_DFT_FP32       the FP32 register-resident transform the step's passes use;
     RG_DFT_TC_BF16X3  the split-BF16 tensor-core form: 256 = 16 x 16, each radix-16 stage a
                       tcgen05 matrix product of hi/lo BF16 operands (three products) with FP32
                       accumulation in tensor memory, about 4.4e-6 relative error per pass.
   spec: device pointer, 16-byte aligned, n_grids * 129 * 256 * 256 complex64.  Both forms
   compute what the y stage of FFTW's 3-D transforms computes (find_HII_bubbles.c:351-370,
   ComputeTs.c:480-581); this entry point exists to compare them.  ReionGridDim other than 256
   returns RG_EUNSUPPORTED; a tensor-core wait that runs out returns RG_ETIMEDOUT. */
#define RG_DFT_FP32 0
#define RG_DFT_TC_BF16X3 1
int rg_dft_y_pass(rg_context* ctx, void* spec, int n_grids, int inverse, int impl);

/* Radius schedule of find_HII_bubbles: fills up to max_r radii, returns the count in *n. */
int rg_radius_schedule(const rg_params* p, double redshift, double* radii, int max_r, int* n);

/* Host-side coefficient engine of ComputeTs (no device work), for nS = TsNumFilterSteps
   shells of snapshot s with n_hist history slots:
     shells[6][nS] : R (Mpc), zpp_edge, zpp, dzpp, dt_dzpp, sum_lyn   (ComputeTs.c:339-478, 900-1011)
     freq[3][14][nS]: heat, ion, lya frequency integrals per x_e node (ComputeTs.c:761-808)
     coef[nS][1 + n_hist]: weight of source k in shell r's source grid, k = 0 this snapshot's
                    sfr / xray_luminosity, k = 1 + h history slot h (the re-weighting of
                    ComputeTs.c:366-478 as a linear combination)
   freq is computed only when freq != NULL. */
int rg_debug_ts_tables(const rg_params* p, const rg_snapshot* s, int n_hist, double x_e_ave,
                       double collapse_fraction, int max_shells, double* shells, double* freq, float* coef);

/* The AGN X-ray band tables of the same engine (Flag_IncludeAGNXray; host only):
     agn[2][3][14][nS]: band (soft, hard) x kind (heat, ion, lya) frequency integrals per x_e node
                        (ComputeTs.c:834-897), zero for a band that is off
     const_zp[3]       : const_zp_prefactor_GAL, _AGN_soft, _AGN_hard (ComputeTs.c:1014-1131) */
int rg_debug_ts_agn_tables(const rg_params* p, const rg_snapshot* s, int n_hist, double x_e_ave,
                           double collapse_fraction, int max_shells, double* agn, double* const_zp);

/* ---- allocation-free round trip (no counterpart in the reference) ----
   rg_debug_filter_roundtrip without a context and without any device allocation, for
   callers that cannot allocate: one that has given the device's memory to its own pool,
   or one for which cudaMalloc's implicit synchronisation is too costly.  Working memory is
   a static device array of RG_NOALLOC_SCRATCH_BYTES bytes per device, which holds grids up
   to RG_NOALLOC_MAX_GRID_DIM; larger ReionGridDim values return RG_EUNSUPPORTED with the
   reason in errbuf.  Runs on the current device, on `stream` (a cudaStream_t; NULL = the
   default stream), asynchronously.  The first call on a device looks up the array's address
   (once per device and CUDA context: after cudaDeviceReset the next call looks it up again);
   make the first call, and the first after a reset, before any stream capture begins.  Nothing in the scratch has
   to start at zero.  Two calls in flight at once on one device race on the scratch: order
   them (one stream, or the caller's own synchronisation).  errbuf (may be NULL) receives
   a message when the status is not RG_OK. */
#define RG_NOALLOC_MAX_GRID_DIM 64
#define RG_NOALLOC_SCRATCH_BYTES 2163200   /* 2 x (33 x 64 x 64) complex spectra + 64 twiddles */
int rg_filter_roundtrip_noalloc(const rg_params* p, const float* d_in_padded, float* d_out_padded, double R,
                                int filter_type, void* stream, char* errbuf, size_t errlen);

#ifdef __cplusplus
}
#endif

#endif /* RG_B200_H */
