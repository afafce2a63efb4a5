/* Driver of the reference's own reionization step -- TEST INFRASTRUCTURE ONLY (oracle/_ref).
 *
 * The reference's sources (src/core/find_HII_bubbles.c, ComputeTs.c, XRayHeatingFunctions.c,
 * BrightnessTemperature.c, reionization.c, recombinations.c, misc_tools.c, virial_properties.c,
 * utils.c) are compiled unmodified from the reference tree next to this file; this driver plays
 * the part of Meraxes' start-up for one rank:
 *   - parameters by name into run_globals.params (rg_ref_set_param / rg_ref_set_string);
 *   - set_units() (src/core/init.c:203-225), gsl_set_error_handler_off() (init.c:257), the
 *     snapshot redshifts, the stored_* averages (init.c:157-166), then the reference's own
 *     malloc_reionization_grids(), which assigns the slabs and runs init_reion_grids() (rg_ref_setup);
 *   - the grids of run_globals.reion_grids by name, for the caller to fill and read (rg_ref_grid);
 *   - the reference's _ComputeTs(), _find_HII_bubbles() and ComputeBrightnessTemperatureBox()
 *     (rg_ref_compute_Ts, rg_ref_find_HII_bubbles, rg_ref_delta_T), with ABORT() turned into
 *     a status code through myexit().
 * Only tests and the benchmark's reference arm load the library this builds.
 */
#include <math.h>
#include <setjmp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define _MAIN
#include "BrightnessTemperature.h"
#include "ComputeTs.h"
#include "XRayHeatingFunctions.h"
#include "find_HII_bubbles.h"
#include "gsl/gsl_errno.h"
#include "meraxes.h"
#include "reionization.h"

void _find_HII_bubbles(const int snapshot);
void _ComputeTs(int snapshot);

static jmp_buf g_abort_jmp;
static int g_in_call = 0;
static int g_abort_code = 0;

/* ABORT() of the reference ends in myexit() (src/core/misc_tools.c:15), which calls MPI_Abort:
   the one-rank MPI_Abort hands the code here, and a call in progress returns it as its status */
void rg_ref_on_abort(int code) {
  g_abort_code = code ? code : 1;
  if (g_in_call) longjmp(g_abort_jmp, 1);
  fprintf(stderr, "reference ABORT outside a driver call (%d)\n", code);
  abort();
}

/* ---- parameters by name ---- */

typedef struct {
  const char* name;
  void* addr;
  int is_int;
} param_entry;

#define P_D(field) {#field, &run_globals.params.field, 0}
#define P_I(field) {#field, &run_globals.params.field, 1}
#define PH_D(field) {#field, &run_globals.params.physics.field, 0}
#define PH_I(field) {#field, &run_globals.params.physics.field, 1}

static param_entry* params_table(size_t* n) {
  static param_entry t[] = {
      P_D(BoxSize), P_D(Hubble_h), P_D(BaryonFrac), P_D(OmegaM), P_D(OmegaK), P_D(OmegaR), P_D(OmegaLambda),
      P_D(wLambda), P_D(ReionDeltaRFactor), P_D(ReionSfrTimescale), P_I(ReionGridDim), P_I(ReionFilterType),
      P_I(TsHeatingFilterType), P_I(ReionRtoMFilterType), P_I(ReionUVBFlag), P_I(Flag_IncludeSpinTemp),
      P_I(Flag_IncludeLymanWerner), P_I(Flag_IncludeRecombinations), P_I(Flag_EvolvingReionRBubbleMax),
      P_I(Flag_TemperatureDependentRec), P_I(Flag_Compute21cmBrightTemp), P_I(Flag_IncludePecVelsFor21cm),
      P_I(TsNumFilterSteps), P_I(TsVelocityComponent), P_I(SnaplistLength), P_I(Flag_PatchyReion),
      PH_D(ReionEfficiency), PH_D(ReionEfficiencyIII), PH_D(ReionNionPhotPerBary), PH_D(ReionNionPhotPerBaryIII),
      PH_D(Y_He), PH_D(LXrayGal), PH_D(NuXrayThreshold), PH_D(SpecIndexXrayGal), PH_D(LXrayGalIII),
      PH_D(SpecIndexXrayIII), PH_D(NuXraySoftCut), PH_D(NuXrayMax), PH_I(Flag_IncludeAGNXray),
      PH_D(SpecIndexXrayAGNSoft), PH_D(SpecIndexXrayAGNHard), PH_D(SpecIndexUVAGNSoft), PH_D(SpecIndexUVAGNHard),
      PH_D(AGNLWEfficiency), PH_D(ReionMaxHeatingRedshift), PH_D(ReionGammaHaloBias), PH_D(ReionAlphaUV),
      PH_D(ReionAlphaUVBH), PH_D(ReionRBubbleMin), PH_D(ReionRBubbleMax), PH_D(ReionRBubbleMaxRecomb),
      PH_I(Flag_BHFeedback),
  };
  *n = sizeof(t) / sizeof(t[0]);
  return t;
}

int rg_ref_set_param(const char* name, double value) {
  size_t n;
  param_entry* t = params_table(&n);
  for (size_t i = 0; i < n; ++i)
    if (strcmp(t[i].name, name) == 0) {
      if (t[i].is_int)
        *(int*)t[i].addr = (int)value;
      else
        *(double*)t[i].addr = value;
      return 0;
    }
  return -1;
}

int rg_ref_set_string(const char* name, const char* value) {
  char* dst = NULL;
  if (strcmp(name, "TablesForXHeatingDir") == 0) dst = run_globals.params.TablesForXHeatingDir;
  if (strcmp(name, "RecombinationDir") == 0) dst = run_globals.params.RecombinationDir;
  if (!dst) return -1;
  strncpy(dst, value, STRLEN - 1);
  dst[STRLEN - 1] = '\0';
  return 0;
}

/* ---- start-up of one rank ---- */

static void set_units_ref(double length_cm, double mass_g, double velocity_cm_s) {
  run_units_t* u = &run_globals.units;
  u->UnitLength_in_cm = length_cm;
  u->UnitMass_in_g = mass_g;
  u->UnitVelocity_in_cm_per_s = velocity_cm_s;
  u->UnitTime_in_s = u->UnitLength_in_cm / u->UnitVelocity_in_cm_per_s;
  u->UnitTime_in_Megayears = u->UnitTime_in_s / SEC_PER_MEGAYEAR;
  run_globals.G = GRAVITY / pow(u->UnitLength_in_cm, 3) * u->UnitMass_in_g * pow(u->UnitTime_in_s, 2);
  run_globals.Csquare = pow(SPEED_OF_LIGHT / u->UnitVelocity_in_cm_per_s, 2);
  u->UnitDensity_in_cgs = u->UnitMass_in_g / pow(u->UnitLength_in_cm, 3);
  u->UnitPressure_in_cgs = u->UnitMass_in_g / u->UnitLength_in_cm / pow(u->UnitTime_in_s, 2);
  u->UnitCoolingRate_in_cgs = u->UnitPressure_in_cgs / u->UnitTime_in_s;
  u->UnitEnergy_in_cgs = u->UnitMass_in_g * pow(u->UnitLength_in_cm, 2) / pow(u->UnitTime_in_s, 2);
  run_globals.Hubble = HUBBLE * u->UnitTime_in_s;
  run_globals.RhoCrit = 3 * run_globals.Hubble * run_globals.Hubble / (8 * M_PI * run_globals.G);
}

static int g_setup = 0;

/* After the parameters: units, redshifts, history depth, then the reference's own allocation
   and initialisation of the grids.  n_hist is NstoreSnapshots_Heating (history slots). */
int rg_ref_setup(int n_snapshots, const double* ZZ, int n_hist, double length_cm, double mass_g,
                 double velocity_cm_s) {
  if (g_setup) return -2;
  gsl_set_error_handler_off();
  run_globals.mpi_comm = MPI_COMM_WORLD;
  run_globals.mpi_rank = 0;
  run_globals.mpi_size = 1;
  set_units_ref(length_cm, mass_g, velocity_cm_s);
  run_globals.params.SnaplistLength = n_snapshots;
  run_globals.ZZ = (double*)malloc(sizeof(double) * (size_t)n_snapshots);
  run_globals.AA = (double*)malloc(sizeof(double) * (size_t)n_snapshots);
  for (int i = 0; i < n_snapshots; ++i) {
    run_globals.ZZ[i] = ZZ[i];
    run_globals.AA[i] = 1.0 / (1.0 + ZZ[i]);
  }
  run_globals.NStoreSnapshots = 1;
  run_globals.NstoreSnapshots_Heating = n_hist > 0 ? n_hist : 1;
  run_globals.LTTime = (double*)calloc((size_t)n_snapshots, sizeof(double));
  run_globals.rhocrit = (double*)calloc((size_t)n_snapshots, sizeof(double));
  stored_fcoll = (double*)calloc((size_t)n_snapshots, sizeof(double));
  stored_fcollIII = (double*)calloc((size_t)n_snapshots, sizeof(double));
  stored_XrayEmissivity_hard = (double*)calloc((size_t)n_snapshots, sizeof(double));
  stored_XrayEmissivity_soft = (double*)calloc((size_t)n_snapshots, sizeof(double));
  stored_XrayEmissivity_HMXB = (double*)calloc((size_t)n_snapshots, sizeof(double));
  run_globals.params.FFTW3WisdomDir[0] = '\0';
  g_in_call = 1;
  if (setjmp(g_abort_jmp)) {
    g_in_call = 0;
    return g_abort_code;
  }
  malloc_reionization_grids(); /* assigns the slabs and initialises the grids itself */
#if USE_MINI_HALOS
  if (run_globals.params.Flag_IncludeSpinTemp) init_LW_diagnostics();
#endif
  g_in_call = 0;
  g_setup = 1;
  return 0;
}

double* rg_ref_stored_fcoll(void) { return stored_fcoll; }

/* ---- grids and scalars by name ---- */

#define G_ENTRY(field) {#field, (void**)&run_globals.reion_grids.field}

float* rg_ref_grid(const char* name) {
  static struct {
    const char* name;
    void** addr;
  } t[] = {
      G_ENTRY(deltax), G_ENTRY(stars), G_ENTRY(weighted_sfr), G_ENTRY(xH), G_ENTRY(r_bubble),
      G_ENTRY(z_at_ionization), G_ENTRY(J_21_at_ionization), G_ENTRY(temp_kinetic_all_gas), G_ENTRY(x_e_box),
      G_ENTRY(x_e_box_prev), G_ENTRY(Tk_box), G_ENTRY(TS_box), G_ENTRY(delta_T), G_ENTRY(sfr),
      G_ENTRY(xray_luminosity), G_ENTRY(sfr_histories), G_ENTRY(xray_luminosity_histories), G_ENTRY(N_rec),
      G_ENTRY(Gamma12), G_ENTRY(residual_xH), G_ENTRY(clumping_factor), G_ENTRY(t_resp), G_ENTRY(effective_bhm),
      G_ENTRY(effective_bhar), G_ENTRY(vel), G_ENTRY(BHXrayEmissivity_soft), G_ENTRY(BHXrayEmissivity_hard),
      G_ENTRY(bh_xray_histories_soft), G_ENTRY(bh_xray_histories_hard),
#if USE_MINI_HALOS
      G_ENTRY(starsIII), G_ENTRY(weighted_sfrIII), G_ENTRY(sfrIII), G_ENTRY(sfrIII_histories),
#endif
  };
  for (size_t i = 0; i < sizeof(t) / sizeof(t[0]); ++i)
    if (strcmp(t[i].name, name) == 0) return (float*)*t[i].addr;
  return NULL;
}

#define S_ENTRY(field) {#field, &run_globals.reion_grids.field}

int rg_ref_scalar(const char* name, double* out) {
  static struct {
    const char* name;
    double* addr;
  } t[] = {
      S_ENTRY(volume_weighted_global_xH), S_ENTRY(volume_weighted_global_r_bubble),
      S_ENTRY(volume_weighted_global_weighted_sfr), S_ENTRY(volume_weighted_global_effective_bhar),
      S_ENTRY(volume_weighted_global_temp_kinetic_all_gas), S_ENTRY(mass_weighted_global_xH),
      S_ENTRY(mass_weighted_global_r_bubble), S_ENTRY(mass_weighted_global_temp_kinetic_all_gas),
      S_ENTRY(volume_ave_J_alpha), S_ENTRY(volume_ave_xalpha), S_ENTRY(volume_ave_Xheat), S_ENTRY(volume_ave_Xion),
      S_ENTRY(volume_ave_TS), S_ENTRY(volume_ave_TK), S_ENTRY(volume_ave_xe), S_ENTRY(volume_ave_Tb),
      S_ENTRY(volume_ave_Xheat_AGN_soft), S_ENTRY(volume_ave_Xheat_AGN_hard),
#if USE_MINI_HALOS
      S_ENTRY(volume_weighted_global_weighted_sfrIII),
#endif
  };
  for (size_t i = 0; i < sizeof(t) / sizeof(t[0]); ++i)
    if (strcmp(t[i].name, name) == 0) {
      *out = *t[i].addr;
      return 0;
    }
  return -1;
}

/* ---- the step ---- */

#define GUARDED_CALL(expr)        \
  do {                            \
    if (!g_setup) return -2;      \
    g_in_call = 1;                \
    if (setjmp(g_abort_jmp)) {    \
      g_in_call = 0;              \
      return g_abort_code;        \
    }                             \
    expr;                         \
    g_in_call = 0;                \
    return 0;                     \
  } while (0)

int rg_ref_find_HII_bubbles(int snapshot) { GUARDED_CALL(_find_HII_bubbles(snapshot)); }
int rg_ref_compute_Ts(int snapshot) { GUARDED_CALL(_ComputeTs(snapshot)); }
int rg_ref_delta_T(int snapshot) { GUARDED_CALL(ComputeBrightnessTemperatureBox(snapshot)); }
