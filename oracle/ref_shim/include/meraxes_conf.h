/* The configure-time header of the reference (meraxes_conf.h.in), with the values of its
   default CMake options: N_HISTORY_SNAPS 17, no stochastic sources, no magnitudes.
   Test infrastructure for oracle/_ref only. */
#define N_HISTORY_SNAPS 17
#define USE_STOCHASTICITY 0
#define MERAXES_GITREF_STR "oracle-ref"
#define MERAXES_GITDIFF_STR ""
#define FEATURE_FLAG_CALC_MAGS 0
