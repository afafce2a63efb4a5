"""CPU oracle for the reionization grid step -- TEST INFRASTRUCTURE ONLY.

This module restates, in numpy, the reference's CPU algorithm for
``_find_HII_bubbles`` (src/core/find_HII_bubbles.c:27-710), its k-space
``filter`` (src/core/reionization.c:3373-3433) and the brightness temperature
``ComputeBrightnessTemperatureBox`` (src/core/BrightnessTemperature.c:24-124,
512-548, the Flag_IncludePecVelsFor21cm = 0 form).  It is used only by
``tests/``, by ``__graft_entry__.smoke()`` and by ``bench.py``'s CPU baseline
leg, as the checker.  The product never imports it.

Parity status: **parity unpinned**.  The reference cannot be compiled here (it
needs FFTW3f-MPI, GSL, HDF5, MPI and the empty ``mlog`` submodule) and its
tests hold no golden vector for this path (its regression tests summarise whole
Meraxes runs on a dataset that is not available).  This restatement is pinned
instead by known answers derived from the code: the radius-schedule counts,
the window's closed forms, analytic uniform-field cases and FFT round trips.

Two precisions:

* ``"fp32"`` -- the reference's own arithmetic: single-precision FFTs (scipy's
  pocketfft in float32 stands in for FFTW's float plans; the rounding differs,
  so comparisons are statistical), float storage, double per-cell logic where
  the C code promotes.
* ``"fp64"`` -- every FFT, window and clamp in double; this is the FP64 oracle
  that each GPU output's error is stated against (pocketfft in float64 stands in
  for an FP64 FFTW plan).
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np
import scipy.fft as sfft

# ---------------------------------------------------------------------------
# constants (src/meraxes.h:21-67, src/core/reionization.h:10-44)
GRAVITY = 6.672e-8
SOLAR_MASS = 1.989e33
PLANCK = 6.6262e-27
PROTONMASS = 1.6726e-24
HUBBLE = 3.2407789e-18
SEC_PER_YEAR = 3.155e7
SEC_PER_MEGAYEAR = 3.155e13
MPC = 3.086e24
TCMB = 2.728
T_RE = 1e4
REL_TOL = np.float32(1e-5)
ABS_TOL = np.float32(1e-8)
SIGMA_HI = 6.3e-18
L_FACTOR = 0.620350491
# The aliasing clamps of find_HII_bubbles.c:377,410 are float constants: fmaxf(x, -1 + REL_TOL)
# evaluates -1 + REL_TOL in float (-0.99998999), and fminf(x, 0.999) rounds 0.999 to float.  The
# FP64 form keeps these constants (they define the algorithm; 1 + delta at the floor is 1.00136e-5,
# not 1e-5) and evaluates everything else in double.
CLAMP_DELTAX = float(np.float32(-1) + REL_TOL)
CLAMP_XE = float(np.float32(0.999))


@dataclasses.dataclass
class Params:
    """The run_globals.params / physics fields the hot path reads."""
    ReionGridDim: int
    BoxSize: float                 # Mpc/h
    Hubble_h: float = 0.6751
    OmegaM: float = 0.3121
    OmegaK: float = 0.0
    OmegaLambda: float = 0.6879
    OmegaR: float = 0.0
    BaryonFrac: float = 0.15714
    wLambda: float = -1.0
    UnitLength_in_cm: float = 3.08568e24
    UnitMass_in_g: float = 1.989e43
    UnitVelocity_in_cm_per_s: float = 1.0e5
    ReionDeltaRFactor: float = 1.1
    ReionRBubbleMax: float = 20.34
    ReionRBubbleMaxRecomb: float = 33.9
    ReionRBubbleMin: float = 0.4068
    Flag_EvolvingReionRBubbleMax: int = 1
    ReionFilterType: int = 0
    ReionRtoMFilterType: int = 0
    ReionUVBFlag: int = 1
    ReionEfficiency: float = 1.0
    ReionNionPhotPerBary: float = 4000.0
    ReionGammaHaloBias: float = 2.0
    ReionAlphaUV: float = 2.0
    ReionAlphaUVBH: float = 2.0
    ReionSfrTimescale: float = 0.5
    Y_He: float = 0.24
    Flag_IncludeSpinTemp: int = 0
    Flag_IncludeRecombinations: int = 0
    Flag_BHFeedback: int = 0
    # ComputeTs (input/params/defaults.par)
    TsHeatingFilterType: int = 1
    TsNumFilterSteps: int = 40
    Flag_IncludeAGNXray: int = 0
    ReionMaxHeatingRedshift: float = 30.0
    NuXrayThreshold: float = 500.0
    NuXraySoftCut: float = 2000.0
    NuXrayMax: float = 10000.0
    SpecIndexXrayGal: float = 1.0
    Flag_TemperatureDependentRec: int = 1
    SpecIndexXrayAGNSoft: float = 2.2
    SpecIndexXrayAGNHard: float = 1.7
    UseMiniHalos: int = 0
    ReionEfficiencyIII: float = 1.0
    ReionNionPhotPerBaryIII: float = 4000.0


@dataclasses.dataclass
class Units:
    UnitTime_in_s: float
    Hubble: float       # internal units
    G: float
    RhoCrit: float


def run_units(p: Params) -> Units:
    """set_units() (src/core/init.c:203-225)."""
    ut = p.UnitLength_in_cm / p.UnitVelocity_in_cm_per_s
    g = GRAVITY / p.UnitLength_in_cm ** 3 * p.UnitMass_in_g * ut ** 2
    hub = HUBBLE * ut
    rho = 3 * hub * hub / (8 * math.pi * g)
    return Units(ut, hub, g, rho)


def hubble_time(p: Params, z: float) -> float:
    """1 / (Hubble * E(z)), src/core/virial_properties.c:6-20,79-96."""
    u = run_units(p)
    opz = 1.0 + z
    ez = math.sqrt(p.OmegaM * opz ** 3 + p.OmegaK * opz ** 2 + p.OmegaLambda)
    return 1.0 / (u.Hubble * ez)


def dtdz(p: Params, z: float) -> float:
    """src/core/XRayHeatingFunctions.c:426-440 (float argument as in the C)."""
    opz = float(np.float32(1) + np.float32(z))       # 1 + z is a float sum in the C
    oml, omm = p.OmegaLambda, p.OmegaM
    x = math.sqrt(oml / omm) * opz ** (-1.5)
    dxdz = math.sqrt(oml / omm) * opz ** (-2.5) * (-1.5)
    const1 = 2 * math.sqrt(1 + omm / oml) / (3.0 * HUBBLE * p.Hubble_h)
    numer = dxdz * (1 + x * (x * x + 1) ** -0.5)
    denom = x + math.sqrt(x * x + 1)
    return const1 * numer / denom


def rtom(p: Params, R: float) -> float:
    """RtoM(), src/core/find_HII_bubbles.c:27-46."""
    u = run_units(p)
    if p.ReionRtoMFilterType == 0:
        return (4.0 / 3.0) * math.pi * R ** 3 * (p.OmegaM * u.RhoCrit)
    if p.ReionRtoMFilterType == 1:
        return (2 * math.pi) ** 1.5 * p.OmegaM * u.RhoCrit * R ** 3
    raise ValueError("unrecognised ReionRtoMFilterType")


def cT_approx(z: float) -> np.float32:
    """src/core/XRayHeatingFunctions.c:566-569 (float arithmetic)."""
    return np.float32(0.58 - 0.006 * (float(np.float32(z)) - 10.0))


def radius_schedule(p: Params, z: float) -> list[tuple[float, bool]]:
    """The filter radii of the excursion-set loop, find_HII_bubbles.c:256-285,546."""
    box, n = p.BoxSize, p.ReionGridDim
    cell_len_factor = L_FACTOR
    if box / n < 1.0:                     # find_HII_bubbles.c:147-148
        cell_len_factor = 1.0
    if p.Flag_EvolvingReionRBubbleMax:
        rmax = 25.483241248322766 if z > 6.0 else 112.0 * ((1.0 + z) / 5.0) ** -4.4
    else:
        rmax = p.ReionRBubbleMaxRecomb if p.Flag_IncludeRecombinations else p.ReionRBubbleMax
    R = min(rmax, L_FACTOR * box)
    out = []
    last = False
    while not last:
        if (R / p.ReionDeltaRFactor <= cell_len_factor * box / n) or (R / p.ReionDeltaRFactor <= p.ReionRBubbleMin):
            last = True
            R = cell_len_factor * box / n
        out.append((R, last))
        R /= p.ReionDeltaRFactor
    return out


# ---------------------------------------------------------------------------
# FFT layer (FFTW semantics: unnormalised r2c / c2r on padded real grids)

def forward(real: np.ndarray, precision: str) -> np.ndarray:
    """r2c of an [N][N][N] grid, then the /N^3 normalisation (find_HII_bubbles.c:235-253)."""
    n = real.shape[0]
    n3 = float(n) ** 3
    if precision == "fp32":
        spec = sfft.rfftn(real.astype(np.float32), workers=-1)
        return (spec.astype(np.complex128) / n3).astype(np.complex64)
    spec = sfft.rfftn(real.astype(np.float64), workers=-1)
    return spec / n3


def inverse(spec: np.ndarray, n: int) -> np.ndarray:
    """Unnormalised c2r (FFTW's backward plan) in the precision of ``spec``."""
    return sfft.irfftn(spec, s=(n, n, n), norm="forward", workers=-1)


def kmag(n: int, box: float, precision: str) -> np.ndarray:
    """|k| on the Hermitian half grid, filter() index decode (reionization.c:3375-3400)."""
    if precision == "fp32":
        f = np.float32
        delta_k = f(2.0 * math.pi / float(f(box)))
        idx = np.arange(n)
        signed = np.where(idx > n // 2, idx - n, idx).astype(f)
        kx = signed * delta_k
        kz = np.arange(n // 2 + 1).astype(f) * delta_k
        k2 = (kx[:, None, None] * kx[:, None, None] + kx[None, :, None] * kx[None, :, None]) + kz[None, None, :] * kz[None, None, :]
        return np.sqrt(k2.astype(f))
    delta_k = 2.0 * math.pi / box
    idx = np.arange(n)
    signed = np.where(idx > n // 2, idx - n, idx).astype(np.float64)
    kx = signed * delta_k
    kz = np.arange(n // 2 + 1) * delta_k
    return np.sqrt(kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2)


def window(n: int, box: float, R: float, ftype: int, precision: str) -> np.ndarray:
    """The k-space window W(kR) of filter(), reionization.c:3404-3428."""
    if ftype not in (0, 1, 2):
        raise ValueError("ReionFilterType undefined")
    k = kmag(n, box, precision)
    if precision == "fp32":
        f = np.float32
        kR = (k * f(R)).astype(f)
        if ftype == 0:
            with np.errstate(divide="ignore", invalid="ignore"):
                w = f(3.0) * (np.sin(kR) / (kR * kR * kR) - np.cos(kR) / (kR * kR))
            return np.where(kR > f(1e-4), w, f(1.0)).astype(f)
        if ftype == 1:
            kRs = (kR.astype(np.float64) * 0.413566994).astype(f)
            return np.where(kRs > 1, f(0.0), f(1.0)).astype(f)
        kRg = (kR.astype(np.float64) * 0.643).astype(f)
        expo = (-(kRg.astype(np.float64) * kRg.astype(np.float64)) / 2.0).astype(f)
        return np.power(f(math.e), expo).astype(f)
    kR = k * R
    if ftype == 0:
        with np.errstate(divide="ignore", invalid="ignore"):
            w = 3.0 * (np.sin(kR) / kR ** 3 - np.cos(kR) / kR ** 2)
        return np.where(kR > 1e-4, w, 1.0)
    if ftype == 1:
        return np.where(kR * 0.413566994 > 1, 0.0, 1.0)
    kRg = kR * 0.643
    return np.exp(-kRg * kRg / 2.0)


# ---------------------------------------------------------------------------
# temperatures (find_HII_bubbles.c:48-84)

def fully_ionized_temperature(z_re: np.ndarray, z: float, delta: np.ndarray) -> np.ndarray:
    """ComputeFullyIoinizedTemperature(), vectorised; float in, float out."""
    f = np.float32
    z_re = z_re.astype(f)
    zf = f(z)
    delta = delta.astype(f)
    same = np.abs((zf - z_re).astype(np.float64)) < 1e-4
    delta_re = (delta.astype(np.float64) * (1.0 + float(zf)) / (1.0 + z_re.astype(np.float64))).astype(f)
    delta_re = np.where(delta_re <= -1, f(-1.0 + 1e-8), delta_re).astype(f)
    dcl = np.where(delta <= -1, f(-1.0 + 1e-8), delta).astype(f)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        res = ((1.0 + dcl.astype(np.float64)) / (1.0 + delta_re.astype(np.float64))) ** 1.1333
        res = res.astype(f).astype(np.float64)
        res = (res * ((1.0 + float(zf)) / (1.0 + z_re.astype(np.float64))) ** 3.4).astype(f).astype(np.float64)
        ex = np.exp(((((1.0 + float(zf)) / 7.1) ** 2.5 - ((1.0 + z_re.astype(np.float64)) / 7.1) ** 2.5)).astype(f))
        res = (res * ex.astype(np.float64)).astype(f).astype(np.float64)
    res = np.where(same, 1.0, res)
    res = (res * T_RE ** 1.7).astype(f).astype(np.float64)
    one_plus_delta = (f(1) + np.where(same, delta, dcl)).astype(f).astype(np.float64)
    res = (res + (1e4 * ((1.0 + float(zf)) / 4.0)) ** 1.7 * one_plus_delta).astype(f).astype(np.float64)
    return (res ** 0.5882).astype(f)


def partially_ionized_temperature(t_hi: np.ndarray, res_xh: np.ndarray) -> np.ndarray:
    """ComputePartiallyIoinizedTemperature(), vectorised."""
    f = np.float32
    t_hi = t_hi.astype(f)
    res_xh = res_xh.astype(f)
    # T_HI * res_xH is a float product in the C; T_RE * (1. - res_xH) is double
    mid = ((t_hi * res_xh).astype(f).astype(np.float64) + T_RE * (1.0 - res_xh.astype(np.float64))).astype(f)
    out = np.where(res_xh >= 1, t_hi, mid)
    return np.where(res_xh <= 0, f(T_RE), out).astype(f)


# ---------------------------------------------------------------------------

@dataclasses.dataclass
class HIIState:
    """Persistent per-cell state that lives across snapshots in reion_grids_t."""
    z_at_ionization: np.ndarray            # [N^3] float32, -1 = never
    J_21_at_ionization: np.ndarray         # [N^3] float32
    temp_kinetic_all_gas: np.ndarray       # [N^3] float32
    Gamma12: np.ndarray | None = None      # recombinations: [N^3] float32
    N_rec: np.ndarray | None = None        # recombinations: [N^3] float32 (real part of the padded grid)

    @staticmethod
    def fresh(n: int, rec: bool = False) -> "HIIState":
        """init_reion_grids() values (src/core/reionization.c:557-595,698)."""
        st = HIIState(np.full((n, n, n), -1.0, np.float32), np.zeros((n, n, n), np.float32),
                      np.zeros((n, n, n), np.float32))
        if rec:
            st.Gamma12 = np.zeros((n, n, n), np.float32)
            st.N_rec = np.zeros((n, n, n), np.float32)
        return st

    def copy(self) -> "HIIState":
        c = lambda a: None if a is None else a.copy()
        return HIIState(self.z_at_ionization.copy(), self.J_21_at_ionization.copy(),
                        self.temp_kinetic_all_gas.copy(), c(self.Gamma12), c(self.N_rec))


def hii_scalars_names() -> list[str]:
    return ["volume_weighted_global_xH", "volume_weighted_global_r_bubble",
            "volume_weighted_global_weighted_sfr", "volume_weighted_global_effective_bhar",
            "volume_weighted_global_temp_kinetic_all_gas", "mass_weighted_global_xH",
            "mass_weighted_global_r_bubble", "mass_weighted_global_temp_kinetic_all_gas"]


def find_hii_bubbles(p: Params, z: float, deltax: np.ndarray, stars: np.ndarray, weighted_sfr: np.ndarray,
                     state: HIIState, precision: str = "fp32", x_e_box: np.ndarray | None = None,
                     Tk_box: np.ndarray | None = None, effective_bhm: np.ndarray | None = None,
                     effective_bhar: np.ndarray | None = None, record_margins: bool = False,
                     radius_subset: int | None = None, with_dead_grids: bool = False, rec_tables=None,
                     prev_z: float | None = None, starsIII: np.ndarray | None = None,
                     weighted_sfrIII: np.ndarray | None = None, spectra_in: dict | None = None,
                     radius_indices=None, skip_final: bool = False):
    """Restatement of _find_HII_bubbles() (find_HII_bubbles.c:86-710), one rank.

    With ``Flag_IncludeRecombinations`` the state carries Gamma12 and N_rec, ``rec_tables`` is a
    ``rec_oracle.RecTables`` and ``prev_z`` the previous snapshot's redshift (``z`` at the first
    snapshot); N_rec and weighted_sfr (and effective_bhar) are filtered too, the barrier is
    tested against 1 + N_rec (:467-483), Gamma12, r_bubble (and J_21 for ReionUVBFlag 2) are
    recorded at each cell's first crossing (:488-508), and the closing pass updates N_rec and
    returns residual_xH, clumping_factor and t_resp in ``diag["rec"]`` (:612-644).

    With ``UseMiniHalos`` (a USE_MINI_HALOS build) the padded Pop III grids ``starsIII`` and
    ``weighted_sfrIII`` add f_coll_starsIII x f_coll_prefactorIII to the barrier, to J_21 and
    (with recombinations) to Gamma12 (:104-117,190-202,443-545), and weighted_sfrIII to the
    closing-pass averages.

    Inputs are padded float32 grids; ``state`` is updated in place.  Returns
    ``(xH, r_bubble, scalars, diag)`` where ``diag`` holds, when
    ``record_margins`` is set, the per-cell minimum over radii of the relative
    barrier margin ``|lhs/rhs - 1|`` and the index of the first crossing radius,
    and wall-clock times of the phases.  ``radius_subset = k`` runs only the first
    k radii and the last one (a bounded timing sample; the outputs are then not
    the reference's).  ``with_dead_grids`` also transforms weighted_sfr every
    radius as the reference does, although without recombinations nothing reads
    the result (used when timing the CPU baseline).

    Timing hooks for the CPU baseline (the outputs are then partial): ``spectra_in``
    reuses the forward spectra of an earlier call (``diag["spectra"]``) instead of
    transforming again, ``radius_indices`` runs only those radii of the schedule, and
    ``skip_final`` returns before the closing pass.
    """
    import time as _time
    t_start = _time.perf_counter()
    rec = bool(p.Flag_IncludeRecombinations)
    mini = bool(p.UseMiniHalos)
    if mini and (starsIII is None or weighted_sfrIII is None):
        raise ValueError("UseMiniHalos needs starsIII and weighted_sfrIII")
    if rec and (rec_tables is None or state.Gamma12 is None or state.N_rec is None):
        raise ValueError("recombinations need rec_tables and a state with Gamma12 and N_rec")
    n = p.ReionGridDim
    box = p.BoxSize
    u = run_units(p)
    f32 = np.float32
    pixel_volume = (box / n) ** 3
    sfr_timescale = p.ReionSfrTimescale * hubble_time(p, z)
    TK = f32(T_RECFAST_at(z))
    cT_ad = cT_approx(z)

    xH = np.ones((n, n, n), f32)
    r_bubble = np.zeros((n, n, n), f32)
    z_in = state.z_at_ionization
    J21 = state.J_21_at_ionization
    temp = state.temp_kinetic_all_gas

    dx_real = deltax[:, :, :n]
    grids = {"deltax": dx_real, "stars": stars[:, :, :n]}
    if p.Flag_IncludeSpinTemp:
        grids["x_e"] = x_e_box[:, :, :n]
    if p.Flag_BHFeedback:
        grids["bhm"] = effective_bhm[:, :, :n]
    if mini:
        grids["starsIII"] = starsIII[:, :, :n]
    if rec:
        grids["nrec"] = state.N_rec
        grids["wsfr"] = weighted_sfr[:, :, :n]
        if p.Flag_BHFeedback:
            grids["bhar"] = effective_bhar[:, :, :n]
        if mini:
            grids["wsfrIII"] = weighted_sfrIII[:, :, :n]
    if with_dead_grids:
        grids["wsfr"] = weighted_sfr[:, :, :n]
    if spectra_in is not None:
        spectra = spectra_in
    else:
        spectra = {k: forward(v, precision) for k, v in grids.items()}
    t_forward = _time.perf_counter() - t_start
    radius_times = []

    J_aux_common = None
    min_margin = np.full((n, n, n), np.inf) if record_margins else None
    first_cross = np.full((n, n, n), -1, np.int16) if record_margins else None

    sched = radius_schedule(p, z)
    for ir, (R, last) in enumerate(sched):
        if radius_subset is not None and ir >= radius_subset and not last:
            continue
        if radius_indices is not None and ir not in radius_indices:
            continue
        t_r0 = _time.perf_counter()
        filt = {}
        for k, s in spectra.items():
            if not last:
                w = window(n, box, float(f32(R)) if precision == "fp32" else R, p.ReionFilterType, precision)
                s = (s * w).astype(s.dtype)
            filt[k] = inverse(s, n)
        fd = filt["deltax"]
        if precision == "fp32":
            fd = np.maximum(fd, f32(-1) + REL_TOL).astype(f32)
            fs = np.maximum(filt["stars"], f32(0)).astype(f32)
            fs = np.where(fs < ABS_TOL, f32(0), fs)
        else:
            fd = np.maximum(fd, CLAMP_DELTAX)
            fs = np.maximum(filt["stars"], 0.0)
            fs = np.where(fs < float(ABS_TOL), 0.0, fs)
        if p.Flag_IncludeSpinTemp:
            fx = filt["x_e"]
            if precision == "fp32":
                fx = np.maximum(fx, f32(0)).astype(f32)
                fx = np.where(fx < ABS_TOL, f32(0), fx)
                fx = np.minimum(fx, f32(0.999)).astype(f32)
            else:
                fx = np.minimum(np.where(np.maximum(fx, 0.0) < float(ABS_TOL), 0.0, np.maximum(fx, 0.0)), CLAMP_XE)
            neutral = 1.0 - fx.astype(np.float64)
        else:
            neutral = np.ones((n, n, n))
        fb = None
        if p.Flag_BHFeedback:
            fb = filt["bhm"]
            fb = np.maximum(fb, 0).astype(fb.dtype)
            fb = np.where(fb < (ABS_TOL if precision == "fp32" else float(ABS_TOL)), 0, fb).astype(fb.dtype)

        def clamped(key):
            f = filt[key]
            f = np.maximum(f, 0).astype(f.dtype)
            return np.where(f < (ABS_TOL if precision == "fp32" else float(ABS_TOL)), 0, f).astype(f.dtype)

        M_mean = rtom(p, R)
        g_pref = ((1.0 + z) * (1.0 + z) * R * p.UnitLength_in_cm / pixel_volume * p.UnitLength_in_cm ** -3.0)
        g_pref *= (p.UnitMass_in_g / u.UnitTime_in_s) / PROTONMASS * p.ReionNionPhotPerBary
        J_aux = f32(g_pref * PLANCK * 1e21 / (4.0 * math.pi) * p.ReionGammaHaloBias / sfr_timescale * p.ReionAlphaUV)
        J_aux_bh = f32(g_pref * PLANCK * 1e21 / (4.0 * math.pi) * p.ReionGammaHaloBias / sfr_timescale * p.ReionAlphaUVBH)
        fcoll_pref = p.ReionEfficiency * (4.0 / 3.0) * math.pi / pixel_volume / M_mean * R ** 3
        G_pref_bh = g_pref * (SIGMA_HI * p.ReionAlphaUVBH / (p.ReionAlphaUVBH + 2.75) * 1e12)
        G_pref = g_pref * (SIGMA_HI * p.ReionAlphaUV / (p.ReionAlphaUV + 2.75) * 1e12)
        # Pop III (find_HII_bubbles.c:443-450)
        J_auxIII = f32(J_aux * f32(p.ReionNionPhotPerBaryIII / p.ReionNionPhotPerBary))
        G_prefIII = G_pref * p.ReionNionPhotPerBaryIII / p.ReionNionPhotPerBary
        fcoll_prefIII = fcoll_pref / p.ReionEfficiency * p.ReionEfficiencyIII

        dom = 1.0 + fd.astype(np.float64)
        fcs = fs.astype(np.float64) / dom
        fbh = fb.astype(np.float64) / dom if fb is not None else 0.0
        lhs = (fbh + fcs) * fcoll_pref
        lhs_II = lhs
        fsIII = clamped("starsIII") if mini else None
        if mini:
            lhs = lhs + fsIII.astype(np.float64) / dom * fcoll_prefIII
        recf = clamped("nrec").astype(np.float64) / dom if rec else 0.0
        rhs = neutral * (1.0 + recf)
        ion = lhs > rhs
        if rec:
            # first crossing of the snapshot (find_HII_bubbles.c:488-508)
            first = ion & (xH > REL_TOL)
            gam = (clamped("wsfr")[first].astype(f32) * f32(G_pref)).astype(f32)
            if mini:
                gam = (gam + (clamped("wsfrIII")[first].astype(f32) * f32(G_prefIII)).astype(f32)).astype(f32)
            if p.Flag_BHFeedback:
                gam = (gam + (clamped("bhar")[first].astype(f32) * f32(G_pref_bh)).astype(f32)).astype(f32)
            state.Gamma12[first] = gam
            r_bubble[first] = f32(R)
            if p.ReionUVBFlag == 2:
                jj = (fs[first].astype(f32) * J_aux).astype(f32)
                if mini:
                    jj = (jj + (fsIII[first].astype(f32) * J_auxIII).astype(f32)).astype(f32)
                if fb is not None:
                    jj = (jj + (fb[first].astype(f32) * J_aux_bh).astype(f32)).astype(f32)
                J21[first] = jj
        if record_margins:
            m = np.abs(lhs / rhs - 1.0)
            np.minimum(min_margin, m, out=min_margin)
            newc = ion & (first_cross < 0)
            first_cross[newc] = ir
        xH[ion] = 0
        partial = (~ion) & last & (xH > REL_TOL)
        if np.any(partial):
            if p.Flag_IncludeSpinTemp:
                t_hi = Tk_box[partial]
            else:
                t_hi = (float(TK) * (1.0 + (cT_ad * dx_real[partial]).astype(f32).astype(np.float64))).astype(f32)
            temp[partial] = partially_ionized_temperature(t_hi, xH[partial])
            v = (neutral[partial] - lhs_II[partial]).astype(f32)
            if mini:
                v = (v - (fsIII[partial].astype(np.float64) / dom[partial] * fcoll_prefIII).astype(f32)).astype(f32)
            xH[partial] = np.clip(v, 0, 1)
        new = (xH < REL_TOL) & (z_in < 0)
        z_in[new] = f32(z)
        if p.ReionUVBFlag == 1:
            jj = (fs[new].astype(f32) * J_aux).astype(f32)
            if mini:
                jj = (jj + (fsIII[new].astype(f32) * J_auxIII).astype(f32)).astype(f32)
            if fb is not None:
                jj = (jj + (fb[new].astype(f32) * J_aux_bh).astype(f32)).astype(f32)
            J21[new] = jj

        radius_times.append(_time.perf_counter() - t_r0)

    if skip_final:
        diag = {"n_radii": len(sched), "spectra": spectra,
                "timing": {"forward": t_forward, "per_radius": float(np.mean(radius_times)) if radius_times else 0.0,
                           "final": 0.0}}
        return xH, r_bubble, {}, diag

    # final pass (find_HII_bubbles.c:577-702)
    t_f0 = _time.perf_counter()
    dxu = dx_real.astype(f32)
    dom = 1.0 + dxu.astype(np.float64)
    ionized = (z_in > 0) & (xH < REL_TOL)
    if np.any(ionized):
        temp[ionized] = fully_ionized_temperature(z_in[ionized], z, dxu[ionized])
    if p.Flag_IncludeSpinTemp:
        temp[:] = np.where(temp < Tk_box, Tk_box, temp)
    else:
        thistk = (float(TK) * (1.0 + (cT_ad * dxu).astype(f32).astype(np.float64))).astype(f32)
        temp[:] = np.where(temp < thistk, thistk, temp)
    n3 = float(n) ** 3
    s = {}
    s["volume_weighted_global_xH"] = xH.astype(np.float64).sum() / n3
    s["volume_weighted_global_r_bubble"] = r_bubble.astype(np.float64).sum() / n3
    wsfr = weighted_sfr[:, :, :n].astype(np.float64).sum() / n3
    s["volume_weighted_global_weighted_sfr"] = wsfr * p.UnitMass_in_g / u.UnitTime_in_s * SEC_PER_YEAR / SOLAR_MASS
    if p.Flag_BHFeedback and effective_bhar is not None:
        bh = effective_bhar[:, :, :n].astype(np.float64).sum() / n3
        s["volume_weighted_global_effective_bhar"] = bh * p.UnitMass_in_g / u.UnitTime_in_s * SEC_PER_YEAR / SOLAR_MASS
    else:
        s["volume_weighted_global_effective_bhar"] = 0.0
    s["volume_weighted_global_temp_kinetic_all_gas"] = temp.astype(np.float64).sum() / n3
    s["volume_weighted_global_weighted_sfrIII"] = 0.0
    if mini:
        w3 = weighted_sfrIII[:, :, :n].astype(np.float64).sum() / n3
        s["volume_weighted_global_weighted_sfrIII"] = w3 * p.UnitMass_in_g / u.UnitTime_in_s * SEC_PER_YEAR / SOLAR_MASS
    mw = dom.sum()
    s["mass_weighted_global_xH"] = (xH.astype(np.float64) * dom).sum() / mw
    s["mass_weighted_global_r_bubble"] = (r_bubble.astype(np.float64) * dom).sum() / mw
    s["mass_weighted_global_temp_kinetic_all_gas"] = (temp.astype(np.float64) * dom).sum() / mw
    rec_out = None
    if rec:
        # closing pass with recombinations (find_HII_bubbles.c:612-644)
        h = p.Hubble_h
        z_eff = (1.0 + z) * dom ** (1.0 / 3.0) - 1.0
        trec = temp.astype(np.float64) if p.Flag_TemperatureDependentRec else np.full(dom.shape, 1e4)
        gam = state.Gamma12.astype(np.float64) * h * h
        rate, rnh, cf = rec_tables.splined(z_eff, gam, trec)
        zstep = f32((z if prev_z is None else prev_z) - z)
        fabs_dtdz = f32(abs(dtdz(p, float(f32(z))) / h))
        inc = ((rate.astype(f32) * fabs_dtdz).astype(f32) * zstep).astype(f32)
        state.N_rec[:] = (state.N_rec.astype(np.float64) + inc.astype(np.float64) *
                          (1.0 - xH.astype(np.float64))).astype(f32)
        residual = rnh.astype(f32)
        clump = cf.astype(f32)
        tr = (gam * 1e-12 + rate).astype(f32)
        with np.errstate(divide="ignore"):
            t_resp = np.where(tr > 0, (1.0 / tr.astype(np.float64) / SEC_PER_MEGAYEAR).astype(f32), f32(1e30))
        rec_out = {"residual_xH": residual, "clumping_factor": clump, "t_resp": t_resp.astype(f32)}
        for name, a in (("Gamma12", state.Gamma12), ("N_rec", state.N_rec), ("residual_xH", residual),
                        ("clumping_factor", clump)):
            s["volume_weighted_global_" + name] = a.astype(np.float64).sum() / n3
            s["mass_weighted_global_" + name] = (a.astype(np.float64) * dom).sum() / mw
        s["volume_weighted_global_r_bubble"] = r_bubble.astype(np.float64).sum() / n3
        s["mass_weighted_global_r_bubble"] = (r_bubble.astype(np.float64) * dom).sum() / mw
    t_final = _time.perf_counter() - t_f0
    diag = {"min_margin": min_margin, "first_cross": first_cross, "n_radii": len(sched), "rec": rec_out,
            "timing": {"forward": t_forward, "per_radius": float(np.mean(radius_times)) if radius_times else 0.0,
                       "final": t_final}, "spectra": spectra}
    return xH, r_bubble, s, diag


# ---------------------------------------------------------------------------
# RECFAST temperature table (XRayHeatingFunctions.c:134-192) -- set by the caller

_RECFAST_T = None


def set_recfast(fn):
    """Install the T_RECFAST(z) evaluator (a natural cubic spline of recfast_LCDM.dat)."""
    global _RECFAST_T
    _RECFAST_T = fn


def T_RECFAST_at(z: float) -> float:
    if _RECFAST_T is None:
        raise RuntimeError("T_RECFAST table not loaded: call set_recfast()")
    return _RECFAST_T(float(np.float32(z)))


# ---------------------------------------------------------------------------

def delta_T(p: Params, z: float, xH: np.ndarray, deltax: np.ndarray, TS_box: np.ndarray | None = None):
    """ComputeBrightnessTemperatureBox(), velocity-free form (BrightnessTemperature.c:24-124,512-548)."""
    f = np.float32
    n = p.ReionGridDim
    redshift = f(z)
    h = f(p.Hubble_h)
    om = f(p.OmegaM)
    ob = f(om * f(p.BaryonFrac))
    const_factor = f(27.0 * (float(f(f(ob * h) * h)) / 0.023) *
                     math.sqrt((0.15 / float(om) / float(h) / float(h)) * (1.0 + float(redshift)) / 10.0))
    dx = deltax[:, :, :n].astype(np.float64)
    dT = (float(const_factor) * xH.astype(np.float64) * (1.0 + dx)).astype(f)
    if p.Flag_IncludeSpinTemp:
        t_rad = TCMB * (1.0 + float(redshift))
        fac = 1.0 - t_rad / TS_box.astype(np.float64)
        dT = (dT.astype(np.float64) * fac).astype(f)
    ave = dT.astype(np.float64).sum() / float(n) ** 3
    return dT, ave
