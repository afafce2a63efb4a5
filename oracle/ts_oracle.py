"""CPU oracle for the spin-temperature step -- TEST INFRASTRUCTURE ONLY.

Restates in numpy the reference's ``_ComputeTs`` (src/core/ComputeTs.c:85-1554)
with the AGN X-ray and mini-halo channels off, and the X-ray heating helpers it
calls (src/core/XRayHeatingFunctions.c): the shell radii and the SFR-history
re-weighting (:339-478), the frequency-integral tables (:760-898) built with
QAG / Gauss-Kronrod-61 and Brent's method, the Lyman-n sums with their kink
correction (:900-1011), the per-snapshot prefactors (:1014-1109), evolveInt and
the per-cell update (:1171-1407), get_Ts, and the homogeneous branch
(:252-331).  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg use it, as the checker; the product never imports it.

GSL is absent here: ``qag61`` restates QUADPACK's QAGE (the adaptive bisection
GSL's ``gsl_integration_qag`` performs) and ``brent`` restates Brent's 1973
zero finder as GSL's ``brent`` solver iterates it; the Gauss-Kronrod rule comes
from ``gk61.rule()``.

Parity status: **parity unpinned** (no reference build, no golden vectors for
this path); pinned by known answers: QAG on integrals with closed forms, Brent
on known roots, the Gauss-Kronrod rule's exactness, and the homogeneous branch
against the RECFAST tables.

The history combination is done in real space as the reference does it (in
place on float grids); the product forms the same combination in k-space.
Precision ``"fp32"`` reproduces the reference's float storage and float FFTs;
``"fp64"`` runs every FFT and window in double.
"""

from __future__ import annotations

import math
import os

import numpy as np

import reion_oracle as ro
import tables as tb
from gk61 import rule as gk61_rule

f32 = np.float32

# constants (src/meraxes.h, src/core/reionization.h:10-44, XRayHeatingFunctions.h)
BOLTZMANN = 1.3806e-16
SPEED_OF_LIGHT = 2.9979e10
PLANCK = ro.PLANCK
PROTONMASS = ro.PROTONMASS
SOLAR_MASS = ro.SOLAR_MASS
GRAVITY = ro.GRAVITY
HUBBLE = ro.HUBBLE
MPC = ro.MPC
TCMB = ro.TCMB
NU_over_EV = 1.60217646e-12 / PLANCK
NUIONIZATION = 13.60 * NU_over_EV
HeI_NUIONIZATION = 24.59 * NU_over_EV
HeII_NUIONIZATION = NUIONIZATION * 4
NU_LA = 10.2 * NU_over_EV
SIGMA_HI = 6.3e-18
TINY = 1e-30
FRACT_FLOAT_ERR = 1e-7
CLUMPING_FACTOR = 2.0
T21 = 0.0628
A10_HYPERFINE = 2.85e-15
MAX_TK = f32(5e4)
MIN_TK = f32(0.1)
R_XLy_MAX = 500.0
XRAY_LUMINOSITY_UNIT = 1.0e40
SOLAR_LUM = 3.826e33
NSPEC_MAX = 23
L_FACTOR = ro.L_FACTOR
DBL_EPSILON = np.finfo(np.float64).eps
DBL_MIN = np.finfo(np.float64).tiny

# kappa_10 of Zygelman (2005), table 2 column 4 (XRayHeatingFunctions.c:1738-1793)
_K10_T = [1.0, 2.0, 4.0, 6.0, 8.0, 10.0, 15.0, 20.0, 25.0, 30.0, 40.0, 50.0, 60.0, 70.0, 80.0, 90.0, 100.0,
          200.0, 300.0, 501.0, 701.0, 1000.0, 2000.0, 3000.0, 5000.0, 7000.0, 10000.0]
_K10_K = [1.38e-13, 1.43e-13, 2.71e-13, 6.60e-13, 1.47e-12, 2.88e-12, 9.10e-12, 1.78e-11, 2.73e-11, 3.67e-11,
          5.38e-11, 6.86e-11, 8.14e-11, 9.25e-11, 1.02e-10, 1.11e-10, 1.19e-10, 1.75e-10, 2.09e-10, 2.565e-10,
          2.91e-10, 3.31e-10, 4.27e-10, 4.97e-10, 6.03e-10, 6.87e-10, 7.87e-10]


# ---------------------------------------------------------------------------
# QAG with the 61-point Gauss-Kronrod rule (QUADPACK QAGE / gsl_integration_qag)

def _rescale_error(err, result_abs, result_asc):
    err = abs(err)
    if result_asc != 0 and err != 0:
        scale = (200 * err / result_asc) ** 1.5
        err = result_asc * scale if scale < 1 else result_asc
    if result_abs > DBL_MIN / (50 * DBL_EPSILON):
        min_err = 50 * DBL_EPSILON * result_abs
        if min_err > err:
            err = min_err
    return err


def _qk61(f, a, b):
    xgk, wgk, wg = gk61_rule()
    center = 0.5 * (a + b)
    half = 0.5 * (b - a)
    x = np.concatenate([center - half * xgk[:30], center + half * xgk[:30], [center]])
    fv = np.asarray(f(x), dtype=np.float64)
    f1, f2, fc = fv[:30], fv[30:60], fv[60]
    result_gauss = float(np.sum(wg * (f1 + f2)))
    result_kronrod = float(fc * wgk[30] + np.sum(wgk[:30] * (f1 + f2)))
    result_abs = float(abs(fc) * wgk[30] + np.sum(wgk[:30] * (np.abs(f1) + np.abs(f2))))
    mean = result_kronrod * 0.5
    result_asc = float(wgk[30] * abs(fc - mean) + np.sum(wgk[:30] * (np.abs(f1 - mean) + np.abs(f2 - mean))))
    err = (result_kronrod - result_gauss) * half
    result_kronrod *= half
    result_abs *= abs(half)
    result_asc *= abs(half)
    return result_kronrod, _rescale_error(err, result_abs, result_asc), result_abs, result_asc


def qag61(f, a, b, epsabs, epsrel, limit=1000):
    """Returns (status, result, abserr); status 0 on success.  ``f`` takes an array."""
    r0, e0, ra0, rc0 = _qk61(f, a, b)
    tolerance = max(epsabs, epsrel * abs(r0))
    round_off = 50 * DBL_EPSILON * ra0
    if e0 <= round_off and e0 > tolerance:
        return 2, r0, e0
    if (e0 <= tolerance and e0 != rc0) or e0 == 0.0:
        return 0, r0, e0
    if limit == 1:
        return 3, r0, e0
    iv = [[a, b, r0, e0]]
    area, errsum = r0, e0
    iteration, rt1, rt2, error_type = 1, 0, 0, 0
    while True:
        im = max(range(len(iv)), key=lambda i: iv[i][3])
        ca, cb, cr, ce = iv[im]
        a1, b1 = ca, 0.5 * (ca + cb)
        a2, b2 = b1, cb
        area1, error1, _, resasc1 = _qk61(f, a1, b1)
        area2, error2, _, resasc2 = _qk61(f, a2, b2)
        area12, error12 = area1 + area2, error1 + error2
        errsum += error12 - ce
        area += area12 - cr
        if resasc1 != error1 and resasc2 != error2:
            delta = cr - area12
            if abs(delta) <= 1.0e-5 * abs(area12) and error12 >= 0.99 * ce:
                rt1 += 1
            if iteration >= 10 and error12 > ce:
                rt2 += 1
        tolerance = max(epsabs, epsrel * abs(area))
        if errsum > tolerance:
            if rt1 >= 6 or rt2 >= 20:
                error_type = 2
            tmp = (1 + 100 * DBL_EPSILON) * (abs(a2) + 1000 * DBL_MIN)
            if abs(a1) <= tmp and abs(b2) <= tmp:
                error_type = 3
        iv[im] = [a1, b1, area1, error1]
        iv.append([a2, b2, area2, error2])
        iteration += 1
        if not (iteration < limit and not error_type and errsum > tolerance):
            break
    result = sum(x[2] for x in iv)
    if errsum <= tolerance:
        return 0, result, errsum
    return (error_type if error_type else 1), result, errsum


# ---------------------------------------------------------------------------
# Brent's zero finder (Brent 1973; the iteration of GSL's brent solver) with
# gsl_root_test_interval as the stopping rule (XRayHeatingFunctions.c:305-316)

def brent(fn, x_lower, x_upper, epsabs, epsrel, max_iter):
    a, b = x_lower, x_upper
    fa, fb = fn(a), fn(b)
    if (fa < 0 and fb < 0) or (fa > 0 and fb > 0):
        return b, 1
    c, fc, d, e = b, fb, b - a, b - a
    root, lo, hi = b, x_lower, x_upper
    for _ in range(max_iter):
        ac_equal = False
        if (fb < 0 and fc < 0) or (fb > 0 and fc > 0):
            ac_equal = True
            c, fc = a, fa
            d = e = b - a
        if abs(fc) < abs(fb):
            ac_equal = True
            a, b, c = b, c, b
            fa, fb, fc = fb, fc, fb
        tol = 0.5 * DBL_EPSILON * abs(b)
        m = 0.5 * (c - b)
        if fb == 0:
            root, lo, hi = b, b, b
        elif abs(m) <= tol:
            root = b
            lo, hi = (b, c) if b < c else (c, b)
        else:
            if abs(e) < tol or abs(fa) <= abs(fb):
                d = e = m
            else:
                s = fb / fa
                if ac_equal:
                    p, q = 2 * m * s, 1 - s
                else:
                    q, r = fa / fc, fb / fc
                    p = s * (2 * m * q * (q - r) - (b - a) * (r - 1))
                    q = (q - 1) * (r - 1) * (s - 1)
                if p > 0:
                    q = -q
                else:
                    p = -p
                if 2 * p < min(3 * m * q - abs(tol * q), abs(e * q)):
                    e, d = d, p / q
                else:
                    d = e = m
            a, fa = b, fb
            b += d if abs(d) > tol else (tol if m > 0 else -tol)
            fb = fn(b)
            root = b
            if (fb < 0 and fc < 0) or (fb > 0 and fc > 0):
                c = a
            lo, hi = (b, c) if b < c else (c, b)
        min_abs = min(abs(lo), abs(hi)) if ((lo > 0 and hi > 0) or (lo < 0 and hi < 0)) else 0.0
        if abs(hi - lo) < epsabs + epsrel * min_abs:
            return root, 0
    return root, 2


# ---------------------------------------------------------------------------
# cosmology (XRayHeatingFunctions.c:426-552, 1595-1637; reionization.h:15-32)

class Cosmo:
    def __init__(self, p: ro.Params):
        self.p = p
        h = p.Hubble_h
        rho_cgs = 3.0 * HUBBLE * HUBBLE * h * h / (8.0 * math.pi * GRAVITY)
        omb = p.BaryonFrac * p.OmegaM
        self.No = rho_cgs * omb * (1 - p.Y_He) / PROTONMASS
        self.He_No = rho_cgs * omb * p.Y_He / (4.0 * PROTONMASS)
        self.N_b0 = self.No + self.He_No
        self.f_H = self.No / (self.No + self.He_No)
        self.f_He = self.He_No / (self.No + self.He_No)

    def dtdz(self, z):
        """dtdz(float z): 1 + z is a float sum."""
        p = self.p
        opz = (f32(1) + np.asarray(z).astype(f32)).astype(np.float64)
        oml, omm = p.OmegaLambda, p.OmegaM
        x = math.sqrt(oml / omm) * opz ** (-1.5)
        dxdz = math.sqrt(oml / omm) * opz ** (-2.5) * (-1.5)
        const1 = 2 * math.sqrt(1 + omm / oml) / (3.0 * HUBBLE * p.Hubble_h)
        numer = dxdz * (1 + x * (x * x + 1) ** -0.5)
        denom = x + np.sqrt(x * x + 1)
        r = const1 * numer / denom
        return float(r) if np.ndim(r) == 0 else r

    def drdz(self, z):
        zf = float(f32(z))
        return (1.0 + zf) * SPEED_OF_LIGHT * self.dtdz(z)

    def hubble(self, z):
        p = self.p
        opz = (f32(1) + np.asarray(z).astype(f32)).astype(np.float64)
        r = HUBBLE * p.Hubble_h * np.sqrt(p.OmegaM * opz ** 3 + p.OmegaR * opz ** 4 + p.OmegaLambda)
        return float(r) if np.ndim(r) == 0 else r

    def dicke(self, z):
        p = self.p
        tiny = 1e-4
        omm, oml, omr = p.OmegaM, p.OmegaLambda, p.OmegaR
        if abs(omm - 1.0) < tiny:
            return 1.0 / (1.0 + z)
        if oml > -tiny and abs(oml + omm + omr - 1.0) < 0.01 and abs(p.wLambda + 1.0) < tiny:
            om_z = omm * (1 + z) ** 3 / (oml + omm * (1 + z) ** 3 + omr * (1 + z) ** 4)
            dz = 2.5 * om_z / (1.0 / 70.0 + om_z * (209 - om_z) / 140.0 + om_z ** (4.0 / 7.0))
            d0 = 2.5 * omm / (1.0 / 70.0 + omm * (209 - omm) / 140.0 + omm ** (4.0 / 7.0))
            return dz / (d0 * (1.0 + z))
        raise NotImplementedError("dicke: only the flat Lambda (and EdS) cases are restated")

    def ddicke_dz(self, z):
        dz = float(f32(1e-10))
        return (self.dicke(z + dz) - self.dicke(z)) / dz


def cross_sections(nu):
    """HI, HeI, HeII photo-ionisation cross sections (XRayHeatingFunctions.c:471-516), vectorised."""
    nu = np.asarray(nu, np.float64)
    with np.errstate(all="ignore"):
        nh = np.where(nu == NUIONIZATION, nu + TINY, nu)
        eps = np.sqrt(nh / NUIONIZATION - 1)
        hi = SIGMA_HI * (NUIONIZATION / nh) ** 4 * np.exp(4 - (4 * np.arctan(eps) / eps)) / (1 - np.exp(-2 * math.pi / eps))
        hi = np.where(nu < NUIONIZATION, 0.0, hi)
        x = nu / NU_over_EV / 13.61 - 0.4434
        y = np.sqrt(x * x + 2.136 ** 2)
        hei = 9.492e-16 * ((x - 1) * (x - 1) + 2.039 * 2.039) * y ** (0.5 * 3.188 - 5.5) * (1.0 + np.sqrt(y / 1.469)) ** -3.188
        hei = np.where(nu < HeI_NUIONIZATION, 0.0, hei)
        n2 = np.where(nu == HeII_NUIONIZATION, nu + TINY, nu)
        eps2 = np.sqrt(n2 / HeII_NUIONIZATION - 1)
        heii = (6.3e-18) / 4 * (HeII_NUIONIZATION / n2) ** 4 * np.exp(4 - (4 * np.arctan(eps2) / eps2)) / (1 - np.exp(-2 * math.pi / eps2))
        heii = np.where(nu < HeII_NUIONIZATION, 0.0, heii)
    return hi, hei, heii


# ---------------------------------------------------------------------------
# data tables and the electron interpolation (XRayHeatingFunctions.c:861-1276)

class TsTables:
    def __init__(self, tables_dir: str | None = None, nion_phot_per_bary: float = 4000.0):
        from scipy.interpolate import CubicSpline
        d = tables_dir or tb.default_tables_dir()
        self.recfast = tb.Recfast(d)
        self.k10_x = np.log(np.array(_K10_T))
        self.k10_y = np.log(np.array(_K10_K))
        self.k10 = CubicSpline(self.k10_x, self.k10_y, bc_type="natural")
        self.kel_x, self.kel_y = tb.read_kappa(d, "kappa_eH_table.dat", tb.KAPPA_10_elec_NPTS)
        self.kel = CubicSpline(self.kel_x, self.kel_y, bc_type="natural")
        self.kpH_x, self.kpH_y = tb.read_kappa(d, "kappa_pH_table.dat", tb.KAPPA_10_pH_NPTS)
        self.kpH = CubicSpline(self.kpH_x, self.kpH_y, bc_type="natural")
        # stellar spectra (spectral_emissivity flag 1, :670-702), indices 1..22
        sp = tb.read_stellar_spectra(d)
        self.spec_n = np.zeros(NSPEC_MAX, np.int64)
        self.spec_nu = np.zeros(NSPEC_MAX, f32)
        self.alpha2 = np.zeros(NSPEC_MAX, f32)
        self.N0_2 = np.zeros(NSPEC_MAX, f32)
        self.spec_n[1:] = sp[:, 0].astype(np.int64)
        self.N0_2[1:] = sp[:, 1]
        self.alpha2[1:] = sp[:, 2]
        for i in range(1, NSPEC_MAX):
            self.spec_nu[i] = f32(4.0 / 3.0 * (1.0 - 1.0 / float(self.spec_n[i]) ** 2.0))
        for i in range(1, NSPEC_MAX - 1):
            a = float(self.alpha2[i])
            n0_fac = float(self.spec_nu[i + 1]) ** (a + 1) - float(self.spec_nu[i]) ** (a + 1)
            self.N0_2[i] = f32(float(self.N0_2[i]) * ((a + 1) / n0_fac * nion_phot_per_bary))
        (self.E, self.fheat, self.n_lya, self.nion_hi, self.nion_hei, self.nion_heii) = tb.read_x_int_tables(d)
        self.X = tb.X_INT_XHII

    # kappa_10, kappa_10_elec, kappa_10_pH (:1728-1966)
    def kappa_10(self, TK):
        lt = np.log(TK)
        hi = np.log(math.exp(self.k10_y[-1]) * (TK / math.exp(self.k10_x[-1])) ** 0.381)
        mid = self.k10(np.clip(lt, self.k10_x[0], self.k10_x[-1]))
        return np.exp(np.where(lt < self.k10_x[0], self.k10_y[0], np.where(lt > self.k10_x[-1], hi, mid)))

    @staticmethod
    def _kappa_tab(spl, xs, ys, T):
        t = np.log(T)
        hi = ys[-1] + (ys[-1] - ys[-2]) / (xs[-1] - xs[-2]) * (t - xs[-1])
        mid = spl(np.clip(t, xs[0], xs[-1]))
        return np.exp(np.where(t < xs[0], ys[0], np.where(t > xs[-1], hi, mid)))

    def kappa_elec(self, T):
        return self._kappa_tab(self.kel, self.kel_x, self.kel_y, T)

    def kappa_pH(self, T):
        return self._kappa_tab(self.kpH, self.kpH_x, self.kpH_y, T)

    def interp(self, tab, En, xHII, below):
        """interp_fheat / interp_n_Lya / interp_nion_* (:970-1248) in float arithmetic, vectorised
        over En (float32 array); xHII a float32 scalar."""
        E, X = self.E, self.X
        En = np.asarray(En, f32).copy()
        top = En.astype(np.float64) > 0.999 * float(E[-1])
        En[top] = f32(float(E[-1]) * 0.999)
        low = En < E[0]
        x = f32(xHII)
        if float(x) > float(X[-1]) * 0.999:
            x = f32(float(X[-1]) * 0.999)
        elif x < X[0]:
            x = f32(1.001 * float(X[0]))
        Es = np.where(low, E[0], En)
        with np.errstate(divide="ignore"):
            n_low = np.where(Es.astype(np.float64) < 1008.88,
                             (np.log(Es.astype(np.float64) / 10.0) / 1.98026273e-2).astype(np.int64),
                             232 + (np.log(Es.astype(np.float64) / 1008.88) / 9.53101798e-2).astype(np.int64))
        n_low = np.clip(n_low, 0, len(E) - 2)
        n_high = n_low + 1
        m = len(X) - 1
        while x < X[m]:
            m -= 1
        lo, hi = tab[m], tab[m + 1]
        dE = (E[n_high] - E[n_low]).astype(f32)
        el = ((lo[n_high] - lo[n_low]) / dE).astype(f32)
        el = (el * (Es - E[n_low]).astype(f32)).astype(f32)
        el = (el + lo[n_low]).astype(f32)
        eh = ((hi[n_high] - hi[n_low]) / dE).astype(f32)
        eh = (eh * (Es - E[n_low]).astype(f32)).astype(f32)
        eh = (eh + hi[n_low]).astype(f32)
        r = ((eh - el) / f32(X[m + 1] - X[m])).astype(f32)
        r = (r * f32(x - X[m])).astype(f32)
        r = (r + el).astype(f32)
        return np.where(low, f32(below), r)

    def spectral_emissivity(self, nu_norm):
        """flag 0, Pop II (:707-727)."""
        for i in range(1, NSPEC_MAX - 1):
            if nu_norm >= float(self.spec_nu[i]) and nu_norm < float(self.spec_nu[i + 1]):
                return float(self.N0_2[i]) * nu_norm ** float(self.alpha2[i]) / NU_LA
        i = NSPEC_MAX - 1
        return float(self.N0_2[i]) * nu_norm ** float(self.alpha2[i]) / NU_LA


def frecycle(n: int) -> float:
    """Ly-n recycling fractions (XRayHeatingFunctions.c:572-640)."""
    t = [1, 1, 1, 0, 0.2609, 0.3078, 0.3259, 0.3353, 0.3410, 0.3448, 0.3476, 0.3496, 0.3512, 0.3524, 0.3535,
         0.3543, 0.3550, 0.3556, 0.3561, 0.3565, 0.3569, 0.3572, 0.3575, 0.3578, 0.3580, 0.3582, 0.3584, 0.3586,
         0.3587, 0.3589, 0.3590]
    return float(t[n]) if 0 <= n <= 30 else 0.0


def zmax(z: float, n: int) -> float:
    num = 1 - (n + 1) ** -2.0
    den = 1 - n ** -2.0
    return float(f32(float(f32(1) + f32(z)) * num / den - 1))


def nu_n(n: int) -> float:
    return (1.0 - n ** -2.0) / 0.75


# ---------------------------------------------------------------------------
# shells and the SFR-history re-weighting (ComputeTs.c:339-478), applied in real
# space to float grids the way the reference does it in place

class Shells:
    pass


def shells_and_sources(p: ro.Params, ZZ, snapshot: int, sfr, xray, sfr_hist, xray_hist, want_grids=True,
                       extra=()):
    """Returns (Shells, per-shell list of (sfr, xray, *extra) float32 grids or None).  ``extra`` holds
    (grid, histories) pairs re-weighted like the sfr grids: the AGN emissivity bands
    (load_reion_bh_grids).  ``Shells.max_slot`` is the highest history slot the shells read (-1:
    none); with ``want_grids=False`` the histories may be None (the schedule alone)."""
    cm = Cosmo(p)
    nS = p.TsNumFilterSteps
    box = p.BoxSize / p.Hubble_h
    n = p.ReionGridDim
    zp = float(ZZ[snapshot])
    prev_redshift = float(ZZ[snapshot]) if snapshot == 0 else float(ZZ[snapshot - 1])
    dzp = zp - prev_redshift
    dt_dzp = cm.dtdz(zp)
    R = L_FACTOR * box / float(f32(n))
    R_factor = (R_XLy_MAX / R) ** float(f32(1) / f32(nS))   # 1 / (float)nS is a float quotient
    sh = Shells()
    sh.max_slot = -1
    sh.R = np.zeros(nS)
    sh.zpp_edge = np.zeros(nS)
    scb = np.zeros(nS, np.int64)
    hists = [sfr_hist, xray_hist] + [e[1] for e in extra]
    cur = None if not want_grids else [a.astype(f32).copy() for a in [sfr, xray] + [e[0] for e in extra]]
    grids = []

    def load(idx, weight, new_load):
        nonlocal cur
        sh.max_slot = max(sh.max_slot, int(idx))
        if sfr_hist is None:          # schedule only: which history slots the shells read
            return
        if idx < 0 or idx >= len(sfr_hist):
            raise ValueError("history slot %d missing" % idx)
        if not want_grids:
            return
        w = f32(weight)
        if new_load:
            cur = [(h[idx].astype(f32) * w).astype(f32) for h in hists]
        else:
            cur = [(c + (h[idx].astype(f32) * w).astype(f32)).astype(f32) for c, h in zip(cur, hists)]

    def clear():
        nonlocal cur
        if want_grids:
            cur = [np.zeros_like(c) for c in cur]

    weight = 1.0
    scb[0] = 1
    for R_ct in range(nS):
        sh.R[R_ct] = R
        if R_ct == 0:
            prev_zpp, prev_R = zp, 0.0
        else:
            prev_zpp, prev_R = sh.zpp_edge[R_ct - 1], sh.R[R_ct - 1]
            scb[R_ct] = scb[R_ct - 1]
        sh.zpp_edge[R_ct] = prev_zpp - (R - prev_R) * MPC / cm.drdz(prev_zpp)
        zpp = (sh.zpp_edge[R_ct] + prev_zpp) * 0.5
        total_weight = (prev_zpp - sh.zpp_edge[R_ct]) * cm.dtdz(zpp)
        if snapshot - scb[R_ct] >= 0:
            if snapshot - scb[R_ct] == 0 and weight < 0:
                clear()
                scb[R_ct] += 1
            elif sh.zpp_edge[R_ct] > ZZ[snapshot - scb[R_ct]]:
                if R_ct == 0:
                    weight = dt_dzp * dzp / total_weight
                    if want_grids:
                        cur = [(c * weight).astype(f32) for c in cur]
                else:
                    if ZZ[snapshot - scb[R_ct]] > sh.zpp_edge[R_ct - 1]:
                        weight = -cm.dtdz(0.5 * (ZZ[snapshot - scb[R_ct]] + sh.zpp_edge[R_ct - 1]))
                        weight *= ZZ[snapshot - scb[R_ct]] - sh.zpp_edge[R_ct - 1]
                        weight /= total_weight
                        load(scb[R_ct] - 1, weight, 1)
                    else:
                        clear()
                while sh.zpp_edge[R_ct] > ZZ[snapshot - scb[R_ct]]:
                    if snapshot - scb[R_ct] == 0:
                        weight = -1
                        break
                    if sh.zpp_edge[R_ct] < ZZ[snapshot - scb[R_ct] - 1]:
                        zedge = prev_zpp if prev_zpp > ZZ[snapshot - scb[R_ct]] else ZZ[snapshot - scb[R_ct]]
                        weight = sh.zpp_edge[R_ct] - zedge
                        weight *= -cm.dtdz(0.5 * (sh.zpp_edge[R_ct] + zedge))
                    else:
                        weight = ZZ[snapshot - scb[R_ct] - 1] - ZZ[snapshot - scb[R_ct]]
                        weight *= -cm.dtdz(0.5 * (ZZ[snapshot - scb[R_ct] - 1] + ZZ[snapshot - scb[R_ct]]))
                    weight /= total_weight
                    load(scb[R_ct], weight, 0)
                    scb[R_ct] += 1
            else:
                if R_ct > 0 and weight != 1:
                    weight = 1
                    load(scb[R_ct] - 1, weight, 1)
        if want_grids:
            grids.append(tuple(cur))
        R *= R_factor
    sh.final_weight = weight
    sh.zpp = np.zeros(nS)
    sh.dzpp = np.zeros(nS)
    sh.dt_dzpp = np.zeros(nS)
    for ct in range(nS):
        if ct == 0:
            sh.zpp[ct] = (sh.zpp_edge[0] + zp) * 0.5
            sh.dzpp[ct] = zp - sh.zpp_edge[0]
        else:
            sh.zpp[ct] = (sh.zpp_edge[ct] + sh.zpp_edge[ct - 1]) * 0.5
            sh.dzpp[ct] = sh.zpp_edge[ct - 1] - sh.zpp_edge[ct]
        sh.dt_dzpp[ct] = cm.dtdz(sh.zpp[ct])
    return sh, (grids if want_grids else None)


# ---------------------------------------------------------------------------
# frequency tables and Lyman-n sums (ComputeTs.c:760-1011)

def freq_tables(p: ro.Params, T: TsTables, sh, zp, x_e_ave, collapse_fraction, ZZ, stored_fcoll, snapshot,
                agn_bands=()):
    """Galaxy X-ray tables heat, ion, lya [14][nS], the Lyman-n sums, and for each AGN band b in
    ``agn_bands`` (0 soft, 1 hard) its tables (ComputeTs.c:834-897) in the returned dict."""
    cm = Cosmo(p)
    nS = len(sh.R)
    ion_eff = p.ReionEfficiency
    nx = len(T.X)
    heat = np.zeros((nx, nS))
    ion = np.zeros((nx, nS))
    lya = np.zeros((nx, nS))

    def fcoll_at(z):
        if snapshot == 0:
            v = np.full_like(np.asarray(z, np.float64), collapse_fraction)
        else:
            v = stored_fcoll[snapshot - 1] + (z - ZZ[snapshot - 1]) * (collapse_fraction - stored_fcoll[snapshot - 1]) / (
                ZZ[snapshot] - ZZ[snapshot - 1])
        return np.where(v < 0.0, 0.0, v)

    def tauX(nu, x_e, zpv, zpp):
        nu_0 = nu / (1 + zpv)

        def integrand(zhat):
            drpropdz = SPEED_OF_LIGHT * cm.dtdz(zhat)
            nb = cm.N_b0 * (1 + zhat) ** 3
            nuhat = nu_0 * (1 + zhat)
            fc = fcoll_at(zhat)
            ff = np.where(fc < 1e-20, 1.0, 1 - (ion_eff * fc) / (1.0 - x_e_ave))
            ff = np.where(ff < 1e-4, 1e-4, ff)
            hi, hei, heii = cross_sections(nuhat)
            sig = cm.f_H * (1 - x_e) * hi + cm.f_He * (1 - x_e) * hei + cm.f_He * x_e * heii
            return drpropdz * nb * ff * sig

        st, res, _ = qag61(integrand, zpp, zpv, 0, 0.005, 1000)
        return 1e10 if st != 0 else res

    def nu_tau_one(zpv, zpp, x_e):
        if x_e > 0.9999:
            return -1.0
        if tauX(HeI_NUIONIZATION, x_e, zpv, zpp) < 1:
            return HeI_NUIONIZATION
        r, _ = brent(lambda nu: tauX(nu, x_e, zpv, zpp) - 1, HeI_NUIONIZATION, 1e6 * NU_over_EV, 0, 0.02, 100)
        return r

    thresh = p.NuXrayThreshold

    def integrate_over_nu(local_x_e, lo, hi, flag, alpha=p.SpecIndexXrayGal):
        if lo >= hi:
            return 0.0
        xf = f32(local_x_e)

        def fn(nu):
            hi_s, hei_s, heii_s = cross_sections(nu)
            pw = (nu / (thresh * NU_over_EV)) ** (-alpha - 1)
            en = [((nu - e0) / NU_over_EV).astype(f32) for e0 in (NUIONIZATION, HeI_NUIONIZATION, HeII_NUIONIZATION)]
            w = [cm.f_H * (1 - local_x_e) * hi_s, cm.f_He * (1 - local_x_e) * hei_s, cm.f_He * local_x_e * heii_s]
            s = 0.0
            for j, e0 in enumerate((NUIONIZATION, HeI_NUIONIZATION, HeII_NUIONIZATION)):
                if flag == 0:
                    s = s + T.interp(T.fheat, en[j], xf, 1.0).astype(np.float64) * PLANCK * (nu - e0) * w[j]
                elif flag == 1:
                    Fi = (T.interp(T.nion_hi, en[j], xf, 0.0).astype(np.float64) + T.interp(T.nion_hei, en[j], xf, 0.0)
                          + T.interp(T.nion_heii, en[j], xf, 0.0) + 1)
                    s = s + Fi * w[j]
                else:
                    s = s + T.interp(T.n_lya, en[j], xf, 0.0).astype(np.float64) * w[j]
            return s * pw

        st, res, _ = qag61(fn, lo, hi, 0, 0.01, 1000)
        if st != 0:
            return 0.0
        if flag == 2:
            return res * SPEED_OF_LIGHT / (4 * math.pi) / NU_LA / cm.hubble(zp)
        return res

    agn = {b: [np.zeros((nx, nS)) for _ in range(3)] for b in agn_bands}
    sum_lyn = np.zeros(nS)
    first_radii, first_zero = True, True
    weight = sh.final_weight
    n_pts_radii = 1000
    for R_ct in range(nS):
        prev_zpp = zp if R_ct == 0 else sh.zpp_edge[R_ct - 1]
        prev_R = 0.0 if R_ct == 0 else sh.R[R_ct - 1]
        zpp = (sh.zpp_edge[R_ct] + prev_zpp) * 0.5
        ntone = nu_tau_one(zp, zpp, x_e_ave)
        lower = max(ntone, thresh * NU_over_EV)
        upper = p.NuXrayMax * NU_over_EV
        for k in range(nx):
            xe = float(T.X[k])
            heat[k, R_ct] = integrate_over_nu(xe, lower, upper, 0)
            ion[k, R_ct] = integrate_over_nu(xe, lower, upper, 1)
            lya[k, R_ct] = integrate_over_nu(xe, lower, upper, 2)
        zf = (1.0 + zp) / (1.0 + zpp)
        for b in agn_bands:
            lo_b = max(ntone, (p.NuXraySoftCut if b else thresh) * NU_over_EV * zf)
            hi_b = (p.NuXrayMax if b else p.NuXraySoftCut) * NU_over_EV * zf
            a_b = p.SpecIndexXrayAGNHard if b else p.SpecIndexXrayAGNSoft
            for k in range(nx):
                for kind in range(3):
                    agn[b][kind][k, R_ct] = integrate_over_nu(float(T.X[k]), lo_b, hi_b, kind, a_b)
        for n_ct in range(NSPEC_MAX, 1, -1):
            if zpp > zmax(zp, n_ct):
                continue
            nuprime = nu_n(n_ct) * (1 + zpp) / (1.0 + zp)
            sum_lyn[R_ct] += frecycle(n_ct) * T.spectral_emissivity(nuprime)
        if R_ct > 2 and sum_lyn[R_ct] == 0.0 and sum_lyn[R_ct - 1] > 0.0 and first_radii:
            tmax = (prev_zpp - (sh.R[R_ct] - prev_R) * MPC / cm.drdz(prev_zpp) + prev_zpp) * 0.5
            tmin = (sh.zpp_edge[R_ct - 2] - (sh.R[R_ct - 1] - sh.R[R_ct - 2]) * MPC / cm.drdz(sh.zpp_edge[R_ct - 2])
                    + sh.zpp_edge[R_ct - 2]) * 0.5
            for ii in range(n_pts_radii):
                trial = tmin + (tmax - tmin) * float(f32(ii)) / (float(f32(n_pts_radii)) - 1.0)
                counter = sum(1 for n_ct in range(NSPEC_MAX, 1, -1) if not (trial > zmax(zp, n_ct)))
                if counter == 0 and first_zero:
                    first_zero = False
                    weight = float(f32(f32(ii) / f32(n_pts_radii)))
            sum_lyn[R_ct] = weight * sum_lyn[R_ct - 1]
            first_radii = False
    if agn_bands:
        return heat, ion, lya, sum_lyn, agn
    return heat, ion, lya, sum_lyn


def prefactors(p: ro.Params, zp: float):
    """ComputeTs.c:1014-1062."""
    cm = Cosmo(p)
    if abs(p.SpecIndexXrayGal - 1.0) < float(ro.REL_TOL):
        L = (p.NuXrayThreshold * NU_over_EV) * math.log(p.NuXraySoftCut / p.NuXrayThreshold)
        L = 1.0 / L
    else:
        L = (p.NuXraySoftCut * NU_over_EV) ** (1.0 - p.SpecIndexXrayGal) - (p.NuXrayThreshold * NU_over_EV) ** (
            1.0 - p.SpecIndexXrayGal)
        L = 1.0 / L
        L *= (p.NuXrayThreshold * NU_over_EV) ** (-p.SpecIndexXrayGal) * (1 - p.SpecIndexXrayGal)
    L *= 1.0 / PLANCK
    const_zp = L / (p.NuXrayThreshold * NU_over_EV) * SPEED_OF_LIGHT * (1 + zp) ** (p.SpecIndexXrayGal + 3)
    # AGN bands (ComputeTs.c:1049-1081,1116-1131): soft NuXrayThreshold..NuXraySoftCut, hard
    # NuXraySoftCut..NuXrayMax, both normalised at NuXrayThreshold
    const_agn = []
    for b in (0, 1):
        a = p.SpecIndexXrayAGNHard if b else p.SpecIndexXrayAGNSoft
        lo, hi = (p.NuXraySoftCut, p.NuXrayMax) if b else (p.NuXrayThreshold, p.NuXraySoftCut)
        if abs(a - 1.0) < float(ro.REL_TOL):
            La = 1.0 / ((p.NuXrayThreshold * NU_over_EV) * math.log(hi / lo))
        else:
            La = 1.0 / ((hi * NU_over_EV) ** (1.0 - a) - (lo * NU_over_EV) ** (1.0 - a))
            La *= (p.NuXrayThreshold * NU_over_EV) ** (-a) * (1.0 - a)
        La /= PLANCK
        const_agn.append(La / (p.NuXrayThreshold * NU_over_EV) * SPEED_OF_LIGHT * (1.0 + zp) ** (a + 3.0))
    return dict(growth=cm.dicke(zp), dgrowth=cm.ddicke_dz(zp), dt_dzp=cm.dtdz(zp), const_zp=const_zp,
                const_agn=const_agn)


# ---------------------------------------------------------------------------
# per-cell physics (XRayHeatingFunctions.c:1564-1690, 1973-2008)

def alpha_A(T):
    lt = np.log(T / 1.1604505e4)
    return np.exp(-28.6130338 - 0.72411256 * lt - 2.02604473e-2 * lt ** 2 - 2.38086188e-3 * lt ** 3
                  - 3.21260521e-4 * lt ** 4 - 1.42150291e-5 * lt ** 5 + 4.98910892e-6 * lt ** 6
                  + 5.75561414e-7 * lt ** 7 - 1.85676704e-8 * lt ** 8 - 3.07113524e-9 * lt ** 9)


def get_Ts(cm: Cosmo, T: TsTables, z, delta, TK, xe, Jalpha):
    """get_Ts(float z, float delta, float TK, float xe, float Jalpha) vectorised; returns (TS, xalpha) float32."""
    zd = float(f32(z))
    shape = np.shape(TK)
    delta = np.asarray(delta, f32).astype(np.float64).ravel()
    TKd = np.asarray(TK, f32).astype(np.float64).ravel()
    xe = np.asarray(xe, f32).astype(np.float64).ravel()
    Ja = np.asarray(Jalpha, f32).astype(np.float64).ravel()
    Trad = TCMB * (1.0 + zd)
    opz3 = (1.0 + zd) ** 3.0
    nH = (1.0 - xe) * cm.No * opz3 * (1.0 + delta)
    ne = xe * cm.N_b0 * opz3 * (1.0 + delta)
    npr = xe * cm.No * opz3 * (1.0 + delta)
    xc = (T21 / Trad * nH * T.kappa_10(TKd) / A10_HYPERFINE + T21 / Trad * ne * T.kappa_elec(TKd) / A10_HYPERFINE
          + T21 / Trad * npr * T.kappa_pH(TKd) / A10_HYPERFINE)
    TS = np.full_like(TKd, Trad)
    xa = np.zeros_like(TKd)
    wf = Ja > 1.0e-20
    tgp = 1.342881e-7 / cm.hubble(zd) * cm.No * (1 + zd) ** 3 * (1.0 + delta) * (1.0 - xe)
    told = np.zeros_like(TKd)
    active = wf.copy()
    for _ in range(10000):
        if not active.any():
            break
        idx = np.nonzero(active)[0]
        ts, tk = TS[idx], TKd[idx]
        told[idx] = ts
        xi = (1.0e-7 * tgp[idx] / tk / tk) ** (1.0 / 3.0)
        st = 1.0 - 0.0631789 / tk + 0.115995 / tk / tk - 0.401403 / ts / tk
        st = st + 0.336463 / ts / tk / tk
        st = st / (1.0 + 2.98394 * xi + 1.53583 * xi * xi + 3.85289 * xi * xi * xi)
        xat = 1.66e11 / (1.0 + zd) * st * Ja[idx]
        tce = 1.0 / tk + 0.405535 / tk * (1.0 / ts - 1.0 / tk)
        tce = 1.0 / tce
        tsinv = (1.0 / Trad + xat / tce + xc[idx] / tk) / (1.0 + xat + xc[idx])
        TS[idx] = 1.0 / tsinv
        xa[idx] = xat
        active[idx] = np.abs(TS[idx] - told[idx]) / TS[idx] > 1.0e-3
    coll = ~wf
    TS[coll] = 1.0 / ((1.0 / Trad + xc[coll] / TKd[coll]) / (1.0 + xc[coll]))
    TS = np.where(TS < 0.0, np.abs(TS), TS)
    return TS.astype(f32).reshape(shape), xa.astype(f32).reshape(shape)


def dT_comp(cm: Cosmo, z, TK, xe):
    Trad = TCMB * (1.0 + z)
    ans = (-1.51e-4) * (xe / (1.0 + xe + cm.f_He)) / (cm.hubble(z) / (HUBBLE * cm.p.Hubble_h)) / cm.p.Hubble_h * Trad ** 4.0 / (1.0 + z)
    return ans * (Trad - TK)


# ---------------------------------------------------------------------------
# the step

def compute_ts(p: ro.Params, T: TsTables, ZZ, snapshot: int, stored_fcoll, g: dict, precision: str = "fp64",
               tables_out: dict | None = None):
    """One _ComputeTs call.  ``g`` holds [N]^3 arrays: deltax, stars, x_e_box_prev, Tk_box, sfr,
    xray_luminosity (float32), and lists sfr_histories / xray_luminosity_histories; x_e_box_prev
    and Tk_box are updated in place, x_e_box and TS_box are set.  Returns the scalars."""
    n = p.ReionGridDim
    n3 = float(n) ** 3
    cm = Cosmo(p)
    zp = float(ZZ[snapshot])
    box = p.BoxSize / p.Hubble_h
    pv = (box / float(n)) ** 3
    deltax = g["deltax"].astype(f32)
    stars = g["stars"].astype(f32)
    R0 = L_FACTOR * box / float(f32(n))
    dom = 1.0 + deltax.astype(np.float64)
    cfc = stars.astype(np.float64) / (ro.rtom(p, R0) * p.Hubble_h * p.Hubble_h * dom) * (4.0 / 3.0) * math.pi * R0 ** 3.0 / pv
    collapse_fraction = float(np.sum(np.minimum(cfc, 1.0)) / n3)
    out = dict(collapse_fraction=collapse_fraction)
    if (zp - p.ReionMaxHeatingRedshift) >= -0.0001:
        xe0 = f32(T.recfast.xe(zp))
        TK0 = f32(T.recfast.T(zp))
        cT = ro.cT_approx(zp)
        tk = (float(TK0) * (1.0 + (cT * deltax).astype(f32).astype(np.float64))).astype(f32)
        ts, _ = get_Ts(cm, T, zp, deltax, tk, np.full_like(tk, xe0), np.zeros_like(tk))
        g["x_e_box_prev"][...] = xe0
        g["Tk_box"][...] = tk
        g["TS_box"] = ts
        g["x_e_box"] = g["x_e_box_prev"].copy()
        out.update(homogeneous=1, x_e_ave=0.0, volume_ave_TS=float(np.sum(ts.astype(np.float64)) / n3),
                   volume_ave_TK=float(np.sum(tk.astype(np.float64)) / n3), volume_ave_xe=float(xe0),
                   volume_ave_J_alpha=0.0, volume_ave_xalpha=0.0, volume_ave_Xheat=0.0, volume_ave_Xion=0.0)
        return out
    xprev = g["x_e_box_prev"].astype(f32)
    x_e_ave = float(np.sum(xprev.astype(np.float64)) / n3)
    out.update(homogeneous=0, x_e_ave=x_e_ave)
    # AGN X-ray bands in use (Flag_IncludeAGNXray 1 soft + hard, 2 hard, 3 soft)
    bands = [b for b, on in ((0, p.Flag_IncludeAGNXray in (1, 3)), (1, p.Flag_IncludeAGNXray in (1, 2))) if on]
    names = ("soft", "hard")
    extra = [(g["bh_xray_" + names[b]], g.get("bh_xray_histories_" + names[b], [])) for b in bands]
    sh, grids = shells_and_sources(p, ZZ, snapshot, g["sfr"], g["xray_luminosity"], g.get("sfr_histories", []),
                                   g.get("xray_luminosity_histories", []), extra=extra)
    nS = len(sh.R)
    no_light = not (collapse_fraction > 0.0)
    prevz = zp if snapshot == 0 else float(ZZ[snapshot - 1])
    dzp = zp - prevz
    pf = prefactors(p, zp)
    sums = [np.zeros(deltax.shape) for _ in range(4)]
    sums_agn = {b: [np.zeros(deltax.shape) for _ in range(3)] for b in bands}
    if not no_light:
        sf = stored_fcoll if stored_fcoll is not None else np.zeros(len(ZZ))
        ft = freq_tables(p, T, sh, zp, x_e_ave, collapse_fraction, ZZ, sf, snapshot, agn_bands=tuple(bands))
        heat, ion, lya, sum_lyn = ft[:4]
        agn_tabs = ft[4] if bands else {}
        if tables_out is not None:
            tables_out.update(heat=heat, ion=ion, lya=lya, sum_lyn=sum_lyn, shells=sh, agn=agn_tabs)
        xi = xe_interp_index(T, xprev)
        for r in range(nS):
            agn = [(b, grids[r][2 + j], agn_tabs[b], sums_agn[b]) for j, b in enumerate(bands)]
            shell_accumulate(p, sh, r, grids[r][0], grids[r][1], xi, (heat, ion, lya), sum_lyn, zp, sums, precision,
                             agn=agn)
        finish_sums(p, cm, pf, zp, deltax, sums, sums_agn)
    # the AGN heating terms of dT_K/dz (XRayHeatingFunctions.c:1519-1520), averaged
    xd = xprev.astype(np.float64)
    for b in (0, 1):
        v = 0.0
        if b in sums_agn and not no_light:
            v = float(np.sum(sums_agn[b][0] * pf["dt_dzp"] * 2.0 / 3.0 / BOLTZMANN / (1.0 + xd)) / n3)
        out["volume_ave_Xheat_AGN_" + names[b]] = v
    res = evolve_cells(p, cm, T, pf, zp, dzp, deltax, xprev, g["Tk_box"], sums)
    xn, tk, ts = res["x_e"], res["Tk"], res["TS"]
    g["x_e_box_prev"][...] = xn
    g["Tk_box"][...] = tk
    g["TS_box"] = ts
    g["x_e_box"] = xn.copy()
    out.update(volume_ave_J_alpha=float(np.sum(res["J_alpha"]) / n3),
               volume_ave_xalpha=float(np.sum(res["xalpha"].astype(np.float64)) / n3),
               volume_ave_Xheat=float(np.sum(res["dxheat_dzp"]) / n3), volume_ave_Xion=float(np.sum(res["dxion"]) / n3),
               volume_ave_TS=float(np.sum(ts.astype(np.float64)) / n3),
               volume_ave_TK=float(np.sum(tk.astype(np.float64)) / n3),
               volume_ave_xe=float(np.sum(xn.astype(np.float64)) / n3))
    out["_cells"] = dict(dxheat_dzp=res["dxheat_dzp"], dxion=res["dxion"], J_alpha=res["J_alpha"])
    return out


def xe_interp_index(T: TsTables, xprev):
    """Per-cell x_e interpolation node and clamped x_e (ComputeTs.c:1198-1209)."""
    X = T.X
    xh = np.asarray(xprev, f32).astype(np.float64)
    xh = np.where(xh > float(X[-1]) * 0.999, float(X[-1]) * 0.999, np.where(xh < float(X[0]), 1.001 * float(X[0]), xh))
    xhf = xh.astype(f32)
    m_lo = np.full(xh.shape, len(X) - 1)
    for m in range(len(X) - 1, -1, -1):
        m_lo = np.where(xhf < X[m], m - 1, m_lo)
    m_lo = np.clip(m_lo, 0, len(X) - 2)
    return dict(xh=xh, m_lo=m_lo, Xl=X[m_lo].astype(np.float64), Xh=X[m_lo + 1].astype(np.float64))


def shell_accumulate(p: ro.Params, sh, r: int, s_grid, x_grid, xi: dict, tabs, sum_lyn, zp: float, sums: list,
                     precision: str = "fp64", agn=()):
    """One shell R_ct: FFT, filter (R_ct > 0), inverse, clamp and unit conversion of the sfr and
    X-ray grids (ComputeTs.c:480-744), then its terms of the evolveInt sums
    (XRayHeatingFunctions.c:1379-1432) added to sums = [heat, ion, lya, star].  ``agn`` holds
    (band, grid, tables, band sums) for the AGN X-ray bands: the grid clamped at 0 and converted
    (ComputeTs.c:615-630), its terms (XRayHeatingFunctions.c:1420-1432) added to the band sums."""
    n = p.ReionGridDim
    box = p.BoxSize / p.Hubble_h
    pv = (box / float(n)) ** 3
    u = ro.run_units(p)
    prec = "fp32" if precision == "fp32" else "fp64"
    ss = ro.forward(s_grid, prec)
    xs = ro.forward(x_grid, prec)
    if r > 0:
        w = ro.window(n, p.BoxSize, float(f32(sh.R[r])), p.TsHeatingFilterType, prec)
        ss = ss * w
        xs = xs * w
    s_f = ro.inverse(ss, n)
    x_f = ro.inverse(xs, n)
    if precision == "fp32":
        s_f = s_f.astype(f32)
        x_f = x_f.astype(f32)
    s_f = np.maximum(s_f, 0.0)
    SFR = (s_f.astype(np.float64) / pv) * (p.UnitMass_in_g / u.UnitTime_in_s) * p.UnitLength_in_cm ** -3.0 / SOLAR_MASS
    XR = (x_f.astype(np.float64) / pv) * XRAY_LUMINOSITY_UNIT * p.UnitLength_in_cm ** -3.0
    m_lo, xh, Xl, Xh = xi["m_lo"], xi["xh"], xi["Xl"], xi["Xh"]

    def fi(tbl):
        lo = tbl[m_lo, r]
        hi = tbl[m_lo + 1, r]
        return (hi - lo) / (Xh - Xl) * (xh - Xl) + lo

    zpp, dzpp, dt_dzpp = sh.zpp[r], sh.dzpp[r], sh.dt_dzpp[r]
    integ = XR * (1 + zpp) ** (-p.SpecIndexXrayGal)
    for k in range(3):
        sums[k] += dt_dzpp * dzpp * integ * fi(tabs[k])
    sums[3] += SFR * float(f32(1) + f32(zp)) ** 2 * (1 + zpp) * sum_lyn[r] * dt_dzpp * dzpp
    for b, grid, tabs_b, sa in agn:
        sp = ro.forward(grid, prec)
        if r > 0:
            sp = sp * ro.window(n, p.BoxSize, float(f32(sh.R[r])), p.TsHeatingFilterType, prec)
        a_f = ro.inverse(sp, n)
        if precision == "fp32":
            a_f = a_f.astype(f32)
        a_f = np.maximum(a_f, 0.0)
        XA = a_f.astype(np.float64) * 1e10 * SOLAR_LUM / pv * p.UnitLength_in_cm ** -3.0
        ia = XA * (1 + zpp) ** (-(p.SpecIndexXrayAGNHard if b else p.SpecIndexXrayAGNSoft))
        for k in range(3):
            sa[k] += dt_dzpp * dzpp * ia * fi(tabs_b[k])


def finish_sums(p: ro.Params, cm: Cosmo, pf: dict, zp: float, deltax, sums: list, sums_agn: dict | None = None):
    """The prefactors evolveInt applies after its shell loop (XRayHeatingFunctions.c:1436-1470);
    the AGN bands' terms join the heat, ion and lya sums (:1484-1540)."""
    n_b = cm.N_b0 * float(f32(1) + f32(zp)) ** 3 * (f32(1) + np.asarray(deltax, f32)).astype(np.float64)
    sums[0] *= pf["const_zp"]
    sums[1] *= pf["const_zp"]
    sums[2] *= pf["const_zp"] * n_b
    sums[3] *= (SPEED_OF_LIGHT / (4.0 * math.pi)) / (PROTONMASS / SOLAR_MASS)
    for b, sa in (sums_agn or {}).items():
        c = pf["const_agn"][b]
        sa[0] *= c
        sa[1] *= c
        sa[2] *= c * n_b
        for k in range(3):
            sums[k] += sa[k]


def evolve_cells(p: ro.Params, cm: Cosmo, T: TsTables, pf: dict, zp: float, dzp: float, deltax, xprev, Tk_box,
                 sums: list) -> dict:
    """The rest of evolveInt, the Euler step of x_e and T_K and get_Ts, per cell
    (XRayHeatingFunctions.c:1472-1561, ComputeTs.c:1371-1407); any subset of cells."""
    dxheat, dxion, dxlya, dstar = sums
    deltax = np.asarray(deltax, f32)
    zpf = float(f32(zp))
    n_b = cm.N_b0 * float(f32(1) + f32(zp)) ** 3 * (f32(1) + deltax).astype(np.float64)
    x_e = np.asarray(xprev, f32).astype(np.float64)
    Tk = np.asarray(Tk_box, f32)
    Td = Tk.astype(np.float64)
    sink = alpha_A(Td) * CLUMPING_FACTOR * x_e * x_e * cm.f_H * n_b
    dxe_dzp = pf["dt_dzp"] * (dxion - sink)
    dadia = np.full(x_e.shape, 3 / (1.0 + zpf))
    dl = deltax.astype(np.float64)
    big = np.abs(dl) > FRACT_FLOAT_ERR
    with np.errstate(divide="ignore"):
        dadia = np.where(big, dadia + pf["dgrowth"] / (1.0 / dl + pf["growth"]), dadia)
    dadia *= (2.0 / 3.0) * Td
    dspec = -dxe_dzp * Td / (1 + x_e)
    dcomp = dT_comp(cm, zpf, Td, x_e)
    dxheat_dzp = dxheat * pf["dt_dzp"] * 2.0 / 3.0 / BOLTZMANN / (1.0 + x_e)
    d1 = dxheat_dzp + dcomp + dspec + dadia
    d2 = dxlya + dstar
    d4 = pf["dt_dzp"] * dxion
    xn = (x_e + dxe_dzp * dzp).astype(f32)
    xn = np.where(xn > 1, f32(1 - FRACT_FLOAT_ERR), np.where(xn < 0, f32(0), xn)).astype(f32)
    tk = np.where(Tk < MAX_TK, (Td + d1 * dzp).astype(f32), Tk).astype(f32)
    tk = np.where(tk < MIN_TK, f32(TCMB * (1 + zp)), tk).astype(f32)
    ts, xa = get_Ts(cm, T, zp, deltax, tk, xn, d2.astype(f32))
    return dict(x_e=xn, Tk=tk, TS=ts, xalpha=xa, J_alpha=d2, dxheat_dzp=dxheat_dzp, dxion=d4)

