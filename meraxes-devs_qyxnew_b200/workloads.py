"""Seeded synthetic inputs for the reionization grid step.

Meraxes builds its source grids from galaxies (``construct_baryon_grids``,
src/core/reionization.c:2025) and reads the density grid from N-body files
(src/core/read_grids.c).  Neither is available here, so these generators make
grids with the same layouts, units and value ranges:

* ``deltax``  : lognormal density contrast ``exp(g - sigma^2/2) - 1`` where ``g``
  is a Gaussian random field with P(k) ~ k^-2 and a Gaussian cut-off at half the
  Nyquist wavenumber, normalised to sigma = 0.8;
* ``stars``   : 1e7 Msun x (1+deltax)^2 x LN(0, 0.5), zeroed in a seeded 80% of
  the cells, in internal mass units (1e10 Msun/h per cell);
* ``sfr``     : stars x 1e-8 /yr x LN(0, 0.3), internal mass per internal time;
  also used as ``weighted_sfr``;
* ``xray``    : LXrayGal (3.16e40 erg/s per Msun/yr) x SFR, in units of 1e40 erg/s
  (XRAY_LUMINOSITY_UNIT, src/meraxes.h:36).

Real grids use the FFTW in-place padded layout ``[N][N][2(N/2+1)]``
(``INDEX_PADDED``, src/core/misc_tools.c:249) with zeros in the padding.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

# cgs constants, src/meraxes.h:21-37
SOLAR_MASS = 1.989e33
SEC_PER_YEAR = 3.155e7

# Genesis cosmology and units (input/params/simulations/Genesis_L10_N512.par:17-31)
COSMO = dict(OmegaM=0.3121, OmegaK=0.0, OmegaLambda=0.6879, OmegaR=0.0,
             BaryonFrac=0.15714, Hubble_h=0.6751, wLambda=-1.0)
UNITS = dict(UnitLength_in_cm=3.08568e24, UnitMass_in_g=1.989e43,
             UnitVelocity_in_cm_per_s=1.0e5)


def padded_shape(n: int) -> tuple[int, int, int]:
    return (n, n, 2 * (n // 2 + 1))


def to_padded(real: np.ndarray) -> np.ndarray:
    """Embed an [N][N][N] array in the FFTW in-place padded layout (float32)."""
    n = real.shape[0]
    out = np.zeros(padded_shape(n), dtype=np.float32)
    out[:, :, :n] = real
    return out


def from_padded(pad: np.ndarray) -> np.ndarray:
    n = pad.shape[0]
    return pad[:, :, :n]


def gaussian_field(n: int, box: float, rng: np.random.Generator, sigma: float = 0.8) -> np.ndarray:
    """Gaussian random field with P(k) ~ k^-2 exp(-k^2 / (2 kc^2)), kc = 0.5 k_Nyq."""
    white = rng.standard_normal((n, n, n))
    wk = np.fft.rfftn(white)
    kf = 2.0 * np.pi / box
    kx = np.fft.fftfreq(n, d=1.0 / n) * kf
    kz = np.fft.rfftfreq(n, d=1.0 / n) * kf
    k2 = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    k_nyq = np.pi * n / box
    kc = 0.5 * k_nyq
    with np.errstate(divide="ignore"):
        pk = np.where(k2 > 0, 1.0 / k2, 0.0) * np.exp(-k2 / (2.0 * kc * kc))
    g = np.fft.irfftn(wk * np.sqrt(pk), s=(n, n, n), axes=(0, 1, 2))
    g -= g.mean()
    g *= sigma / g.std()
    return g


@dataclasses.dataclass
class SourceGrids:
    n: int
    box: float
    deltax: np.ndarray        # padded float32
    stars: np.ndarray         # padded float32, internal mass units
    sfr: np.ndarray           # padded float32, internal mass / internal time
    xray: np.ndarray          # padded float32, 1e40 erg/s


def make_sources(n: int, box: float, seed: int, source_scale: float = 1.0) -> SourceGrids:
    rng = np.random.default_rng(seed)
    sigma = 0.8
    g = gaussian_field(n, box, rng, sigma)
    deltax = np.exp(g - 0.5 * sigma * sigma) - 1.0
    h = COSMO["Hubble_h"]
    unit_time_s = UNITS["UnitLength_in_cm"] / UNITS["UnitVelocity_in_cm_per_s"]
    msun_internal = h / 1e10                      # 1 Msun in 1e10 Msun/h
    stars = 1e7 * msun_internal * (1.0 + deltax) ** 2 * rng.lognormal(0.0, 0.5, size=deltax.shape)
    stars *= source_scale
    stars[rng.random(deltax.shape) < 0.8] = 0.0
    per_year_internal = unit_time_s / SEC_PER_YEAR   # 1/yr -> 1/internal time
    sfr = stars * 1e-8 * per_year_internal * rng.lognormal(0.0, 0.3, size=deltax.shape)
    # SFR in Msun/yr, then L_X in 1e40 erg/s
    sfr_msun_yr = sfr * UNITS["UnitMass_in_g"] / SOLAR_MASS / per_year_internal
    xray = 3.16e40 * sfr_msun_yr / 1.0e40
    return SourceGrids(n=n, box=box, deltax=to_padded(deltax), stars=to_padded(stars),
                       sfr=to_padded(sfr), xray=to_padded(xray))


def snapshot_redshifts(z_target: float, z_first: float = 40.0, n_before: int = 60,
                       dlog: float | None = None) -> tuple[np.ndarray, int]:
    """Descending snapshot redshift list ending at ``z_target`` (index returned).

    Snapshots are uniform in log(1+z) from ``z_first`` down to ``z_target``,
    the way N-body snapshot lists usually are.  Two extra later snapshots
    follow so the list looks like a run in progress.
    """
    if dlog is None:
        dlog = (math.log1p(z_first) - math.log1p(z_target)) / n_before
    zz = [math.expm1(math.log1p(z_target) + dlog * (n_before - i)) for i in range(n_before + 1)]
    zz += [math.expm1(math.log1p(z_target) - dlog * j) for j in (1, 2)]
    return np.asarray(zz, dtype=np.float64), n_before


# ReionEfficiency as set_ReionEfficiency() (src/core/reionization.c:299-328) makes it
# from the defaults: 1/BaryonFrac * ReionNionPhotPerBary / (1 - 0.75 Y_He).
DEFAULT_REION_EFFICIENCY = 1.0 / 0.15714 * 4000.0 / (1.0 - 0.75 * 0.24)


@dataclasses.dataclass
class GridConfig:
    """One workload configuration: grid size, box, redshift and reionization params."""
    name: str
    n: int
    box: float               # Mpc/h
    z: float
    filter_type: int = 0
    delta_r_factor: float = 1.1
    r_bubble_max: float = 50.0
    r_bubble_min: float = 0.4068
    evolving_rmax: int = 0
    efficiency: float = 1.0
    uvb_flag: int = 1
    spin_temp: int = 0
    ts_filter_type: int = 1
    ts_steps: int = 40
    seed: int = 1809
    source_scale: float = 1.0


CONFIGS = {
    # plain find_HII_bubbles, 64^3, 64 Mpc/h, z=8, tophat, R from 50 Mpc/h, f=1.1, eff=1.0
    "c0_64": GridConfig("c0_64", 64, 64.0, 8.0, seed=1809),
    # the same generators at 256^3, 250 Mpc/h, z=7
    "c1_256": GridConfig("c1_256", 256, 250.0, 7.0, seed=1810),
    # ComputeTs + delta_T at 128^3, 128 Mpc/h, z=15, 40 shells, sharp-k heating filter
    "c3_128": GridConfig("c3_128", 128, 128.0, 15.0, spin_temp=1, seed=1812),
    # full step at 512^3, 500 Mpc/h, z=8, R0 = 0.62*L (about 60 radii), then Ts and delta_T
    "c4_512": GridConfig("c4_512", 512, 500.0, 8.0, r_bubble_max=1000.0, spin_temp=1, seed=1813),
    # the same step at 256^3 (250 Mpc/h): the small case for kernel captures (inputs still > L2)
    "c4_256": GridConfig("c4_256", 256, 250.0, 8.0, r_bubble_max=1000.0, spin_temp=1, seed=1813),
}


@dataclasses.dataclass
class TsInputs:
    """Spin-temperature inputs besides the source grids (all padded float32 unless noted)."""
    x_e_box_prev: np.ndarray
    Tk_box: np.ndarray                 # real [N]^3
    sfr_histories: list                # slot h = snapshot (current - h)
    xray_histories: list
    stored_fcoll: np.ndarray           # float64 [n_snapshots]


def rec_stand_in_tables(nz: int = 200, nt: int = 100, ng: int = 150):
    """Smooth stand-in MHR recombination tables (lnGamma knots, then ln rate, clumping factor and ln
    residual xH, each [nz][nt][ng]) with the real tables' sample grid (z = 0.2 i, log10 T =
    2 + 0.03 j, ln Gamma12 = -10 + 0.1 k as float sums) and ranges (ln rate about -48 to -30,
    clumping 1 to 5, ln residual xH about -14 to 7).  The MHR integrals themselves are not
    evaluated: the step only interpolates the tables the caller hands over."""
    f32 = np.float32
    knots = np.array([f32(f32(-10.0) + f32(f32(0.1) * f32(i))) for i in range(ng)], np.float64)
    z = np.arange(nz) * float(f32(0.2))
    lt = float(f32(2.0)) + np.arange(nt) * float(f32(0.03))
    Z, T, G = np.meshgrid(z, lt, knots, indexing="ij")
    RR = -36.3 - 8.0 * np.exp(-(G + 10.0) / 2.5) + 0.15 * (Z - 8.0) - 0.3 * (T - 4.0) + 0.02 * np.sin(1.3 * G)
    CF = 1.0 + 4.0 / (1.0 + np.exp(-(G + 2.5) / 1.5)) * (1.0 + 0.01 * Z) * (1.0 + 0.05 * (T - 4.0) ** 2)
    RNH = 6.7 - 1.2 * (G + 10.0) + 0.05 * Z + 0.4 * (T - 4.0) + 0.03 * np.cos(0.7 * G)
    return knots, RR, CF, RNH


def history_scale(zz: np.ndarray, snap: int, h: int) -> float:
    """SFR history amplitude of slot h relative to this snapshot: ((1 + z_h) / (1 + z))^-3."""
    zh = zz[snap - h] if snap - h >= 0 else zz[0]
    return ((1.0 + zh) / (1.0 + zz[snap])) ** -3.0


def make_config_ts_inputs(src: SourceGrids, zz: np.ndarray, snap: int, n_hist: int,
                          fcoll_prev: float = 1e-5) -> TsInputs:
    """The ComputeTs workload's state: uniform T_K = 12 K and x_e = 2e-4, and per-slot
    SFR / X-ray histories = this snapshot's grids x ((1 + z_h) / (1 + z))^-3."""
    n = src.n
    xe = np.full(padded_shape(n), 2e-4, np.float32)
    xe[:, :, n:] = 0.0
    tk = np.full((n, n, n), 12.0, np.float32)
    sfr_h = [(src.sfr * np.float32(history_scale(zz, snap, h))).astype(np.float32) for h in range(n_hist)]
    xr_h = [(src.xray * np.float32(history_scale(zz, snap, h))).astype(np.float32) for h in range(n_hist)]
    sf = np.zeros(len(zz))
    if snap > 0:
        sf[snap - 1] = fcoll_prev
    return TsInputs(x_e_box_prev=xe, Tk_box=tk, sfr_histories=sfr_h, xray_histories=xr_h, stored_fcoll=sf)


def make_ts_inputs(src: SourceGrids, zz: np.ndarray, snap: int, n_hist: int, seed: int,
                   fcoll_prev: float = 1e-5) -> TsInputs:
    """Synthetic ComputeTs state: x_e ~ 2e-4 LN(0, 0.3), T_K ~ 12 K (1 + 0.3 delta) floored at
    2 K, and SFR / X-ray histories that decay towards higher redshift as exp(-0.4 (z_h - z))
    with a per-slot LN(0, 0.2) cell modulation (slot 0 is this snapshot's grids)."""
    rng = np.random.default_rng(seed)
    n = src.n
    d = from_padded(src.deltax).astype(np.float64)
    xe = 2e-4 * rng.lognormal(0.0, 0.3, size=d.shape)
    tk = np.maximum(12.0 * (1.0 + 0.3 * d), 2.0).astype(np.float32)
    sfr_h, xr_h = [src.sfr.copy()], [src.xray.copy()]
    for h in range(1, n_hist):
        zh = zz[snap - h] if snap - h >= 0 else zz[0]
        mod = rng.lognormal(0.0, 0.2, size=d.shape) * math.exp(-0.4 * (zh - zz[snap]))
        sfr_h.append(to_padded(from_padded(src.sfr) * mod))
        xr_h.append(to_padded(from_padded(src.xray) * mod))
    sf = np.zeros(len(zz))
    if snap > 0:
        sf[snap - 1] = fcoll_prev
    return TsInputs(x_e_box_prev=to_padded(xe), Tk_box=tk, sfr_histories=sfr_h, xray_histories=xr_h,
                    stored_fcoll=sf)


# The batched workload: 48 independent snapshots spanning z = 16 -> 6 over boxes of uneven size
# (64^3, 96^3, 128^3, 192^3, 12 each, L = N Mpc/h).  The sources are the generators above; the
# ionising efficiency per redshift is interpolated (in log) from a calibration of the 64^3 box
# against the CPU oracle so that mean xH runs linearly from 0.99 at z = 16 to 0.1 at z = 6.
BATCH_EFFICIENCY = [(16.0, 563.0), (14.0, 11913.0), (12.0, 19338.0), (10.0, 24313.0), (8.0, 28013.0),
                    (6.0, 29729.0)]
BATCH_SIZES = (64, 96, 128, 192)
BATCH_UNITS = 48


def batch_efficiency(z: float) -> float:
    zs = [a for a, _ in BATCH_EFFICIENCY][::-1]
    ls = [math.log(b) for _, b in BATCH_EFFICIENCY][::-1]
    return math.exp(float(np.interp(z, zs, ls)))


@dataclasses.dataclass
class BatchUnit:
    index: int
    n: int
    box: float
    z: float
    efficiency: float
    seed: int


def batch_units(count: int = BATCH_UNITS) -> list[BatchUnit]:
    out = []
    for i in range(count):
        z = 16.0 - 10.0 * i / (count - 1)
        n = BATCH_SIZES[i % len(BATCH_SIZES)]
        out.append(BatchUnit(i, n, float(n), z, batch_efficiency(z), 1811 + i))
    return out
