"""CPU oracle for the peculiar-velocity modes of the brightness temperature -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy, ComputeBrightnessTemperatureBox with the spin temperature and
Flag_IncludePecVelsFor21cm 1-3 (src/core/BrightnessTemperature.c:24-124 prefactors, :150-509
velocity block, :512-548 average) and velocity_gradient (src/core/reionization.c:3435-3450):

* the velocity grid converted to comoving units in float steps (:173-196);
* its z derivative by FFT: r2c, / N^3, * Hubble_h, * i k_z, c2r (FP64 transforms here);
* flag 1: delta_T / (dv/dz / H + 1) with |dv/dz| capped at MAX_DVDR H; flags 2-3: the
  optical-depth form (1 - exp(-delta_T / |dv/dz / H + 1|)) 1000 (T_S - T_CMB) / (1 + z);
* flag 3: every cell with |delta_T| and x_H >= 1e-7 splits into 50 sub-cells, moves each by the
  displacement v / H interpolated between neighbouring cell centres, and adds it (or its two
  parts) to the cells it lands in along z, periodically (accumulated here in FP64).

Used only by ``tests/`` as the checker.  Parity status: **parity unpinned** (no golden vectors);
pinned by known answers in ``tests/test_vel_oracle.py`` (zero velocity leaves delta_T unchanged,
a uniform shift moves whole columns, the re-binning conserves the line sums).
"""

from __future__ import annotations

import math

import numpy as np

import reion_oracle as ro

N_RSD_STEPS = 50
MAX_DVDR = np.float32(0.2)
FRACT_FLOAT_ERR = 1e-7


def hubble(p, z: float) -> float:
    """hubble(float z) (XRayHeatingFunctions.c:443-452)."""
    opz = float(np.float32(1) + np.float32(z))
    return ro.HUBBLE * p.Hubble_h * math.sqrt(p.OmegaM * opz ** 3 + p.OmegaR * opz ** 4 + p.OmegaLambda)


def base_delta_T(p, z: float, xH, deltax, TS):
    """delta_T before the velocity block, spin temperature on (BrightnessTemperature.c:66-118)."""
    f = np.float32
    n = p.ReionGridDim
    redshift = f(z)
    h = f(p.Hubble_h)
    om = f(p.OmegaM)
    ob = f(om * f(p.BaryonFrac))
    cf = f(27.0 * (float(f(f(ob * h) * h)) / 0.023) *
           math.sqrt((0.15 / float(om) / float(h) / float(h)) * (1.0 + float(redshift)) / 10.0))
    dT = (float(cf) * xH.astype(np.float64) * (1.0 + deltax[:, :, :n].astype(np.float64))).astype(f)
    if p.Flag_IncludePecVelsFor21cm > 1:
        dT = (dT.astype(np.float64) * ((1.0 + float(redshift)) / (1000.0 * TS.astype(np.float64)))).astype(f)
    else:
        t_rad = ro.TCMB * (1.0 + float(redshift))
        dT = (dT.astype(np.float64) * (1.0 - t_rad / TS.astype(np.float64))).astype(f)
    return dT


def convert_velocity(vel, trees: int, z: float):
    """Comoving velocity from the tree code's units (BrightnessTemperature.c:173-196), real cells."""
    f = np.float32
    zf = float(f(z))
    v = vel.astype(f)
    if trees == 1:
        v = (math.sqrt(1.0 / (1.0 + zf)) * v.astype(np.float64) / 1000.0).astype(f)
    else:
        v = ((1.0 + zf) * v.astype(np.float64)).astype(f)
    v = (v.astype(np.float64) * (1000.0 * 100.0 / ro.MPC)).astype(f)
    return (v.astype(np.float64) / (1.0 / (1.0 + zf))).astype(f)


def z_gradient(vc, box_h: float, hubble_h: float):
    """d v / d z by FFT (BrightnessTemperature.c:201-215, reionization.c:3435-3450), FP64."""
    n = vc.shape[0]
    spec = np.fft.rfftn(vc.astype(np.float64)) / float(n) ** 3 * hubble_h
    dk = float(np.float32(2.0 * np.pi / float(np.float32(box_h))))
    kz = np.arange(n // 2 + 1) * dk
    spec = spec * (1j * kz)[None, None, :]
    return np.fft.irfftn(spec, s=(n, n, n), axes=(0, 1, 2)) * float(n) ** 3


def rsd(dT, xH, vc, H_z: float, box_mpc: float):
    """Line-of-sight re-binning of 50 sub-cells per cell (BrightnessTemperature.c:307-509), FP64 sums."""
    n = dT.shape[0]
    sub_w = (box_mpc / float(n)) / N_RSD_STEPS
    cell = box_mpc / float(np.float32(n))
    it = np.arange(N_RSD_STEPS)
    x_off = (sub_w * it.astype(np.float32).astype(np.float64) + sub_w / 2.0).astype(np.float32)
    x_pos = (x_off.astype(np.float64) / cell).astype(np.float32)
    hz = np.float32(H_z)
    disp_cell = (vc / hz).astype(np.float32).astype(np.float64)         # v / H (float division)
    prev = np.roll(disp_cell, 1, axis=2)
    nxt = np.roll(disp_cell, -1, axis=2)
    use = (np.abs(dT.astype(np.float64)) >= FRACT_FLOAT_ERR) & (xH.astype(np.float64) >= FRACT_FLOAT_ERR)
    xp = x_pos.astype(np.float64)[None, None, None, :]
    d1l, d2l = prev[..., None], disp_cell[..., None]
    d1h, d2h = disp_cell[..., None], nxt[..., None]
    disp = np.where(xp <= 0.5, d1l + (xp + 0.5) * (d2l - d1l), d1h + (xp - 0.5) * (d2h - d1h))
    pos = (x_off.astype(np.float64)[None, None, None, :] + disp) / cell
    half = (sub_w / 2.0) / cell
    w_sub = sub_w / cell
    lo, hi = pos - half, pos + half
    kk = np.broadcast_to(np.arange(n)[None, None, :, None], lo.shape)
    val = dT.astype(np.float64)[..., None] / N_RSD_STEPS
    val = np.broadcast_to(val, lo.shape)
    targets, weights = [], []

    def add(mask, t, w):
        targets.append(np.where(mask, t, -1))
        weights.append(np.where(mask, w, 0.0))

    c1 = (lo >= 0) & (hi < 1)
    c2 = ~c1 & (lo < 0) & (hi < 0)
    c3 = ~c1 & ~c2 & (lo < 0) & (hi > 0) & (hi < 1)
    c4 = ~c1 & ~c2 & ~c3 & (lo >= 0) & (lo < 1) & (hi >= 1)
    c5 = ~c1 & ~c2 & ~c3 & ~c4
    add(c1, kk, 1.0)
    cd2 = np.ceil(np.abs(lo)) - 1.0
    ic2 = cd2.astype(np.int64)
    whole2 = c2 & (np.abs(hi) > cd2)
    part2 = c2 & ~whole2
    fo2 = (np.abs(lo) - cd2) / w_sub
    add(whole2, kk - (ic2 + 1), 1.0)
    add(part2, kk - ic2, 1.0 - fo2)
    add(part2, kk - (ic2 + 1), fo2)
    fw3 = hi / w_sub
    add(c3, kk - 1, 1.0 - fw3)
    add(c3, kk, fw3)
    fo4 = (hi - 1.0) / w_sub
    add(c4, kk, 1.0 - fo4)
    add(c4, kk + 1, fo4)
    cd5 = np.floor(np.abs(hi))
    ic5 = cd5.astype(np.int64)
    whole5 = c5 & (lo >= cd5)
    part5 = c5 & ~whole5
    fo5 = (hi - cd5) / w_sub
    add(whole5, kk + ic5, 1.0)
    add(part5, kk + ic5 - 1, 1.0 - fo5)
    add(part5, kk + ic5, fo5)
    out = np.zeros((n * n, n))
    line = np.broadcast_to(np.arange(n * n).reshape(n, n)[:, :, None, None], lo.shape)
    usem = np.broadcast_to(use[..., None], lo.shape)
    for t, w in zip(targets, weights):
        m = usem & (w != 0.0)
        np.add.at(out, (line[m], np.mod(t[m], n)), w[m] * val[m])
    return out.reshape(n, n, n)


def delta_T_velocity(p, z: float, xH, deltax, TS, vel):
    """delta_T and its volume average with the velocity block (flags 1-3, spin temperature on)."""
    n = p.ReionGridDim
    f = np.float32
    redshift = float(f(z))
    dT = base_delta_T(p, z, xH, deltax, TS).astype(np.float64)
    vc = convert_velocity(vel[:, :, :n], p.TreesID, z)
    H_z = float(f(hubble(p, z)))
    grad = z_gradient(vc, p.BoxSize, p.Hubble_h)
    t_rad = ro.TCMB * (1.0 + redshift)
    flag = p.Flag_IncludePecVelsFor21cm
    if flag == 1:
        mvd = abs(float(f(MAX_DVDR * f(H_z))))
        dvdx = np.clip(grad, -mvd, mvd)
        dT = dT / (dvdx / H_z + 1.0)
    else:
        gc = np.abs(grad / H_z + 1.0)
        ts = TS.astype(np.float64)
        full = 1000.0 * (ts - t_rad) / (1.0 + redshift)
        with np.errstate(over="ignore"):
            dT = np.where(gc < FRACT_FLOAT_ERR, full, (1.0 - np.exp(-dT / np.maximum(gc, 1e-300))) * full)
    if flag == 3:
        dT = rsd(dT.astype(f), xH, vc, H_z, p.BoxSize / p.Hubble_h)
    return dT, dT.sum() / float(n) ** 3
