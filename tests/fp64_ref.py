"""FP64 restatement of the numpy oracle's excursion set on the GPU -- TEST INFRASTRUCTURE ONLY.

``find_hii_fp64`` is ``reion_oracle.find_hii_bubbles(..., "fp64")`` (src/core/find_HII_bubbles.c:
86-710) for the configurations the benchmark runs: no recombinations, no BH feedback, no Pop III,
ReionUVBFlag 1, with or without the spin-temperature grids.  The FFTs, windows, clamps and the
barrier test run in float64 with torch on the device; the float32 temperature formulas of
find_HII_bubbles.c:48-84 run on the host through the oracle's own functions on the cells that
need them.  It exists because the numpy oracle takes tens of minutes at 512^3; at every size it
can afford, ``tests/test_gpu_configs.py`` checks it against the numpy oracle first, and it is
never the thing measured.

Besides the oracle's barrier margins it marks the cells whose ionisation decision is fragile in
float arithmetic (``diag["fp32_fragile"]``): at some radius, moving each filtered field by its
FP32 error bound (FRAGILE_REL x its rms) can put the cell on either side of the barrier.  These
are mostly cells where the filtered density is close to -1, so that 1 + delta, the denominator of
the collapse fraction, has few correct digits in float; any FP32 evaluation, the reference's own
included, can decide them either way.
"""

from __future__ import annotations

import math

import numpy as np

import reion_oracle as ro


# The FP32 error bound of a filtered field, relative to its rms over the box: the float
# transforms' rounding (about log2(N^3) roundings of 2^-24 each, summed in quadrature) with a
# safety factor of about 4.
FRAGILE_REL = 1e-6


def _kmag(torch, n, box, dev):
    delta_k = 2.0 * math.pi / box
    idx = torch.arange(n, device=dev, dtype=torch.float64)
    signed = torch.where(idx > n // 2, idx - n, idx) * delta_k
    kz = torch.arange(n // 2 + 1, device=dev, dtype=torch.float64) * delta_k
    return torch.sqrt(signed[:, None, None] ** 2 + signed[None, :, None] ** 2 + kz[None, None, :] ** 2)


def _window(torch, k, R, ftype):
    kR = k * R
    if ftype == 0:
        w = 3.0 * (torch.sin(kR) / kR ** 3 - torch.cos(kR) / kR ** 2)
        return torch.where(kR > 1e-4, w, torch.ones_like(kR))
    if ftype == 1:
        return torch.where(kR * 0.413566994 > 1, torch.zeros_like(kR), torch.ones_like(kR))
    if ftype == 2:
        g = kR * 0.643
        return torch.exp(-g * g / 2.0)
    raise ValueError("ReionFilterType undefined")


def find_hii_fp64(p: ro.Params, z: float, deltax: np.ndarray, stars: np.ndarray, weighted_sfr: np.ndarray,
                  state: ro.HIIState, x_e_box: np.ndarray | None = None, Tk_box: np.ndarray | None = None,
                  device: str = "cuda:0"):
    """Same inputs, state update and return value as the oracle's fp64 find_hii_bubbles with
    ``record_margins=True``: (xH, r_bubble, scalars, diag)."""
    import torch
    if p.Flag_IncludeRecombinations or p.Flag_BHFeedback or p.UseMiniHalos or p.ReionUVBFlag != 1:
        raise ValueError("fp64_ref covers the benchmark configurations only")
    dev = torch.device(device)
    f32 = np.float32
    n, box = p.ReionGridDim, p.BoxSize
    u = ro.run_units(p)
    pixel_volume = (box / n) ** 3
    sfr_timescale = p.ReionSfrTimescale * ro.hubble_time(p, z)
    TK = f32(ro.T_RECFAST_at(z))
    cT_ad = ro.cT_approx(z)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    n3 = float(n) ** 3

    dx_real = deltax[:, :, :n]
    grids = {"deltax": dx_real, "stars": stars[:, :, :n]}
    if p.Flag_IncludeSpinTemp:
        grids["x_e"] = x_e_box[:, :, :n]
    spectra = {k: torch.fft.rfftn(T(v.astype(np.float64))) / n3 for k, v in grids.items()}
    kmag = _kmag(torch, n, box, dev)

    xH = torch.ones((n, n, n), dtype=torch.float32, device=dev)
    z_in = T(state.z_at_ionization)
    J21 = T(state.J_21_at_ionization)
    min_margin = torch.full((n, n, n), math.inf, dtype=torch.float64, device=dev)
    fragile = torch.zeros((n, n, n), dtype=torch.bool, device=dev)
    first_cross = torch.full((n, n, n), -1, dtype=torch.int16, device=dev)
    temp = state.temp_kinetic_all_gas
    rel_tol = float(ro.REL_TOL)
    abs_tol = float(ro.ABS_TOL)

    sched = ro.radius_schedule(p, z)
    for ir, (R, last) in enumerate(sched):
        w = None if last else _window(torch, kmag, R, p.ReionFilterType)
        filt = {}
        for k, s in spectra.items():
            filt[k] = torch.fft.irfftn(s if w is None else s * w, s=(n, n, n), norm="forward")
        # FP32 error bound of each filtered field at this radius (FRAGILE_REL x its rms)
        err = {k: FRAGILE_REL * float(torch.sqrt(torch.mean(v * v))) for k, v in filt.items()}
        clamp_d = lambda v: torch.clamp(v, min=ro.CLAMP_DELTAX)

        def clamp_s(v):
            v = torch.clamp(v, min=0.0)
            return torch.where(v < abs_tol, torch.zeros_like(v), v)

        def clamp_x(v):
            return torch.clamp(clamp_s(v), max=ro.CLAMP_XE)

        fd = clamp_d(filt["deltax"])
        fs = clamp_s(filt["stars"])
        if p.Flag_IncludeSpinTemp:
            fx = clamp_x(filt["x_e"])
            neutral = 1.0 - fx
            n_lo, n_hi = 1.0 - clamp_x(filt["x_e"] + err["x_e"]), 1.0 - clamp_x(filt["x_e"] - err["x_e"])
        else:
            neutral = torch.ones_like(fd)
            n_lo = n_hi = neutral
        M_mean = ro.rtom(p, R)
        g_pref = ((1.0 + z) * (1.0 + z) * R * p.UnitLength_in_cm / pixel_volume * p.UnitLength_in_cm ** -3.0)
        g_pref *= (p.UnitMass_in_g / u.UnitTime_in_s) / ro.PROTONMASS * p.ReionNionPhotPerBary
        J_aux = f32(g_pref * ro.PLANCK * 1e21 / (4.0 * math.pi) * p.ReionGammaHaloBias / sfr_timescale * p.ReionAlphaUV)
        fcoll_pref = p.ReionEfficiency * (4.0 / 3.0) * math.pi / pixel_volume / M_mean * R ** 3
        dom = 1.0 + fd
        lhs = (fs / dom) * fcoll_pref
        rhs = neutral
        ion = lhs > rhs
        # the decision is fragile where the filtered fields moved by their FP32 error bound can
        # land on either side of the barrier
        lhs_hi = clamp_s(filt["stars"] + err["stars"]) / (1.0 + clamp_d(filt["deltax"] - err["deltax"])) * fcoll_pref
        lhs_lo = clamp_s(filt["stars"] - err["stars"]) / (1.0 + clamp_d(filt["deltax"] + err["deltax"])) * fcoll_pref
        fragile |= ~((lhs_hi <= n_lo) | (lhs_lo > n_hi))
        del filt, lhs_hi, lhs_lo
        torch.minimum(min_margin, torch.abs(lhs / rhs - 1.0), out=min_margin)
        first_cross[ion & (first_cross < 0)] = ir
        xH[ion] = 0
        partial = (~ion) & (xH > float(ro.REL_TOL)) if last else None
        if partial is not None and bool(partial.any()):
            pm = partial.cpu().numpy()
            if p.Flag_IncludeSpinTemp:
                t_hi = Tk_box[pm]
            else:
                t_hi = (float(TK) * (1.0 + (cT_ad * dx_real[pm]).astype(f32).astype(np.float64))).astype(f32)
            xh_host = xH.cpu().numpy()
            temp[pm] = ro.partially_ionized_temperature(t_hi, xh_host[pm])
            v = (neutral[partial] - lhs[partial]).to(torch.float32)
            xH[partial] = torch.clamp(v, 0, 1)
        new = (xH < float(ro.REL_TOL)) & (z_in < 0)
        z_in[new] = float(f32(z))
        J21[new] = fs[new].to(torch.float32) * float(J_aux)
        del fd, fs, neutral, lhs, rhs, dom

    xH_h = xH.cpu().numpy()
    z_in_h = z_in.cpu().numpy()
    state.z_at_ionization[...] = z_in_h
    state.J_21_at_ionization[...] = J21.cpu().numpy()
    dxu = dx_real.astype(f32)
    dom = 1.0 + dxu.astype(np.float64)
    ionized = (z_in_h > 0) & (xH_h < ro.REL_TOL)
    if np.any(ionized):
        temp[ionized] = ro.fully_ionized_temperature(z_in_h[ionized], z, dxu[ionized])
    if p.Flag_IncludeSpinTemp:
        temp[:] = np.where(temp < Tk_box, Tk_box, temp)
    else:
        thistk = (float(TK) * (1.0 + (cT_ad * dxu).astype(f32).astype(np.float64))).astype(f32)
        temp[:] = np.where(temp < thistk, thistk, temp)
    r_bubble = np.zeros((n, n, n), f32)
    s = {"volume_weighted_global_xH": xH_h.astype(np.float64).sum() / n3,
         "volume_weighted_global_r_bubble": 0.0,
         "volume_weighted_global_temp_kinetic_all_gas": temp.astype(np.float64).sum() / n3}
    wsfr = weighted_sfr[:, :, :n].astype(np.float64).sum() / n3
    s["volume_weighted_global_weighted_sfr"] = wsfr * p.UnitMass_in_g / u.UnitTime_in_s * ro.SEC_PER_YEAR / ro.SOLAR_MASS
    mw = dom.sum()
    s["mass_weighted_global_xH"] = (xH_h.astype(np.float64) * dom).sum() / mw
    s["mass_weighted_global_temp_kinetic_all_gas"] = (temp.astype(np.float64) * dom).sum() / mw
    diag = {"min_margin": min_margin.cpu().numpy(), "first_cross": first_cross.cpu().numpy(),
            "n_radii": len(sched), "fp32_fragile": fragile.cpu().numpy()}
    return xH_h, r_bubble, s, diag
