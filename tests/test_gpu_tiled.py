"""Full-size parity (512^3) through a property of the transforms.

A field that repeats every 8 cells has power only at the modes k = 2 pi m / (L / 64).  On a 512^3
box of size L such fields give the 8^3 problem of box size L / 64 tiled 64 times per axis: the
cell size is the same, so are ComputeTs' shells (from the cell size to 500 Mpc) and, with
ReionRBubbleMax below 0.62 L / 64, find_HII_bubbles' radii; every filtered field is the tiled
8^3 one.  The oracle solves the 8^3 problem in about a second; the GPU runs the full 512^3 path
(its own transforms, batching, fused passes and reductions).  Tolerances are those of the
small-box parity tests."""

import ctypes as C

import numpy as np
import pytest

import reion_oracle as ro
import rg_b200 as rg
import ts_oracle as to
import workloads as wl
from helpers import DeviceGrids, install_recfast, oracle_params, rel_l2

pytestmark = pytest.mark.gpu

N8, REPS = 8, 64
N = N8 * REPS
BOX = 500.0
BOX8 = BOX / REPS


def tile_real(a):
    return np.tile(np.asarray(a).reshape(N8, N8, N8), (REPS, REPS, REPS))


def tile_padded(a):
    return wl.to_padded(tile_real(wl.from_padded(np.asarray(a).reshape(N8, N8, -1))))


def test_compute_ts_512_tiled_matches_oracle():
    import torch
    import test_gpu_ts as tg
    zz, idx, src8, ti8 = tg.ts_case(N8, BOX8, 15.0, 4242, n_hist=16)
    p8 = rg.make_params(N8, BOX8, Flag_IncludeSpinTemp=1)
    want, wg = tg.run_oracle_ts(p8, to.TsTables(), zz, idx, src8, ti8)
    # device grids filled tile by tile (one full-size host array at a time)
    dg = DeviceGrids(N, spin=True)
    dg.put("deltax", tile_padded(src8.deltax))
    dg.put("stars", tile_padded(src8.stars))
    dg.put("sfr", tile_padded(src8.sfr))
    dg.put("xray_luminosity", tile_padded(src8.xray))
    dg.put("x_e_box_prev", tile_padded(ti8.x_e_box_prev))
    dg.put("Tk_box", tile_real(ti8.Tk_box))
    nh = len(ti8.sfr_histories)
    npad = N * N * 2 * (N // 2 + 1)
    hs = torch.empty(nh * npad, device="cuda")
    hx = torch.empty(nh * npad, device="cuda")
    for h in range(nh):
        hs[h * npad:(h + 1) * npad].copy_(torch.from_numpy(tile_padded(ti8.sfr_histories[h]).ravel()))
        hx[h * npad:(h + 1) * npad].copy_(torch.from_numpy(tile_padded(ti8.xray_histories[h]).ravel()))
    dg.g.sfr_histories = hs.data_ptr()
    dg.g.xray_luminosity_histories = hx.data_ptr()
    dg.g.n_hist = nh
    sf = ti8.stored_fcoll.copy()
    snap = rg.snapshot(zz, idx, sf)
    p = rg.make_params(N, BOX, Flag_IncludeSpinTemp=1)
    out = rg.rg_ts_scalars()
    ctx = rg.Context(N)
    ctx.call("rg_compute_Ts", C.byref(p), C.byref(snap), C.byref(dg.g), C.byref(out))
    ctx.close()
    del hs, hx
    assert out.homogeneous == 0
    assert abs(out.collapse_fraction - want["collapse_fraction"]) <= 1e-7 * abs(want["collapse_fraction"])
    for k in ("x_e_box_prev", "x_e_box"):
        assert rel_l2(wl.from_padded(dg.get(k)), tile_real(wg[k])) <= 1e-5, k
    for k in ("Tk_box", "TS_box"):
        assert rel_l2(dg.get(k), tile_real(wg[k])) <= 1e-5, k
    for k in tg.SCALARS:
        assert abs(getattr(out, k) - want[k]) <= 1e-5 * abs(want[k]) + 1e-300, k


def test_find_hii_512_tiled_matches_oracle():
    install_recfast()
    z, eff = 8.0, 6000.0
    src8 = wl.make_sources(N8, BOX8, seed=4343)
    kw = dict(Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=4.0, ReionEfficiency=eff)
    p8 = rg.make_params(N8, BOX8, **kw)
    st = ro.HIIState.fresh(N8)
    xH_o, _, s_o, diag = ro.find_hii_bubbles(oracle_params(p8), z, src8.deltax, src8.stars, src8.sfr, st, "fp64",
                                             record_margins=True)
    dg = DeviceGrids(N)
    dg.put("deltax", tile_padded(src8.deltax))
    dg.put("stars", tile_padded(src8.stars))
    dg.put("weighted_sfr", tile_padded(src8.sfr))
    p = rg.make_params(N, BOX, **kw)
    zz, snap = wl.snapshot_redshifts(z)
    s = rg.snapshot(zz, snap)
    ctx = rg.Context(N)
    out = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out))
    ctx.close()
    assert out.n_radii == diag["n_radii"]
    xH = dg.get("xH")
    ok = tile_real(diag["min_margin"] > 1e-4)
    ion_g, ion_o = xH < ro.REL_TOL, tile_real(xH_o < ro.REL_TOL)
    assert np.array_equal(ion_g[ok], ion_o[ok])
    part = ok & ~ion_o
    if part.any():
        assert np.max(np.abs(xH[part] - tile_real(xH_o)[part])) <= 1e-4
    assert abs(out.volume_weighted_global_xH - s_o["volume_weighted_global_xH"]) <= 1e-4
    assert rel_l2(dg.get("temp_kinetic_all_gas")[ok], tile_real(st.temp_kinetic_all_gas)[ok]) <= 1e-5
