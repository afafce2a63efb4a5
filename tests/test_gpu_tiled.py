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


def test_find_hii_recombinations_512_tiled_matches_oracle():
    """The recombination branch at 512^3: N_rec and Gamma12 from a previous snapshot (tiled), the
    barrier against 1 + N_rec, the first-crossing records and the recombination closing pass."""
    import rec_oracle as rco
    import test_gpu_rec as tr
    install_recfast()
    zz, snap = wl.snapshot_redshifts(8.0)
    z, prev_z = float(zz[snap]), float(zz[snap - 1])
    src8 = wl.make_sources(N8, BOX8, seed=4545)
    rng = np.random.default_rng(4546)
    nrec8 = (0.4 * rng.random((N8, N8, N8))).astype(np.float32)
    g12_8 = (0.8 * rng.random((N8, N8, N8))).astype(np.float32)
    kw = dict(Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMaxRecomb=4.0, ReionEfficiency=20000.0,
              Flag_IncludeRecombinations=1, ReionUVBFlag=2)
    p8 = rg.make_params(N8, BOX8, **kw)
    st = ro.HIIState.fresh(N8, rec=True)
    st.N_rec[:] = nrec8
    st.Gamma12[:] = g12_8
    xH_o, rb_o, s_o, diag = ro.find_hii_bubbles(oracle_params(p8), z, src8.deltax, src8.stars, src8.sfr, st, "fp64",
                                                record_margins=True, rec_tables=tr.tables(), prev_z=prev_z)
    dg = DeviceGrids(N, rec=True)
    dg.put("deltax", tile_padded(src8.deltax))
    dg.put("stars", tile_padded(src8.stars))
    dg.put("weighted_sfr", tile_padded(src8.sfr))
    dg.put("N_rec", wl.to_padded(tile_real(nrec8)))
    dg.put("Gamma12", tile_real(g12_8))
    p = rg.make_params(N, BOX, **kw)
    ctx = rg.Context(N)
    tr.set_tables(ctx)
    out = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(rg.snapshot(zz, snap)), C.byref(dg.g), C.byref(out))
    ctx.close()
    ok = tile_real(diag["min_margin"] > 1e-4)
    ion_o = tile_real(xH_o < ro.REL_TOL)
    assert 0.05 < ion_o.mean() < 0.95
    assert np.array_equal((dg.get("xH") < ro.REL_TOL)[ok], ion_o[ok])
    assert np.array_equal(dg.get("r_bubble")[ok], tile_real(rb_o)[ok])
    crossed = ok & tile_real(rb_o > 0)
    assert rel_l2(dg.get("Gamma12")[crossed], tile_real(st.Gamma12)[crossed]) <= 1e-4
    assert rel_l2(dg.get("J_21_at_ionization")[crossed], tile_real(st.J_21_at_ionization)[crossed]) <= 1e-4
    # cells whose (z, T) table row is the same on both sides (see test_gpu_rec)
    dxu = tile_real(wl.from_padded(src8.deltax))
    same_row = tr.table_row(z, dxu, dg.get("temp_kinetic_all_gas"), 1) == \
        tr.table_row(z, dxu, tile_real(st.temp_kinetic_all_gas), 1)
    cmp = ok & same_row
    assert cmp.mean() > 0.99
    assert rel_l2(wl.from_padded(dg.get("N_rec"))[cmp], tile_real(st.N_rec)[cmp]) <= 1e-4
    for name in ("residual_xH", "clumping_factor", "t_resp"):
        assert rel_l2(dg.get(name)[cmp], tile_real(diag["rec"][name])[cmp]) <= 1e-4, name
    for k in ("Gamma12", "N_rec", "residual_xH", "clumping_factor"):
        for w in ("volume", "mass"):
            key = f"{w}_weighted_global_{k}"
            assert getattr(out, key) == pytest.approx(s_o[key], rel=1e-4), key


def test_compute_ts_agn_256_tiled_matches_oracle():
    """Both AGN X-ray bands at 256^3 (8^3 tiled 32 times): four grids per shell through the full
    transforms, the band tables and the AGN heating averages."""
    import torch
    import test_gpu_ts as tg
    import test_gpu_ts_agn as ta
    reps = 32
    n, box = N8 * reps, BOX8 * reps

    def tp(a):
        return wl.to_padded(np.tile(wl.from_padded(np.asarray(a).reshape(N8, N8, -1)), (reps, reps, reps)))

    zz, idx, src8, ti8 = tg.ts_case(N8, BOX8, 15.0, 4747, n_hist=16)
    agn8 = ta.agn_inputs(src8, ti8, 4748)
    p8 = rg.make_params(N8, BOX8, Flag_IncludeSpinTemp=1, Flag_IncludeAGNXray=1)
    want, wg = ta.run_oracle(p8, to.TsTables(), zz, idx, src8, ti8, agn8)
    dg = DeviceGrids(n, spin=True)
    for k, v in (("deltax", src8.deltax), ("stars", src8.stars), ("sfr", src8.sfr), ("xray_luminosity", src8.xray),
                 ("x_e_box_prev", ti8.x_e_box_prev)):
        dg.put(k, tp(v))
    dg.put("Tk_box", np.tile(ti8.Tk_box.reshape(N8, N8, N8), (reps, reps, reps)))
    nh = len(ti8.sfr_histories)
    npad = n * n * 2 * (n // 2 + 1)
    keep = []
    hist = {"sfr_histories": ti8.sfr_histories, "xray_luminosity_histories": ti8.xray_histories,
            "bh_xray_histories_soft": agn8["bh_xray_histories_soft"],
            "bh_xray_histories_hard": agn8["bh_xray_histories_hard"]}
    for name, slots in hist.items():
        t = torch.empty(nh * npad, device="cuda")
        for h in range(nh):
            t[h * npad:(h + 1) * npad].copy_(torch.from_numpy(tp(slots[h]).ravel()))
        keep.append(t)
        setattr(dg.g, name, t.data_ptr())
    for b in ("soft", "hard"):
        t = torch.from_numpy(tp(agn8["bh_xray_" + b]).ravel()).cuda()
        keep.append(t)
        setattr(dg.g, "bh_xray_" + b, t.data_ptr())
    dg.g.n_hist = nh
    snap = rg.snapshot(zz, idx, ti8.stored_fcoll.copy())
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1, Flag_IncludeAGNXray=1)
    out = rg.rg_ts_scalars()
    ctx = rg.Context(n)
    ctx.call("rg_compute_Ts", C.byref(p), C.byref(snap), C.byref(dg.g), C.byref(out))
    ctx.close()
    del keep
    assert out.homogeneous == 0
    til = lambda a: np.tile(np.asarray(a), (reps, reps, reps))
    for k in ("x_e_box_prev", "x_e_box"):
        assert rel_l2(wl.from_padded(dg.get(k)), til(wg[k])) <= 1e-5, k
    for k in ("Tk_box", "TS_box"):
        assert rel_l2(dg.get(k), til(wg[k])) <= 1e-5, k
    for k in tg.SCALARS + ["volume_ave_Xheat_AGN_soft", "volume_ave_Xheat_AGN_hard"]:
        assert abs(getattr(out, k) - want[k]) <= 1e-5 * abs(want[k]) + 1e-300, k
    assert out.volume_ave_Xheat_AGN_soft != 0 and out.volume_ave_Xheat_AGN_hard != 0
