"""The combined host-buffer step (rg_reion_step_host) against the three host-buffer calls made one
after another (rg_compute_Ts_host, rg_find_HII_bubbles_host, rg_delta_T_host) on copies of the
same host arrays: every output grid and every scalar must be identical."""

import ctypes as C

import numpy as np
import pytest

import rg_b200 as rg
import workloads as wl

pytestmark = pytest.mark.gpu


def host_arrays(n, src, ti, rng, vel):
    npad = n * n * 2 * (n // 2 + 1)
    a = dict(deltax=src.deltax.copy(), stars=src.stars.copy(), weighted_sfr=src.sfr.copy(), sfr=src.sfr.copy(),
             xray_luminosity=src.xray.copy(), x_e_box_prev=ti.x_e_box_prev.copy(), Tk_box=ti.Tk_box.copy(),
             x_e_box=np.zeros(npad, np.float32), TS_box=np.zeros(n ** 3, np.float32),
             sfr_histories=np.stack(ti.sfr_histories), xray_luminosity_histories=np.stack(ti.xray_histories),
             xH=np.zeros(n ** 3, np.float32), r_bubble=np.full(n ** 3, 3.0, np.float32),
             z_at_ionization=np.full(n ** 3, -1.0, np.float32), J_21_at_ionization=np.zeros(n ** 3, np.float32),
             temp_kinetic_all_gas=np.zeros(n ** 3, np.float32), delta_T=np.zeros(n ** 3, np.float32))
    if vel:
        a["vel"] = (20.0 * rng.standard_normal(npad)).astype(np.float32)
    return a


def grids_of(a, n_hist):
    g = rg.rg_grids()
    for k, v in a.items():
        setattr(g, k, v.ctypes.data)
    g.n_hist = n_hist
    return g


@pytest.mark.parametrize("n,box,pecvel,mode", [(32, 64.0, 0, rg.RG_MODE_FUSED), (32, 64.0, 3, rg.RG_MODE_FUSED),
                                                (64, 96.0, 0, rg.RG_MODE_PLAIN)])
def test_combined_step_matches_three_calls(n, box, pecvel, mode):
    zz, idx = wl.snapshot_redshifts(15.0)
    src = wl.make_sources(n, box, 21)
    ti = wl.make_ts_inputs(src, zz, idx, idx + 1, 22)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=50.0,
                       ReionEfficiency=3000.0, Flag_IncludePecVelsFor21cm=pecvel)
    nh = len(ti.sfr_histories)
    outs = []
    for combined in (False, True):
        a = host_arrays(n, src, ti, np.random.default_rng(5), pecvel > 0)
        g = grids_of(a, nh)
        sf = ti.stored_fcoll.copy()
        s = rg.snapshot(zz, idx, sf)
        ts, hii, tb = rg.rg_ts_scalars(), rg.rg_hii_scalars(), C.c_double()
        ctx = rg.Context(n)
        ctx.call("rg_set_mode", mode)
        if combined:
            ctx.call("rg_reion_step_host", C.byref(p), C.byref(s), C.byref(g), C.byref(ts), C.byref(hii),
                     C.byref(tb))
        else:
            ctx.call("rg_compute_Ts_host", C.byref(p), C.byref(s), C.byref(g), C.byref(ts))
            ctx.call("rg_find_HII_bubbles_host", C.byref(p), C.byref(s), C.byref(g), C.byref(hii))
            ctx.call("rg_delta_T_host", C.byref(p), C.byref(s), C.byref(g), C.byref(tb))
        ctx.close()
        outs.append((a, ts.as_dict() if hasattr(ts, "as_dict") else None, hii.as_dict(), tb.value, sf))
    (a0, t0, h0, b0, s0), (a1, t1, h1, b1, s1) = outs
    for k in ("x_e_box_prev", "x_e_box", "Tk_box", "TS_box", "xH", "r_bubble", "z_at_ionization",
              "J_21_at_ionization", "temp_kinetic_all_gas"):
        assert np.array_equal(a0[k], a1[k]), k
    if pecvel == 3:
        # the line-of-sight shares meet in any order: float-level agreement
        assert np.max(np.abs(a0["delta_T"] - a1["delta_T"])) <= 1e-5 * np.max(np.abs(a0["delta_T"]))
        assert b1 == pytest.approx(b0, rel=1e-6)
    else:
        assert np.array_equal(a0["delta_T"], a1["delta_T"])
        assert b0 == b1
    assert h0 == h1 and t0 == t1
    assert np.array_equal(s0, s1)
    assert np.all(a1["r_bubble"] == 0.0)


def test_combined_step_with_agn_and_recombinations():
    """The same comparison with both AGN X-ray bands in ComputeTs and the recombination branch in
    find_HII_bubbles (their extra grids staged through the host arrays of both forms)."""
    import test_gpu_rec as tr
    import test_gpu_ts_agn as ta
    n, box = 32, 64.0
    zz, idx = wl.snapshot_redshifts(15.0)
    src = wl.make_sources(n, box, 31)
    ti = wl.make_ts_inputs(src, zz, idx, idx + 1, 32)
    agn = ta.agn_inputs(src, ti, 33)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMaxRecomb=50.0,
                       ReionEfficiency=20000.0, Flag_IncludeAGNXray=1, Flag_IncludeRecombinations=1, ReionUVBFlag=2)
    nh = len(ti.sfr_histories)
    rng = np.random.default_rng(34)
    n_rec0 = wl.to_padded((0.3 * rng.random((n, n, n))).astype(np.float32)).ravel()
    g12 = (0.5 * rng.random(n ** 3)).astype(np.float32)
    outs = []
    for combined in (False, True):
        a = host_arrays(n, src, ti, np.random.default_rng(5), False)
        for b in ("soft", "hard"):
            a["bh_xray_" + b] = np.ascontiguousarray(agn["bh_xray_" + b])
            a["bh_xray_histories_" + b] = np.stack(agn["bh_xray_histories_" + b])
        a.update(N_rec=n_rec0.copy(), Gamma12=g12.copy(), residual_xH=np.zeros(n ** 3, np.float32),
                 clumping_factor=np.zeros(n ** 3, np.float32), t_resp=np.zeros(n ** 3, np.float32))
        g = grids_of(a, nh)
        sf = ti.stored_fcoll.copy()
        s = rg.snapshot(zz, idx, sf)
        ts, hii, tb = rg.rg_ts_scalars(), rg.rg_hii_scalars(), C.c_double()
        ctx = rg.Context(n)
        tr.set_tables(ctx)
        if combined:
            ctx.call("rg_reion_step_host", C.byref(p), C.byref(s), C.byref(g), C.byref(ts), C.byref(hii),
                     C.byref(tb))
        else:
            ctx.call("rg_compute_Ts_host", C.byref(p), C.byref(s), C.byref(g), C.byref(ts))
            ctx.call("rg_find_HII_bubbles_host", C.byref(p), C.byref(s), C.byref(g), C.byref(hii))
            ctx.call("rg_delta_T_host", C.byref(p), C.byref(s), C.byref(g), C.byref(tb))
        ctx.close()
        outs.append((a, ts.as_dict(), hii.as_dict(), tb.value, sf))
    (a0, t0, h0, b0, s0), (a1, t1, h1, b1, s1) = outs
    for k in ("x_e_box_prev", "x_e_box", "Tk_box", "TS_box", "xH", "r_bubble", "z_at_ionization",
              "J_21_at_ionization", "temp_kinetic_all_gas", "delta_T", "N_rec", "Gamma12", "residual_xH",
              "clumping_factor", "t_resp"):
        assert np.array_equal(a0[k], a1[k]), k
    assert h0 == h1 and t0 == t1 and b0 == b1
    assert np.array_equal(s0, s1)
    assert t1["volume_ave_Xheat_AGN_soft"] != 0 and h1["volume_weighted_global_N_rec"] > 0
    assert np.any(a1["r_bubble"] > 0)
