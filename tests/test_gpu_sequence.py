"""Three consecutive snapshots through rg_reion_step_host, the way Meraxes calls the block: the
state each snapshot leaves (z_at_ionization, J_21, the temperatures, x_e_box_prev, Tk_box and
stored_fcoll) is the next one's input, on the GPU side from the GPU and on the oracle side from
the oracle, so the two evolve independently.  After every snapshot: the spin-temperature grids
within 2e-5 relative L2 of the oracle, the ionised flags equal outside cells within 1e-4 of the
threshold, <x_H> within 1e-4, <T_b> within 1e-4 relative."""

import ctypes as C

import numpy as np
import pytest

import reion_oracle as ro
import rg_b200 as rg
import ts_oracle as to
import workloads as wl
from helpers import install_recfast, oracle_params, rel_l2

pytestmark = pytest.mark.gpu


def test_three_snapshots_with_carried_state():
    install_recfast()
    T = to.TsTables()
    n, box, eff = 32, 64.0, 3000.0
    zz, last = wl.snapshot_redshifts(13.0)
    seq = [last - 2, last - 1, last]
    n_hist = 14          # the shells reach 13 snapshots back
    U, P = wl.from_padded, wl.to_padded
    src0 = wl.make_sources(n, box, 60)
    ti0 = wl.make_ts_inputs(src0, zz, seq[0], n_hist, 61)
    # carried state: GPU host arrays and the oracle's own copies
    g_xe, g_tk = ti0.x_e_box_prev.copy(), ti0.Tk_box.copy()
    g_zin = np.full(n ** 3, -1.0, np.float32)
    g_j, g_t = np.zeros(n ** 3, np.float32), np.zeros(n ** 3, np.float32)
    sf_g, sf_o = ti0.stored_fcoll.copy(), ti0.stored_fcoll.copy()
    o_xe, o_tk = U(ti0.x_e_box_prev).copy(), ti0.Tk_box.copy()
    st_o = ro.HIIState.fresh(n)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=30.0,
                       ReionEfficiency=eff)
    op = oracle_params(p)
    ctx = rg.Context(n)
    for k, s in enumerate(seq):
        z = float(zz[s])
        src = wl.make_sources(n, box, 70 + k)
        ti = wl.make_ts_inputs(src, zz, s, n_hist, 80 + k)
        h = dict(deltax=src.deltax.copy(), stars=src.stars.copy(), weighted_sfr=src.sfr.copy(), sfr=src.sfr.copy(),
                 xray_luminosity=src.xray.copy(), sfr_histories=np.stack(ti.sfr_histories),
                 xray_luminosity_histories=np.stack(ti.xray_histories), x_e_box_prev=g_xe, Tk_box=g_tk,
                 x_e_box=np.zeros_like(g_xe), TS_box=np.zeros(n ** 3, np.float32), xH=np.zeros(n ** 3, np.float32),
                 r_bubble=np.zeros(n ** 3, np.float32), z_at_ionization=g_zin, J_21_at_ionization=g_j,
                 temp_kinetic_all_gas=g_t, delta_T=np.zeros(n ** 3, np.float32))
        g = rg.rg_grids()
        for name, v in h.items():
            setattr(g, name, v.ctypes.data)
        g.n_hist = len(ti.sfr_histories)
        snap = rg.snapshot(zz, s, sf_g)
        ts, hii, tb = rg.rg_ts_scalars(), rg.rg_hii_scalars(), C.c_double()
        ctx.call("rg_reion_step_host", C.byref(p), C.byref(snap), C.byref(g), C.byref(ts), C.byref(hii),
                 C.byref(tb))
        # the oracle, on its own state
        og = dict(deltax=U(src.deltax), stars=U(src.stars), x_e_box_prev=o_xe, Tk_box=o_tk, sfr=U(src.sfr),
                  xray_luminosity=U(src.xray), sfr_histories=[U(a) for a in ti.sfr_histories],
                  xray_luminosity_histories=[U(a) for a in ti.xray_histories])
        out = to.compute_ts(op, T, zz, s, sf_o, og)
        sf_o[s] = out["collapse_fraction"]
        o_xe, o_tk = og["x_e_box_prev"], og["Tk_box"]
        xH_o, _, s_o, diag = ro.find_hii_bubbles(op, z, src.deltax, src.stars, src.sfr, st_o, "fp64",
                                                 x_e_box=P(og["x_e_box"]), Tk_box=og["Tk_box"], record_margins=True)
        _, tb_o = ro.delta_T(op, z, xH_o, src.deltax, og["TS_box"])
        # compare this snapshot
        for name, want in (("x_e_box_prev", o_xe), ("x_e_box", og["x_e_box"])):
            assert rel_l2(U(h[name].reshape(n, n, -1)), want) <= 2e-5, (k, name)
        for name in ("Tk_box", "TS_box"):
            assert rel_l2(h[name].reshape(n, n, n), og[name]) <= 2e-5, (k, name)
        ok = diag["min_margin"] > 1e-4
        xH = h["xH"].reshape(n, n, n)
        assert np.array_equal((xH < ro.REL_TOL)[ok], (xH_o < ro.REL_TOL)[ok]), k
        assert abs(hii.volume_weighted_global_xH - s_o["volume_weighted_global_xH"]) <= 1e-4, k
        assert tb.value == pytest.approx(tb_o, rel=1e-4), k
        assert sf_g[s] == pytest.approx(sf_o[s], rel=1e-7), k
        g_zin, g_j, g_t = h["z_at_ionization"], h["J_21_at_ionization"], h["temp_kinetic_all_gas"]
        g_xe, g_tk = h["x_e_box_prev"], h["Tk_box"]
    ctx.close()
    # the box ionised somewhat over the three snapshots
    assert 0.0 < hii.volume_weighted_global_xH < 1.0
