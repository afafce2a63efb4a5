"""GPU parity of the spin-temperature step (rg_compute_Ts) against the CPU oracle.

Tolerances (FP32 FFTs and FP32-within-a-shell-batch sums on the GPU vs the FP64 oracle):
* x_e_box, Tk_box and TS_box: relative L2 error <= 1e-5 over the box;
* box averages (J_alpha, xalpha, Xheat, Xion, TS, TK, x_e): relative error <= 1e-5;
* collapse fraction and <x_e> (FP64 reductions of float grids): relative error <= 1e-9.
"""

import ctypes as C

import numpy as np
import pytest

import rg_b200 as rg
import ts_oracle as to
import workloads as wl
from helpers import DeviceGrids, oracle_params, rel_l2

pytestmark = pytest.mark.gpu

SCALARS = ["volume_ave_J_alpha", "volume_ave_xalpha", "volume_ave_Xheat", "volume_ave_Xion",
           "volume_ave_TS", "volume_ave_TK", "volume_ave_xe"]


@pytest.fixture(scope="module")
def ts_tables():
    return to.TsTables()


def ts_case(n, box, z, seed, n_hist=None, stars_scale=1.0):
    zz, idx = wl.snapshot_redshifts(z)
    src = wl.make_sources(n, box, seed, source_scale=stars_scale)
    if n_hist is None:
        n_hist = idx + 1
    ti = wl.make_ts_inputs(src, zz, idx, n_hist, seed + 1)
    return zz, idx, src, ti


def run_gpu_ts(p, zz, idx, src, ti, host=False):
    import torch
    n = src.n
    dg = DeviceGrids(n, spin=True)
    dg.put("deltax", src.deltax)
    dg.put("stars", src.stars)
    dg.put("sfr", src.sfr)
    dg.put("xray_luminosity", src.xray)
    dg.put("x_e_box_prev", ti.x_e_box_prev)
    dg.put("Tk_box", ti.Tk_box)
    nh = len(ti.sfr_histories)
    hs = torch.from_numpy(np.stack(ti.sfr_histories).ravel()).cuda()
    hx = torch.from_numpy(np.stack(ti.xray_histories).ravel()).cuda()
    dg.g.sfr_histories = hs.data_ptr()
    dg.g.xray_luminosity_histories = hx.data_ptr()
    dg.g.n_hist = nh
    sf = ti.stored_fcoll.copy()
    snap = rg.snapshot(zz, idx, sf)
    out = rg.rg_ts_scalars()
    ctx = rg.Context(n)
    if not host:
        ctx.call("rg_compute_Ts", C.byref(p), C.byref(snap), C.byref(dg.g), C.byref(out))
        res = {k: dg.get(k) for k in ("x_e_box_prev", "x_e_box", "Tk_box", "TS_box")}
    else:
        hg = rg.rg_grids()
        arrs = dict(deltax=src.deltax.copy(), stars=src.stars.copy(), sfr=src.sfr.copy(),
                    xray_luminosity=src.xray.copy(), x_e_box_prev=ti.x_e_box_prev.copy(), Tk_box=ti.Tk_box.copy(),
                    x_e_box=np.zeros_like(src.deltax), TS_box=np.zeros_like(ti.Tk_box),
                    sfr_histories=np.stack(ti.sfr_histories), xray_luminosity_histories=np.stack(ti.xray_histories))
        for k, v in arrs.items():
            setattr(hg, k, v.ctypes.data)
        hg.n_hist = nh
        ctx.call("rg_compute_Ts_host", C.byref(p), C.byref(snap), C.byref(hg), C.byref(out))
        res = {k: arrs[k] for k in ("x_e_box_prev", "x_e_box", "Tk_box", "TS_box")}
    ctx.close()
    res["stored_fcoll"] = sf
    return out, res


def run_oracle_ts(p, T, zz, idx, src, ti, precision="fp64"):
    U = wl.from_padded
    g = dict(deltax=U(src.deltax), stars=U(src.stars), x_e_box_prev=U(ti.x_e_box_prev).copy(),
             Tk_box=ti.Tk_box.copy(), sfr=U(src.sfr), xray_luminosity=U(src.xray),
             sfr_histories=[U(a) for a in ti.sfr_histories], xray_luminosity_histories=[U(a) for a in ti.xray_histories])
    out = to.compute_ts(oracle_params(p), T, zz, idx, ti.stored_fcoll, g, precision)
    return out, g


def check_parity(out, res, want, wg, n):
    U = wl.from_padded
    assert abs(out.collapse_fraction - want["collapse_fraction"]) <= 1e-9 * max(abs(want["collapse_fraction"]), 1e-300)
    for k in ("x_e_box_prev", "x_e_box"):
        got = U(res[k].reshape(n, n, -1))
        assert rel_l2(got, wg[k]) <= 1e-5, k
    for k in ("Tk_box", "TS_box"):
        assert rel_l2(res[k].reshape(n, n, n), wg[k]) <= 1e-5, k
    for k in SCALARS:
        w = want[k]
        assert abs(getattr(out, k) - w) <= 1e-5 * abs(w) + 1e-300, (k, getattr(out, k), w)


@pytest.mark.parametrize("n,box,ftype", [(32, 64.0, 1), (32, 64.0, 0), (32, 64.0, 2), (16, 32.0, 1), (64, 96.0, 1),
                                         (128, 128.0, 1)])
def test_compute_ts_matches_oracle(ts_tables, n, box, ftype):
    zz, idx, src, ti = ts_case(n, box, 15.0, 400 + n + ftype)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1, TsHeatingFilterType=ftype)
    out, res = run_gpu_ts(p, zz, idx, src, ti)
    want, wg = run_oracle_ts(p, ts_tables, zz, idx, src, ti)
    assert out.homogeneous == 0
    check_parity(out, res, want, wg, n)
    assert abs(out.x_e_ave - want["x_e_ave"]) <= 1e-9 * want["x_e_ave"]
    # ComputeTs stores this step's collapse fraction (ComputeTs.c:662)
    assert res["stored_fcoll"][idx] == out.collapse_fraction


def test_compute_ts_host_buffers_match_device(ts_tables):
    n, box = 32, 64.0
    zz, idx, src, ti = ts_case(n, box, 15.0, 77)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1)
    a, ra = run_gpu_ts(p, zz, idx, src, ti)
    b, rb = run_gpu_ts(p, zz, idx, src, ti, host=True)
    for k in ("x_e_box_prev", "x_e_box", "Tk_box", "TS_box"):
        assert np.array_equal(np.asarray(ra[k]).ravel(), np.asarray(rb[k]).ravel()), k
    for k in SCALARS:
        assert getattr(a, k) == getattr(b, k)


def test_compute_ts_homogeneous_branch(ts_tables):
    # zp >= ReionMaxHeatingRedshift: RECFAST x_e and T_K with adiabatic fluctuations
    n, box = 32, 64.0
    zz, idx, src, ti = ts_case(n, box, 32.0, 91, n_hist=1)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1)
    out, res = run_gpu_ts(p, zz, idx, src, ti)
    want, wg = run_oracle_ts(p, ts_tables, zz, idx, src, ti)
    assert out.homogeneous == 1
    for k in ("Tk_box", "TS_box"):
        assert rel_l2(res[k].reshape(n, n, n), wg[k]) <= 1e-6, k
    assert rel_l2(wl.from_padded(res["x_e_box"].reshape(n, n, -1)), wg["x_e_box"]) <= 1e-6
    for k in ("volume_ave_TS", "volume_ave_TK", "volume_ave_xe"):
        assert abs(getattr(out, k) - want[k]) <= 1e-6 * abs(want[k]), k


def test_compute_ts_no_light(ts_tables):
    # no stars: collapse fraction 0, the shell sums are skipped (NO_LIGHT, ComputeTs.c:736-744)
    n, box = 32, 64.0
    zz, idx, src, ti = ts_case(n, box, 15.0, 123)
    src.stars[:] = 0.0
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1)
    out, res = run_gpu_ts(p, zz, idx, src, ti)
    want, wg = run_oracle_ts(p, ts_tables, zz, idx, src, ti)
    assert out.collapse_fraction == 0.0
    assert out.volume_ave_J_alpha == 0.0 and out.volume_ave_Xheat == 0.0
    check_parity(out, res, want, wg, n)


def test_compute_ts_invalid_arguments():
    n = 32
    ctx = rg.Context(n)
    zz, idx = wl.snapshot_redshifts(15.0)
    snap = rg.snapshot(zz, idx, np.zeros(len(zz)))
    dg = DeviceGrids(n, spin=True)
    out = rg.rg_ts_scalars()
    lib = rg.load()
    p = rg.make_params(n, 64.0, Flag_IncludeSpinTemp=1, Flag_IncludeAGNXray=5)
    assert lib.rg_compute_Ts(ctx.h, C.byref(p), C.byref(snap), C.byref(dg.g), C.byref(out)) == rg.RG_EINVAL
    p = rg.make_params(n, 64.0, Flag_IncludeSpinTemp=1, TsHeatingFilterType=3)
    assert lib.rg_compute_Ts(ctx.h, C.byref(p), C.byref(snap), C.byref(dg.g), C.byref(out)) == rg.RG_EINVAL
    # shells reaching past the history slots provided
    p = rg.make_params(n, 64.0, Flag_IncludeSpinTemp=1)
    dg.g.n_hist = 0
    assert lib.rg_compute_Ts(ctx.h, C.byref(p), C.byref(snap), C.byref(dg.g), C.byref(out)) == rg.RG_EINVAL
    ctx.close()
    ctx = rg.Context(48)
    p = rg.make_params(48, 64.0, Flag_IncludeSpinTemp=1)
    dg = DeviceGrids(48, spin=True)
    assert lib.rg_compute_Ts(ctx.h, C.byref(p), C.byref(snap), C.byref(dg.g), C.byref(out)) == rg.RG_EUNSUPPORTED
    ctx.close()


def test_compute_ts_dense_snapshot_list(ts_tables):
    """400 snapshots before z = 15: the outer shells combine up to 14 history snapshots each
    (ComputeTs.c:420-458 loops over any number); those beyond four are combined in k-space before
    the shell's x pass.  Parity with the oracle as for the default list."""
    n, box = 32, 64.0
    zz, idx = wl.snapshot_redshifts(15.0, n_before=400)
    src = wl.make_sources(n, box, 700)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1)
    _, _, coef = rg.ts_tables(p, zz, idx, idx + 1, 2e-4, 1e-3, np.zeros(len(zz)), with_freq=False)
    assert (coef != 0).sum(axis=1).max() > 4
    n_hist = int(np.nonzero(np.any(coef != 0, axis=0))[0].max()) + 1
    ti = wl.make_ts_inputs(src, zz, idx, n_hist, 701)
    out, res = run_gpu_ts(p, zz, idx, src, ti)
    want, wg = run_oracle_ts(p, ts_tables, zz, idx, src, ti)
    assert out.homogeneous == 0
    check_parity(out, res, want, wg, n)
