"""GPU parity of the AGN X-ray channels of the spin-temperature step (Flag_IncludeAGNXray 1 soft +
hard, 2 hard, 3 soft) against the CPU oracle, through the C ABI.  The AGN emissivity grids and
their histories are re-weighted per shell like the sfr ones, clamped at zero after filtering and
enter the heating, ionisation and Lyman-alpha sums with their own band tables and prefactors.

Tolerances as for the galaxy-only step: x_e, T_K and T_S relative L2 <= 1e-5 over the box; the
box averages, the two AGN heating averages included, relative error <= 1e-5."""

import ctypes as C

import numpy as np
import pytest

import rg_b200 as rg
import ts_oracle as to
import workloads as wl
from helpers import DeviceGrids, oracle_params, rel_l2

pytestmark = pytest.mark.gpu

SCALARS = ["volume_ave_J_alpha", "volume_ave_xalpha", "volume_ave_Xheat", "volume_ave_Xion", "volume_ave_TS",
           "volume_ave_TK", "volume_ave_xe"]
NAMES = ("soft", "hard")


@pytest.fixture(scope="module")
def ts_tables():
    return to.TsTables()


def agn_inputs(src, ti, seed):
    """Sparse AGN emissivity (1e10 L_sun per cell) of this snapshot and the history slots, scaled so
    their heating is a sizeable fraction of the galaxies'."""
    rng = np.random.default_rng(seed)

    def one(a):
        m = rng.random(a.shape) < 0.1
        return (a * 3e-4 * rng.lognormal(0.0, 1.0, a.shape) * m).astype(np.float32)

    out = {}
    for b in NAMES:
        out["bh_xray_" + b] = one(src.xray)
        out["bh_xray_histories_" + b] = [one(h) for h in ti.xray_histories]
    return out


def run_gpu(p, zz, idx, src, ti, agn, host=False):
    import torch
    n = src.n
    nh = len(ti.sfr_histories)
    sf = ti.stored_fcoll.copy()
    snap = rg.snapshot(zz, idx, sf)
    out = rg.rg_ts_scalars()
    ctx = rg.Context(n)
    keep = []
    if not host:
        dg = DeviceGrids(n, spin=True)
        for k, v in (("deltax", src.deltax), ("stars", src.stars), ("sfr", src.sfr), ("xray_luminosity", src.xray),
                     ("x_e_box_prev", ti.x_e_box_prev), ("Tk_box", ti.Tk_box)):
            dg.put(k, v)
        for name, arr in (("sfr_histories", np.stack(ti.sfr_histories)),
                          ("xray_luminosity_histories", np.stack(ti.xray_histories))):
            t = torch.from_numpy(arr.ravel()).cuda()
            keep.append(t)
            setattr(dg.g, name, t.data_ptr())
        for b in NAMES:
            for name, arr in (("bh_xray_" + b, agn["bh_xray_" + b]),
                              ("bh_xray_histories_" + b, np.stack(agn["bh_xray_histories_" + b]))):
                t = torch.from_numpy(np.ascontiguousarray(arr).ravel()).cuda()
                keep.append(t)
                setattr(dg.g, name, t.data_ptr())
        dg.g.n_hist = nh
        ctx.call("rg_compute_Ts", C.byref(p), C.byref(snap), C.byref(dg.g), C.byref(out))
        res = {k: dg.get(k) for k in ("x_e_box_prev", "x_e_box", "Tk_box", "TS_box")}
    else:
        hg = rg.rg_grids()
        arrs = dict(deltax=src.deltax.copy(), stars=src.stars.copy(), sfr=src.sfr.copy(),
                    xray_luminosity=src.xray.copy(), x_e_box_prev=ti.x_e_box_prev.copy(), Tk_box=ti.Tk_box.copy(),
                    x_e_box=np.zeros_like(src.deltax), TS_box=np.zeros_like(ti.Tk_box),
                    sfr_histories=np.stack(ti.sfr_histories), xray_luminosity_histories=np.stack(ti.xray_histories))
        for b in NAMES:
            arrs["bh_xray_" + b] = np.ascontiguousarray(agn["bh_xray_" + b])
            arrs["bh_xray_histories_" + b] = np.stack(agn["bh_xray_histories_" + b])
        for k, v in arrs.items():
            setattr(hg, k, v.ctypes.data)
        hg.n_hist = nh
        ctx.call("rg_compute_Ts_host", C.byref(p), C.byref(snap), C.byref(hg), C.byref(out))
        res = {k: arrs[k] for k in ("x_e_box_prev", "x_e_box", "Tk_box", "TS_box")}
    ctx.close()
    return out, res


def run_oracle(p, T, zz, idx, src, ti, agn):
    U = wl.from_padded
    g = dict(deltax=U(src.deltax), stars=U(src.stars), x_e_box_prev=U(ti.x_e_box_prev).copy(),
             Tk_box=ti.Tk_box.copy(), sfr=U(src.sfr), xray_luminosity=U(src.xray),
             sfr_histories=[U(a) for a in ti.sfr_histories], xray_luminosity_histories=[U(a) for a in ti.xray_histories])
    for b in NAMES:
        g["bh_xray_" + b] = U(agn["bh_xray_" + b])
        g["bh_xray_histories_" + b] = [U(a) for a in agn["bh_xray_histories_" + b]]
    return to.compute_ts(oracle_params(p), T, zz, idx, ti.stored_fcoll, g, "fp64"), g


@pytest.mark.parametrize("n,box,ftype,flag", [(32, 64.0, 1, 1), (32, 64.0, 1, 2), (32, 64.0, 1, 3), (32, 64.0, 0, 1),
                                              (64, 96.0, 2, 1)])
def test_agn_xray_matches_oracle(ts_tables, n, box, ftype, flag):
    zz, idx = wl.snapshot_redshifts(15.0)
    src = wl.make_sources(n, box, 600 + n + ftype)
    ti = wl.make_ts_inputs(src, zz, idx, idx + 1, 601 + n)
    agn = agn_inputs(src, ti, 602 + flag)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1, TsHeatingFilterType=ftype, Flag_IncludeAGNXray=flag)
    out, res = run_gpu(p, zz, idx, src, ti, agn)
    want, wg = run_oracle(p, ts_tables, zz, idx, src, ti, agn)
    assert out.homogeneous == 0
    U = wl.from_padded
    for k in ("x_e_box_prev", "x_e_box"):
        assert rel_l2(U(res[k].reshape(n, n, -1)), wg[k]) <= 1e-5, k
    for k in ("Tk_box", "TS_box"):
        assert rel_l2(res[k].reshape(n, n, n), wg[k]) <= 1e-5, k
    for k in SCALARS + ["volume_ave_Xheat_AGN_soft", "volume_ave_Xheat_AGN_hard"]:
        w = want[k]
        assert abs(getattr(out, k) - w) <= 1e-5 * abs(w) + 1e-300, (k, getattr(out, k), w)
    on = {1: (1, 1), 2: (0, 1), 3: (1, 0)}[flag]
    for b, name in enumerate(NAMES):
        assert (getattr(out, "volume_ave_Xheat_AGN_" + name) != 0) == bool(on[b])
    # the AGN terms move the heating by more than the tolerance: the channel is exercised
    p0 = rg.make_params(n, box, Flag_IncludeSpinTemp=1, TsHeatingFilterType=ftype)
    o0, _ = run_gpu(p0, zz, idx, src, ti, agn)
    assert abs(o0.volume_ave_Xheat - out.volume_ave_Xheat) > 1e-3 * abs(out.volume_ave_Xheat)


def test_agn_host_buffers_match_device(ts_tables):
    n, box = 32, 64.0
    zz, idx = wl.snapshot_redshifts(15.0)
    src = wl.make_sources(n, box, 700)
    ti = wl.make_ts_inputs(src, zz, idx, idx + 1, 701)
    agn = agn_inputs(src, ti, 702)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1, Flag_IncludeAGNXray=1)
    a, ra = run_gpu(p, zz, idx, src, ti, agn)
    b, rb = run_gpu(p, zz, idx, src, ti, agn, host=True)
    for k in ("x_e_box_prev", "x_e_box", "Tk_box", "TS_box"):
        assert np.array_equal(np.asarray(ra[k]).ravel(), np.asarray(rb[k]).ravel()), k
    assert a.as_dict() == b.as_dict()


def test_agn_missing_grids_rejected():
    n = 32
    zz, idx = wl.snapshot_redshifts(15.0)
    snap = rg.snapshot(zz, idx, np.zeros(len(zz)))
    dg = DeviceGrids(n, spin=True)
    out = rg.rg_ts_scalars()
    ctx = rg.Context(n)
    lib = rg.load()
    for flag, status in ((1, rg.RG_EINVAL), (4, rg.RG_EINVAL)):
        p = rg.make_params(n, 64.0, Flag_IncludeSpinTemp=1, Flag_IncludeAGNXray=flag)
        assert lib.rg_compute_Ts(ctx.h, C.byref(p), C.byref(snap), C.byref(dg.g), C.byref(out)) == status
    ctx.close()
