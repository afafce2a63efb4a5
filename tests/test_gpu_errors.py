"""Status codes of the C ABI on a GPU: invalid arguments and unimplemented configurations return
RG_EINVAL / RG_EUNSUPPORTED with a message (the reference aborts the run instead), nothing is
launched for them, and the context stays usable afterwards.  The two bounded device waits (the
fused pass's wait for a plane's x pass, get_Ts's fixed point) are made to run out through
rg_debug_set_wait_limits: the calls return RG_ETIMEDOUT and the context keeps working."""

import ctypes as C

import numpy as np
import pytest

import rec_oracle as rco
import rg_b200 as rg
import workloads as wl
from helpers import DeviceGrids

pytestmark = pytest.mark.gpu


def status(ctx, name, *args):
    return getattr(ctx.lib, name)(ctx.h, *args)


def test_unsupported_grid_dim_creates_no_context():
    lib = rg.load()
    h = C.c_void_p()
    assert lib.rg_create(0, 40, C.byref(h)) == rg.RG_EUNSUPPORTED
    assert not h.value


def test_find_hii_rejections_leave_context_usable():
    n = 16
    src = wl.make_sources(n, 20.0, seed=1)
    dg = DeviceGrids(n)
    dg.put("deltax", src.deltax)
    dg.put("stars", src.stars)
    dg.put("weighted_sfr", src.sfr)
    zz, snap = wl.snapshot_redshifts(8.0)
    ctx = rg.Context(n)
    out = rg.rg_hii_scalars()

    def run(p, s=None, g=None):
        s = s or rg.snapshot(zz, snap)
        return status(ctx, "rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(g or dg.g), C.byref(out))

    base = dict(Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=20.0, ReionEfficiency=2000.0)
    assert run(rg.make_params(32, 20.0, **base)) == rg.RG_EINVAL                       # N differs
    assert "ReionGridDim" in ctx.lib.rg_last_error(ctx.h).decode()
    # recombinations: the tables first, then the recombination grids
    assert run(rg.make_params(n, 20.0, Flag_IncludeRecombinations=1, **base)) == rg.RG_EINVAL
    assert "rg_set_recombination_tables" in ctx.lib.rg_last_error(ctx.h).decode()
    t = rco.synthetic_tables(8, 6, 150)
    ctx.set_recombination_tables(t.knots, *(t.y[k].reshape(8, 6, 150) for k in range(3)))
    assert run(rg.make_params(n, 20.0, Flag_IncludeRecombinations=1, **base)) == rg.RG_EINVAL   # no N_rec
    bad_knots = t.knots.copy()
    bad_knots[5] = bad_knots[4]
    with pytest.raises(rg.RGError):
        ctx.set_recombination_tables(bad_knots, *(t.y[k].reshape(8, 6, 150) for k in range(3)))
    assert run(rg.make_params(n, 20.0, ReionFilterType=3, **base)) == rg.RG_EINVAL
    assert run(rg.make_params(n, 20.0, ReionDeltaRFactor=1.0, **base)) == rg.RG_EINVAL
    assert run(rg.make_params(n, 20.0, **base), s=rg.snapshot(zz, len(zz) + 3)) == rg.RG_EINVAL
    g = rg.rg_grids.from_buffer_copy(dg.g)
    g.xH = None
    assert run(rg.make_params(n, 20.0, **base), g=g) == rg.RG_EINVAL
    assert run(rg.make_params(n, 20.0, Flag_IncludeSpinTemp=1, **base)) == rg.RG_EINVAL   # no x_e_box
    # the context still works
    assert run(rg.make_params(n, 20.0, **base)) == rg.RG_OK
    assert 0.0 < out.volume_weighted_global_xH <= 1.0
    ctx.close()


def test_compute_ts_rejections():
    for n, kw, code in ((48, {}, rg.RG_EUNSUPPORTED), (16, {"Flag_IncludeAGNXray": 1}, rg.RG_EINVAL),   # no AGN grids
                        (16, {"Flag_IncludeAGNXray": 4}, rg.RG_EINVAL),
                        (16, {"TsNumFilterSteps": 0}, rg.RG_EINVAL), (16, {"TsHeatingFilterType": 5}, rg.RG_EINVAL)):
        dg = DeviceGrids(n, spin=True)
        p = rg.make_params(n, 32.0, Flag_IncludeSpinTemp=1, **kw)
        zz, snap = wl.snapshot_redshifts(15.0)
        s = rg.snapshot(zz, snap, np.zeros(len(zz)))
        ctx = rg.Context(n)
        out = rg.rg_ts_scalars()
        assert status(ctx, "rg_compute_Ts", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out)) == code, (n, kw)
        ctx.close()


def test_delta_T_and_power_spectrum_rejections():
    import torch
    n = 16
    dg = DeviceGrids(n, spin=True)
    zz, snap = wl.snapshot_redshifts(8.0)
    s = rg.snapshot(zz, snap)
    ctx = rg.Context(n)
    tb = C.c_double()
    p = rg.make_params(n, 20.0, Flag_IncludeSpinTemp=1, Flag_IncludePecVelsFor21cm=5)
    assert status(ctx, "rg_delta_T", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(tb)) == rg.RG_EINVAL
    p = rg.make_params(n, 20.0, Flag_IncludeSpinTemp=1, Flag_IncludePecVelsFor21cm=3)
    assert status(ctx, "rg_delta_T", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(tb)) == rg.RG_EINVAL  # no vel
    p = rg.make_params(n, 20.0)
    d = torch.rand(n ** 3, device="cuda") + 1.0
    k = (C.c_float * 2)()
    nb = C.c_int()
    rc = status(ctx, "rg_power_spectrum", C.byref(p), C.c_void_p(d.data_ptr()), 2, k, k, k, C.byref(nb))
    assert rc == rg.RG_EINVAL and nb.value == rg.power_spectrum_length(p)
    assert status(ctx, "rg_smooth_grid", C.c_double(-1.0), 8, C.c_void_p(d.data_ptr()),
                  C.c_void_p(d.data_ptr())) == rg.RG_EINVAL
    # still usable
    kk, ps, err = ctx.power_spectrum(p, d.data_ptr())
    assert len(kk) == nb.value
    ctx.close()


def _hii_case(n, box):
    src = wl.make_sources(n, box, seed=11)
    dg = DeviceGrids(n)
    dg.put("deltax", src.deltax)
    dg.put("stars", src.stars)
    dg.put("weighted_sfr", src.sfr)
    zz, snap = wl.snapshot_redshifts(8.0)
    p = rg.make_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=30.0, ReionEfficiency=3000.0)
    return dg, p, rg.snapshot(zz, snap)


def test_fused_pass_wait_time_out_is_reported_and_context_survives():
    """The fused x/y pass's only cross-block wait, made to run out: X items do not signal (a flag
    that nothing sets), each Y item gives up after 16 checks, the kernel completes and the call
    returns RG_ETIMEDOUT.  Restored limits give the same result as a fresh context, bit for bit."""
    n, box = 64, 64.0
    dg, p, s = _hii_case(n, box)
    ctx = rg.Context(n)
    out = rg.rg_hii_scalars()
    assert status(ctx, "rg_debug_set_wait_limits", 16, 0, -1) == rg.RG_OK
    rc = status(ctx, "rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out))
    assert rc == rg.RG_ETIMEDOUT
    assert "wait" in ctx.lib.rg_last_error(ctx.h).decode()
    assert status(ctx, "rg_debug_set_wait_limits", -1, 1, -1) == rg.RG_OK
    dg.t["z_at_ionization"].fill_(-1.0)
    dg.t["J_21_at_ionization"].zero_()
    dg.t["temp_kinetic_all_gas"].zero_()
    assert status(ctx, "rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out)) == rg.RG_OK
    got = {k: dg.get(k).copy() for k in ("xH", "z_at_ionization", "J_21_at_ionization", "temp_kinetic_all_gas")}
    ctx.close()
    fresh, _, _ = _hii_case(n, box)
    ctx2 = rg.Context(n)
    out2 = rg.rg_hii_scalars()
    assert status(ctx2, "rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(fresh.g), C.byref(out2)) == rg.RG_OK
    ctx2.close()
    for k, v in got.items():
        assert np.array_equal(v, fresh.get(k)), k
    assert out.volume_weighted_global_xH == out2.volume_weighted_global_xH


def test_get_ts_iteration_cap_is_reported_and_context_survives():
    """get_Ts capped at one fixed-point iteration: cells that need more make rg_compute_Ts return
    RG_ETIMEDOUT; with the default cap restored the same context gives the fresh-context result."""
    import torch
    n, box = 32, 64.0
    zz, idx = wl.snapshot_redshifts(15.0)
    src = wl.make_sources(n, box, 400)
    ti = wl.make_ts_inputs(src, zz, idx, idx + 1, 401)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1)

    def run(ctx):
        dg = DeviceGrids(n, spin=True)
        for k, v in (("deltax", src.deltax), ("stars", src.stars), ("sfr", src.sfr), ("xray_luminosity", src.xray),
                     ("x_e_box_prev", ti.x_e_box_prev), ("Tk_box", ti.Tk_box)):
            dg.put(k, v)
        hs = torch.from_numpy(np.stack(ti.sfr_histories).ravel()).cuda()
        hx = torch.from_numpy(np.stack(ti.xray_histories).ravel()).cuda()
        dg.g.sfr_histories, dg.g.xray_luminosity_histories = hs.data_ptr(), hx.data_ptr()
        dg.g.n_hist = len(ti.sfr_histories)
        s = rg.snapshot(zz, idx, ti.stored_fcoll.copy())
        out = rg.rg_ts_scalars()
        rc = status(ctx, "rg_compute_Ts", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out))
        return rc, {k: dg.get(k).copy() for k in ("x_e_box", "Tk_box", "TS_box")}

    ctx = rg.Context(n)
    assert status(ctx, "rg_debug_set_wait_limits", -1, 1, 1) == rg.RG_OK
    rc, _ = run(ctx)
    assert rc == rg.RG_ETIMEDOUT
    assert "get_Ts" in ctx.lib.rg_last_error(ctx.h).decode()
    assert status(ctx, "rg_debug_set_wait_limits", -1, 1, -1) == rg.RG_OK
    rc, got = run(ctx)
    assert rc == rg.RG_OK
    ctx.close()
    ctx2 = rg.Context(n)
    rc2, want = run(ctx2)
    ctx2.close()
    assert rc2 == rg.RG_OK
    for k in got:
        assert np.array_equal(got[k], want[k]), k
