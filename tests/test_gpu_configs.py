"""GPU outputs on the benchmark configurations' own inputs, at their own sizes, against FP64.

The configurations are the workloads of ``workloads.CONFIGS`` (seeded generators):

* c0_64  -- find_HII_bubbles, 64^3, 64 Mpc/h, z = 8 (numpy FP64 oracle);
* c1_256 -- find_HII_bubbles, 256^3, 250 Mpc/h, z = 7, filters 0, 1, 2 (FP64 reference on the
  device, ``fp64_ref``, checked here against the numpy oracle at 64^3 and, for one case, at 256^3);
* c3_128 -- ComputeTs -> find_HII_bubbles -> delta_T at 128^3 with the configuration's uniform
  T_K = 12 K, x_e = 2e-4 and (1+z)^-3 SFR histories (numpy FP64 oracle for every stage);
* c4_512 -- the 512^3 benchmark step: ComputeTs on the GPU, then find_HII_bubbles (against
  ``fp64_ref`` fed the same x_e and T_K grids) and delta_T.

Each case runs at the configuration's literal ReionEfficiency (1.0: no cell ionises, every cell
takes the partial-xH branch) and at 4000 (a partly ionised box, both branches of the barrier
test).  Gates (north_star):

* filtered fields: relative L2 <= 1e-5 against FP64;
* |<xH>_gpu - <xH>_fp64| <= 1e-4;
* ionised-flag disagreements only in cells whose barrier margin |lhs/rhs - 1| is <= 1e-4 at some
  radius, and <= 0.01 % of cells; z_at_ionization equal outside those cells;
* partial xH, J_21 and temp_kinetic_all_gas within 1e-5 relative L2, outside the near-threshold
  cells (the largest per-cell partial-xH difference is reported);
* x_e, T_K, T_S: relative L2 <= 1e-5; delta_T relative L2 <= 2e-5 on the same T_S (5e-5 where
  the GPU and the oracle each carry their own T_S through the chain); <T_b> within 1e-4 relative.

Every measured error is recorded (helpers.record) and written as a table when RG_PARITY_TABLE
names a file.
"""

import ctypes as C

import numpy as np
import pytest

import fp64_ref
import reion_oracle as ro
import rg_b200 as rg
import ts_oracle as to
import workloads as wl
from helpers import DeviceGrids, golden, install_recfast, oracle_params, record, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _recfast():
    install_recfast()


def hii_params(cfg, eff, ftype=None, spin=0):
    return rg.make_params(cfg.n, cfg.box, Flag_EvolvingReionRBubbleMax=cfg.evolving_rmax,
                          ReionRBubbleMax=cfg.r_bubble_max, ReionRBubbleMin=cfg.r_bubble_min,
                          ReionDeltaRFactor=cfg.delta_r_factor,
                          ReionFilterType=cfg.filter_type if ftype is None else ftype,
                          ReionEfficiency=eff, ReionUVBFlag=cfg.uvb_flag, Flag_IncludeSpinTemp=spin,
                          TsHeatingFilterType=cfg.ts_filter_type, TsNumFilterSteps=cfg.ts_steps)


def gpu_hii(p, n, z, src, x_e_pad=None, tk=None, mode=rg.RG_MODE_FUSED):
    dg = DeviceGrids(n, spin=x_e_pad is not None)
    dg.put("deltax", src.deltax)
    dg.put("stars", src.stars)
    dg.put("weighted_sfr", src.sfr)
    if x_e_pad is not None:
        dg.put("x_e_box", x_e_pad)
        dg.put("Tk_box", tk)
    zz, snap = wl.snapshot_redshifts(z)
    s = rg.snapshot(zz, snap)
    ctx = rg.Context(n)
    ctx.call("rg_set_mode", mode)
    out = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out))
    ctx.close()
    res = {k: dg.get(k) for k in ("xH", "z_at_ionization", "J_21_at_ionization", "temp_kinetic_all_gas",
                                   "r_bubble")}
    del dg
    return res, out


def compare_hii(tag, res, out, want, n):
    """Gate and record the find_HII outputs against an FP64 result (xH, r_bubble, scalars, diag, state)."""
    xH_o, rb_o, s_o, diag, st = want
    xH = res["xH"]
    ion_g, ion_o = xH < ro.REL_TOL, xH_o < ro.REL_TOL
    dis = ion_g != ion_o
    near = diag["min_margin"] <= 1e-4
    ok = ~near
    n3 = float(n) ** 3
    record(tag, "ionised flag", "disagreeing cells / N^3", dis.sum() / n3, "<= 1e-4")
    record(tag, "ionised flag", "near-threshold share of disagreements",
           (near[dis].mean() if dis.any() else 1.0), "= 1")
    record(tag, "ionised flag", "cells within 1e-4 of the threshold / N^3", near.sum() / n3, "(reported)")
    if "fp32_fragile" in diag:
        record(tag, "ionised flag", "cells whose decision is fragile in float / N^3",
               diag["fp32_fragile"].sum() / n3, "(reported)")
    assert dis.mean() <= 1e-4
    if dis.any():
        assert np.all(near[dis]), np.max(diag["min_margin"][dis])
    dxh = abs(out.volume_weighted_global_xH - s_o["volume_weighted_global_xH"])
    record(tag, "<xH>", "|gpu - fp64|", dxh, "<= 1e-4")
    record(tag, "<xH>", "value (fp64)", s_o["volume_weighted_global_xH"], "(reported)")
    assert dxh <= 1e-4
    dmw = abs(out.mass_weighted_global_xH - s_o["mass_weighted_global_xH"])
    record(tag, "mass-weighted <xH>", "|gpu - fp64|", dmw, "<= 1e-4")
    assert dmw <= 1e-4
    part = ok & ~ion_o
    if part.any():
        # xH = 1 - f_coll prefactor of the never-ionised cells: continuous in the filtered
        # fields, so gated like them (relative L2); the largest single-cell difference is
        # reported, it sits where a float transform's absolute error is large next to the
        # cell's own stars or 1 + delta (any FP32 evaluation, the reference's included)
        e = rel_l2(xH[part], xH_o[part])
        record(tag, "xH (partial cells)", "relative L2", e, "<= 1e-5")
        assert e <= 1e-5
        d = np.abs(xH[part] - xH_o[part])
        record(tag, "xH (partial cells)", "max |gpu - fp64|", float(d.max()), "(reported)")
        record(tag, "xH (partial cells)", "cells with |gpu - fp64| > 1e-4 / N^3", float((d > 1e-4).sum()) / n3,
               "(reported)")
    record(tag, "xH", "relative L2", rel_l2(xH, xH_o), "(reported)")
    zin = res["z_at_ionization"]
    zd = int((zin[ok] != st.z_at_ionization[ok]).sum())
    record(tag, "z_at_ionization", "differing cells outside near-threshold", zd, "= 0")
    assert zd == 0
    fc = ok & (diag["first_cross"] >= 0)
    if fc.any():
        e = rel_l2(res["J_21_at_ionization"][fc], st.J_21_at_ionization[fc])
        record(tag, "J_21_at_ionization", "relative L2 (newly ionised)", e, "<= 1e-5")
        assert e <= 1e-5
    e = rel_l2(res["temp_kinetic_all_gas"][ok], st.temp_kinetic_all_gas[ok])
    record(tag, "temp_kinetic_all_gas", "relative L2", e, "<= 1e-5")
    assert e <= 1e-5
    rbd = int((res["r_bubble"] != rb_o).sum())
    record(tag, "r_bubble", "differing cells", rbd, "= 0")
    assert rbd == 0
    for k in ("volume_weighted_global_temp_kinetic_all_gas", "mass_weighted_global_temp_kinetic_all_gas",
              "volume_weighted_global_weighted_sfr"):
        e = abs(getattr(out, k) / s_o[k] - 1.0)
        record(tag, k, "relative", e, "<= 1e-5")
        assert e <= 1e-5, k
    assert out.n_radii == diag["n_radii"]


def fp64_hii(p, z, src, x_e=None, tk=None, numpy_oracle=False):
    op = oracle_params(p)
    st = ro.HIIState.fresh(p.ReionGridDim)
    if numpy_oracle:
        xH, rb, s, diag = ro.find_hii_bubbles(op, z, src.deltax, src.stars, src.sfr, st, "fp64", x_e_box=x_e,
                                              Tk_box=tk, record_margins=True)
    else:
        xH, rb, s, diag = fp64_ref.find_hii_fp64(op, z, src.deltax, src.stars, src.sfr, st, x_e_box=x_e, Tk_box=tk)
    return xH, rb, s, diag, st


# ---------------------------------------------------------------------------
# the device FP64 reference against the numpy oracle

@pytest.mark.parametrize("ftype,spin,eff", [(0, 0, 4000.0), (1, 0, 4000.0), (2, 0, 4000.0), (0, 1, 3000.0),
                                            (0, 0, 1.0)])
def test_fp64_ref_matches_numpy_oracle(ftype, spin, eff):
    n, box, z = 64, 64.0, 8.0
    src = wl.make_sources(n, box, 1809)
    x_e = tk = None
    if spin:
        rng = np.random.default_rng(3)
        x_e = wl.to_padded((2e-4 + 0.2 * rng.random((n, n, n))).astype(np.float32))
        tk = (12.0 + 5.0 * rng.random((n, n, n))).astype(np.float32)
    p = rg.make_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=50.0, ReionEfficiency=eff,
                       ReionFilterType=ftype, Flag_IncludeSpinTemp=spin)
    a = fp64_hii(p, z, src, x_e, tk, numpy_oracle=True)
    b = fp64_hii(p, z, src, x_e, tk)
    ok = np.minimum(a[3]["min_margin"], b[3]["min_margin"]) > 1e-9
    assert np.array_equal((a[0] < ro.REL_TOL)[ok], (b[0] < ro.REL_TOL)[ok])
    assert np.max(np.abs(a[0][ok] - b[0][ok])) <= 1e-6
    ma, mb = a[3]["min_margin"], b[3]["min_margin"]
    assert np.all(np.abs(ma - mb) <= 1e-9 * (1.0 + np.abs(ma)))
    assert np.array_equal(a[4].z_at_ionization[ok], b[4].z_at_ionization[ok])
    assert rel_l2(b[4].J_21_at_ionization[ok], a[4].J_21_at_ionization[ok]) <= 1e-6
    assert rel_l2(b[4].temp_kinetic_all_gas[ok], a[4].temp_kinetic_all_gas[ok]) <= 1e-6
    for k in ("volume_weighted_global_xH", "mass_weighted_global_xH"):
        assert abs(a[2][k] - b[2][k]) <= 1e-9


# ---------------------------------------------------------------------------
# c0_64 and c1_256: find_HII_bubbles on the configurations' own inputs

@pytest.mark.parametrize("eff", [1.0, 4000.0])
def test_c0_64_find_hii(eff):
    cfg = wl.CONFIGS["c0_64"]
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed, cfg.source_scale)
    p = hii_params(cfg, eff)
    res, out = gpu_hii(p, cfg.n, cfg.z, src)
    compare_hii(f"c0_64 eff {eff:g}", res, out, fp64_hii(p, cfg.z, src, numpy_oracle=True), cfg.n)


@pytest.mark.parametrize("ftype", [0, 1, 2])
@pytest.mark.parametrize("eff", [1.0, 4000.0])
def test_c1_256_find_hii(ftype, eff):
    cfg = wl.CONFIGS["c1_256"]
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed, cfg.source_scale)
    p = hii_params(cfg, eff, ftype)
    res, out = gpu_hii(p, cfg.n, cfg.z, src)
    compare_hii(f"c1_256 filter {ftype} eff {eff:g}", res, out, fp64_hii(p, cfg.z, src), cfg.n)
    if eff > 1:
        assert 0.0 < out.volume_weighted_global_xH < 1.0


def test_c1_256_find_hii_numpy_oracle():
    """One c1_256 case against the numpy oracle itself (the device FP64 reference is checked
    against it at 64^3 above; this ties the two at the configuration's size)."""
    cfg = wl.CONFIGS["c1_256"]
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed, cfg.source_scale)
    p = hii_params(cfg, 4000.0, 0)
    res, out = gpu_hii(p, cfg.n, cfg.z, src)
    compare_hii("c1_256 filter 0 eff 4000 (numpy oracle)", res, out, fp64_hii(p, cfg.z, src, numpy_oracle=True),
                cfg.n)


def filtered_field_errors(tag, cfg, src, ftype, which):
    """rg_debug_filter_roundtrip (r2c, /N^3, window, c2r) on the configuration's own grids at the
    first, a middle and the second-to-last radius, against the numpy FP64 transforms."""
    import torch
    n = cfg.n
    p = hii_params(cfg, 1.0, ftype)
    radii = [R for R, last in ro.radius_schedule(oracle_params(p), cfg.z) if not last]
    ctx = rg.Context(n)
    worst = 0.0
    for name in which:
        pad = getattr(src, name)
        d_in = torch.from_numpy(pad.ravel()).cuda()
        d_out = torch.zeros_like(d_in)
        spec = ro.forward(wl.from_padded(pad).astype(np.float64), "fp64")
        for R in (radii[0], radii[len(radii) // 2], radii[-1]):
            ctx.call("rg_debug_filter_roundtrip", C.byref(p), d_in.data_ptr(), d_out.data_ptr(), R, ftype)
            got = d_out.cpu().numpy().reshape(n, n, -1)[:, :, :n]
            want = ro.inverse(spec * ro.window(n, cfg.box, R, ftype, "fp64"), n)
            e = rel_l2(got, want)
            record(tag, f"filtered {name}", f"relative L2 at R = {R:.3g} Mpc/h", e, "<= 1e-5")
            worst = max(worst, e)
        del d_in, d_out, spec
    ctx.close()
    assert worst <= 1e-5


@pytest.mark.parametrize("ftype", [0, 1, 2])
def test_c1_256_filtered_fields(ftype):
    cfg = wl.CONFIGS["c1_256"]
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed, cfg.source_scale)
    filtered_field_errors(f"c1_256 filter {ftype}", cfg, src, ftype, ("deltax", "stars"))


# ---------------------------------------------------------------------------
# c3_128: ComputeTs -> find_HII_bubbles -> delta_T against the numpy oracle

def config_ts_setup(cfg):
    zz, snap = wl.snapshot_redshifts(cfg.z)
    op = oracle_params(hii_params(cfg, 1.0, spin=1))
    sh, _ = to.shells_and_sources(op, zz, snap, None, None, None, None, want_grids=False)
    n_hist = sh.max_slot + 1
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed, cfg.source_scale)
    ti = wl.make_config_ts_inputs(src, zz, snap, n_hist)
    return zz, snap, src, ti


def gpu_step(p, zz, snap, src, ti):
    """rg_compute_Ts -> rg_find_HII_bubbles -> rg_delta_T on device grids; returns the host copies."""
    import torch
    n = src.n
    dg = DeviceGrids(n, spin=True)
    for k, v in (("deltax", src.deltax), ("stars", src.stars), ("weighted_sfr", src.sfr), ("sfr", src.sfr),
                 ("xray_luminosity", src.xray), ("x_e_box_prev", ti.x_e_box_prev), ("Tk_box", ti.Tk_box)):
        dg.put(k, v)
    hs = torch.from_numpy(np.stack(ti.sfr_histories).ravel()).cuda()
    hx = torch.from_numpy(np.stack(ti.xray_histories).ravel()).cuda()
    dg.g.sfr_histories, dg.g.xray_luminosity_histories = hs.data_ptr(), hx.data_ptr()
    dg.g.n_hist = len(ti.sfr_histories)
    sf = ti.stored_fcoll.copy()
    s = rg.snapshot(zz, snap, sf)
    ts, hii, tb = rg.rg_ts_scalars(), rg.rg_hii_scalars(), C.c_double()
    ctx = rg.Context(n)
    ctx.call("rg_compute_Ts", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(ts))
    ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(hii))
    ctx.call("rg_delta_T", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(tb))
    ctx.close()
    res = {k: dg.get(k) for k in ("x_e_box_prev", "x_e_box", "Tk_box", "TS_box", "xH", "z_at_ionization",
                                   "J_21_at_ionization", "temp_kinetic_all_gas", "r_bubble", "delta_T")}
    del dg, hs, hx
    return res, ts, hii, tb.value


@pytest.mark.parametrize("eff", [1.0, 4000.0])
def test_c3_128_step(eff):
    cfg = wl.CONFIGS["c3_128"]
    n = cfg.n
    tag = f"c3_128 eff {eff:g}"
    zz, snap, src, ti = config_ts_setup(cfg)
    p = hii_params(cfg, eff, spin=1)
    res, ts, hii, tb = gpu_step(p, zz, snap, src, ti)
    U = wl.from_padded
    op = oracle_params(p)
    og = dict(deltax=U(src.deltax), stars=U(src.stars), x_e_box_prev=U(ti.x_e_box_prev).copy(),
              Tk_box=ti.Tk_box.copy(), sfr=U(src.sfr), xray_luminosity=U(src.xray),
              sfr_histories=[U(a) for a in ti.sfr_histories],
              xray_luminosity_histories=[U(a) for a in ti.xray_histories])
    want_ts = to.compute_ts(op, to.TsTables(), zz, snap, ti.stored_fcoll.copy(), og, "fp64")
    for k in ("x_e_box_prev", "x_e_box"):
        e = rel_l2(U(res[k]), og[k])
        record(tag, k, "relative L2", e, "<= 1e-5")
        assert e <= 1e-5, k
    for k in ("Tk_box", "TS_box"):
        e = rel_l2(res[k], og[k])
        record(tag, k, "relative L2", e, "<= 1e-5")
        assert e <= 1e-5, k
    for k in ("volume_ave_TS", "volume_ave_TK", "volume_ave_xe", "volume_ave_J_alpha", "volume_ave_Xheat"):
        e = abs(getattr(ts, k) / want_ts[k] - 1.0)
        record(tag, k, "relative", e, "<= 1e-5")
        assert e <= 1e-5, k
    # find_HII on the oracle's own x_e and T_K (its chain), the GPU's on its own
    want = fp64_hii(p, cfg.z, src, wl.to_padded(og["x_e_box"]), og["Tk_box"], numpy_oracle=True)
    compare_hii(tag, res, hii, want, n)
    dT_o, tb_o = ro.delta_T(op, cfg.z, want[0], src.deltax, og["TS_box"])
    near = want[3]["min_margin"] <= 1e-4
    # the two chains carry their own T_S (1e-5 apart): (1 - T_CMB / T_S) amplifies it at z = 15
    e = rel_l2(res["delta_T"][~near], dT_o[~near])
    record(tag, "delta_T", "relative L2 (outside near-threshold cells)", e, "<= 5e-5")
    assert e <= 5e-5
    e = abs(tb / tb_o - 1.0)
    record(tag, "<T_b>", "relative", e, "<= 1e-4")
    assert e <= 1e-4


# ---------------------------------------------------------------------------
# c4_512: the benchmark step at its size

@pytest.mark.parametrize("eff", [1.0, 4000.0])
def test_c4_512_step(eff):
    """The benchmark's 512^3 step on its own inputs: ComputeTs on the GPU (checked at 512^3 by
    the tiled test and here by its box averages' consistency), then find_HII_bubbles against the
    FP64 reference fed the same x_e and T_K grids, and delta_T against the FP64 formula on the
    FP64 xH and the GPU's T_S."""
    cfg = wl.CONFIGS["c4_512"]
    n = cfg.n
    tag = f"c4_512 eff {eff:g}"
    zz, snap, src, ti = config_ts_setup(cfg)
    p = hii_params(cfg, eff, spin=1)
    res, ts, hii, tb = gpu_step(p, zz, snap, src, ti)
    assert ts.homogeneous == 0 and np.all(np.isfinite(res["TS_box"]))
    x_e = res["x_e_box"]
    want = fp64_hii(p, cfg.z, src, x_e, res["Tk_box"])
    compare_hii(tag, res, hii, want, n)
    op = oracle_params(p)
    dT_o, tb_o = ro.delta_T(op, cfg.z, want[0], src.deltax, res["TS_box"])
    near = want[3]["min_margin"] <= 1e-4
    e = rel_l2(res["delta_T"][~near], dT_o[~near])
    record(tag, "delta_T", "relative L2 (outside near-threshold cells)", e, "<= 2e-5")
    assert e <= 2e-5
    e = abs(tb / tb_o - 1.0)
    record(tag, "<T_b>", "relative", e, "<= 1e-4")
    assert e <= 1e-4


def test_c4_512_filtered_fields():
    cfg = wl.CONFIGS["c4_512"]
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed, cfg.source_scale)
    filtered_field_errors("c4_512 filter 0", cfg, src, 0, ("deltax", "stars"))


# ---------------------------------------------------------------------------
# the GPU against the reference's own C code (oracle/_ref, built from the reference sources)

def _ref_lib():
    import ref_lib
    if not ref_lib.available(False):
        pytest.skip("oracle/_ref is not built")
    return ref_lib


@pytest.mark.parametrize("ftype", [0, 1, 2])
def test_c0_64_find_hii_against_reference_code(ftype):
    """c0_64's grid, box and redshift at an efficiency that ionises part of the box: the GPU's
    find_HII_bubbles against the reference's compiled _find_HII_bubbles on the same inputs (the
    reference computes in float, so the gates are the FP64 ones with the FP64 oracle's margins).
    The reference's outputs are its golden files (tests/golden), or a run of oracle/_ref."""
    cfg = wl.CONFIGS["c0_64"]
    n = cfg.n
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed, cfg.source_scale)
    p = hii_params(cfg, 4000.0, ftype)
    res, out = gpu_hii(p, n, cfg.z, src)
    zz, snap = wl.snapshot_redshifts(cfg.z)
    ref = golden(f"c0_64_f{ftype}")
    if ref is None:
        ref = _ref_lib().run_step(oracle_params(p), zz, snap, {"deltax": src.deltax, "stars": src.stars,
                                                                "weighted_sfr": src.sfr})
    diag = fp64_hii(p, cfg.z, src, numpy_oracle=True)[3]
    near = diag["min_margin"] <= 1e-4
    tag = f"c0_64 filter {ftype} eff 4000 vs reference code"
    xr = ref["xH"].reshape(n, n, n)
    dis = (res["xH"] < ro.REL_TOL) != (xr < ro.REL_TOL)
    record(tag, "ionised flag", "disagreeing cells / N^3", dis.mean(), "<= 1e-4, near-threshold only")
    assert dis.mean() <= 1e-4 and np.all(near[dis])
    part = ~near & (xr >= ro.REL_TOL)
    e = float(np.max(np.abs(res["xH"][part] - xr[part])))
    record(tag, "xH (partial cells)", "max |gpu - reference|", e, "<= 1e-4")
    assert e <= 1e-4
    zd = int((res["z_at_ionization"][~near] != ref["z_at_ionization"].reshape(n, n, n)[~near]).sum())
    record(tag, "z_at_ionization", "differing cells outside near-threshold", zd, "= 0")
    assert zd == 0
    e = rel_l2(res["temp_kinetic_all_gas"][~near], ref["temp_kinetic_all_gas"].reshape(n, n, n)[~near])
    record(tag, "temp_kinetic_all_gas", "relative L2", e, "<= 1e-5")
    assert e <= 1e-5
    dxh = abs(out.volume_weighted_global_xH - ref["scalars"]["volume_weighted_global_xH"])
    record(tag, "<xH>", "|gpu - reference|", dxh, "<= 1e-4")
    assert dxh <= 1e-4


def test_step_chain_against_reference_code():
    """ComputeTs -> find_HII_bubbles -> delta_T at 32^3 on the GPU against the reference's compiled
    _ComputeTs, _find_HII_bubbles and ComputeBrightnessTemperatureBox (its golden files, or a run
    of oracle/_ref)."""
    n, box, z = 32, 64.0, 13.0
    zz, snap = wl.snapshot_redshifts(z)
    src = wl.make_sources(n, box, 600)
    ti = wl.make_ts_inputs(src, zz, snap, snap + 1, 601)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=50.0,
                       ReionEfficiency=3000.0)
    res, ts, hii, tb = gpu_step(p, zz, snap, src, ti)
    inputs = dict(deltax=src.deltax, stars=src.stars, weighted_sfr=src.sfr, sfr=src.sfr, xray_luminosity=src.xray,
                  x_e_box_prev=ti.x_e_box_prev, Tk_box=ti.Tk_box, sfr_histories=np.stack(ti.sfr_histories),
                  xray_luminosity_histories=np.stack(ti.xray_histories))
    ref = golden("chain_32")
    if ref is None:
        ref = _ref_lib().run_step(oracle_params(p), zz, snap, inputs, stages=("ts", "hii", "dT"),
                                  n_hist=len(ti.sfr_histories), stored_fcoll=ti.stored_fcoll,
                                  outputs=("x_e_box", "Tk_box", "TS_box", "xH", "delta_T"))
    tag = "chain 32^3 vs reference code"
    U = wl.from_padded
    e = rel_l2(U(res["x_e_box"]), U(ref["x_e_box"].reshape(n, n, -1)))
    record(tag, "x_e_box", "relative L2", e, "<= 1e-5")
    assert e <= 1e-5
    for k in ("Tk_box", "TS_box"):
        e = rel_l2(res[k], ref[k].reshape(n, n, n))
        record(tag, k, "relative L2", e, "<= 1e-5")
        assert e <= 1e-5, k
    e = abs(tb / ref["scalars"]["volume_ave_Tb"] - 1.0)
    record(tag, "<T_b>", "relative", e, "<= 1e-4")
    assert e <= 1e-4
    dxh = abs(hii.volume_weighted_global_xH - ref["scalars"]["volume_weighted_global_xH"])
    record(tag, "<xH>", "|gpu - reference|", dxh, "<= 1e-4")
    assert dxh <= 1e-4
