"""GPU parity of the excursion-set step against the CPU oracle (through the C ABI).

Tolerances (floating point, FP32 kernels vs the FP64 oracle):
* filtered fields: relative L2 error <= 1e-5;
* mean xH within 1e-4; ionized-flag disagreements only in cells whose barrier
  margin |lhs/rhs - 1| is <= 1e-4 at some radius, and <= 0.01% of cells;
* partially ionized xH, J_21 and temperatures: per-cell relative error <= 1e-4
  outside the near-threshold cells.
"""

import ctypes as C

import numpy as np
import pytest

import reion_oracle as ro
import rg_b200 as rg
import workloads as wl
from helpers import DeviceGrids, install_recfast, oracle_params, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _recfast():
    install_recfast()


@pytest.mark.parametrize("n,box,ftype", [(n, b, f) for n, b in ((8, 8.0), (16, 20.0), (24, 24.0), (32, 32.0),
                                                                 (48, 48.0), (64, 64.0), (96, 96.0), (128, 100.0),
                                                                 (192, 190.0), (256, 250.0))
                                          for f in (-1, 0, 1, 2)] + [(384, 380.0, 0), (512, 500.0, 0)])
def test_filter_roundtrip_matches_fp64(n, box, ftype):
    import torch
    rng = np.random.default_rng(n * 7 + ftype)
    x = rng.standard_normal((n, n, n)).astype(np.float32)
    pad = wl.to_padded(x)
    d_in = torch.from_numpy(pad.ravel()).cuda()
    d_out = torch.zeros_like(d_in)
    ctx = rg.Context(n)
    p = rg.make_params(n, box)
    R = box / 7.3
    ctx.call("rg_debug_filter_roundtrip", C.byref(p), d_in.data_ptr(), d_out.data_ptr(), R, ftype)
    got = d_out.cpu().numpy().reshape(n, n, -1)[:, :, :n]
    spec = ro.forward(x.astype(np.float64), "fp64")
    if ftype >= 0:
        spec = spec * ro.window(n, box, R, ftype, "fp64")
    want = ro.inverse(spec, n)
    assert rel_l2(got, want) <= 1e-5
    ctx.close()


def run_gpu_hii(n, box, z, src, eff, ftype=0, mode=rg.RG_MODE_FUSED, state=None, **kw):
    dg = DeviceGrids(n)
    dg.put("deltax", src.deltax)
    dg.put("stars", src.stars)
    dg.put("weighted_sfr", src.sfr)
    if state is not None:
        dg.put("z_at_ionization", state.z_at_ionization)
        dg.put("J_21_at_ionization", state.J_21_at_ionization)
        dg.put("temp_kinetic_all_gas", state.temp_kinetic_all_gas)
    p = rg.make_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=50.0, ReionEfficiency=eff,
                       ReionFilterType=ftype, **kw)
    zz, snap = wl.snapshot_redshifts(z)
    s = rg.snapshot(zz, snap)
    ctx = rg.Context(n)
    ctx.call("rg_set_mode", mode)
    out = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out))
    ctx.close()
    return dg, out, p


def check_against_oracle(n, box, z, src, eff, ftype, dg, out, p, bh=None):
    op = oracle_params(p)
    st = ro.HIIState.fresh(n)
    kw = {} if bh is None else {"effective_bhm": bh[0], "effective_bhar": bh[1]}
    xH_o, rb_o, s_o, diag = ro.find_hii_bubbles(op, z, src.deltax, src.stars, src.sfr, st, "fp64",
                                                record_margins=True, **kw)
    xH = dg.get("xH")
    ion_g = xH < ro.REL_TOL
    ion_o = xH_o < ro.REL_TOL
    dis = ion_g != ion_o
    assert dis.mean() <= 1e-4, dis.mean()
    if dis.any():
        assert np.all(diag["min_margin"][dis] <= 1e-4), np.max(diag["min_margin"][dis])
    assert abs(out.volume_weighted_global_xH - s_o["volume_weighted_global_xH"]) <= 1e-4
    near = diag["min_margin"] <= 1e-4
    ok = ~near
    # partially ionized cells: xH = 1 - f prefactor is continuous in the filtered fields
    part = ok & ~ion_o
    if part.any():
        assert np.max(np.abs(xH[part] - xH_o[part])) <= 1e-4
    zin = dg.get("z_at_ionization")
    assert np.array_equal(zin[ok], st.z_at_ionization[ok])
    same_first = ok & (diag["first_cross"] >= 0)
    J = dg.get("J_21_at_ionization")
    if same_first.any():
        assert rel_l2(J[same_first], st.J_21_at_ionization[same_first]) <= 1e-4
    T = dg.get("temp_kinetic_all_gas")
    assert rel_l2(T[ok], st.temp_kinetic_all_gas[ok]) <= 1e-5
    assert np.all(dg.get("r_bubble") == 0)
    for k in ("volume_weighted_global_weighted_sfr", "volume_weighted_global_temp_kinetic_all_gas",
              "mass_weighted_global_temp_kinetic_all_gas"):
        assert getattr(out, k) == pytest.approx(s_o[k], rel=1e-5), k
    assert abs(out.mass_weighted_global_xH - s_o["mass_weighted_global_xH"]) <= 1e-4
    if bh is not None:
        assert out.volume_weighted_global_effective_bhar == pytest.approx(
            s_o["volume_weighted_global_effective_bhar"], rel=1e-5)
    assert out.n_radii == diag["n_radii"]
    return dis.sum()


@pytest.mark.parametrize("n,box", [(32, 32.0), (64, 64.0)])
def test_find_hii_bubbles_bh_feedback(n, box):
    """Flag_BHFeedback: effective_bhm is a fourth filtered field in the barrier test (and in J_21);
    effective_bhar enters the closing-pass average."""
    z = 8.0
    src = wl.make_sources(n, box, seed=31)
    rng = np.random.default_rng(32)
    bhm = (src.stars * 0.05 * rng.random(src.stars.shape)).astype(np.float32)
    bhar = (bhm * 1e-3).astype(np.float32)
    dg = DeviceGrids(n, bh=True)
    dg.put("deltax", src.deltax)
    dg.put("stars", src.stars)
    dg.put("weighted_sfr", src.sfr)
    dg.put("effective_bhm", bhm)
    dg.put("effective_bhar", bhar)
    p = rg.make_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=50.0, ReionEfficiency=3000.0,
                       Flag_BHFeedback=1)
    zz, snap = wl.snapshot_redshifts(z)
    s = rg.snapshot(zz, snap)
    ctx = rg.Context(n)
    out = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out))
    ctx.close()
    check_against_oracle(n, box, z, src, 3000.0, 0, dg, out, p, bh=(bhm, bhar))
    assert 0.0 < out.volume_weighted_global_xH < 1.0


@pytest.mark.parametrize("n,box,z,ftype", [(32, 32.0, 8.0, 0), (64, 64.0, 8.0, 0), (64, 64.0, 8.0, 1),
                                           (64, 64.0, 8.0, 2), (48, 40.0, 7.0, 0), (96, 96.0, 9.0, 0)])
def test_find_hii_bubbles_parity(n, box, z, ftype):
    src = wl.make_sources(n, box, seed=1809 + n)
    eff = 4000.0   # partially ionized box: exercises both branches of the barrier test
    dg, out, p = run_gpu_hii(n, box, z, src, eff, ftype)
    check_against_oracle(n, box, z, src, eff, ftype, dg, out, p)


def test_find_hii_bubbles_config_efficiency():
    """The benchmark configuration's literal ReionEfficiency = 1.0 (no cell ionizes)."""
    n, box, z = 64, 64.0, 8.0
    src = wl.make_sources(n, box, seed=1809)
    dg, out, p = run_gpu_hii(n, box, z, src, 1.0)
    check_against_oracle(n, box, z, src, 1.0, 0, dg, out, p)
    assert out.volume_weighted_global_xH > 0.99


def compare_modes(n, box, z, seed, eff=4000.0, ftype=0):
    """The fused mode (radius batches, windowed inverse passes, two-for-one c2r) against the plain
    mode (one FFT chain per grid per radius, every reference grid).  Both are FP32 evaluations of
    the same sums; where the compiler contracts them differently the rounding differs, so:
    ionised flags differ in <= 0.01% of cells, J_21 (but for <= 0.01% of cells whose first
    crossing radius differs), the temperatures and xH agree to 1e-5 relative L2, the box averages
    to 1e-5.  A single partly ionised cell may differ by more than
    its share of that: in cells without stars a float transform leaves a residue near the ABS_TOL
    clamp that the f_coll prefactor multiplies (up to 5e-4 at 512^3 between the two modes, each
    within the same bound of FP64), so the per-cell bound is 1e-3."""
    src = wl.make_sources(n, box, seed=seed)
    a, oa, _ = run_gpu_hii(n, box, z, src, eff, ftype, mode=rg.RG_MODE_FUSED)
    b, ob, _ = run_gpu_hii(n, box, z, src, eff, ftype, mode=rg.RG_MODE_PLAIN)
    ia, ib = a.get("xH") < ro.REL_TOL, b.get("xH") < ro.REL_TOL
    assert (ia != ib).mean() <= 1e-4
    same = ia == ib
    assert np.array_equal(a.get("z_at_ionization")[same], b.get("z_at_ionization")[same])
    for k in ("J_21_at_ionization", "temp_kinetic_all_gas", "xH"):
        av, bv = a.get(k)[same], b.get(k)[same]
        if k == "J_21_at_ionization":
            # J_21 is set at the radius where a cell first crosses the barrier, so a cell whose
            # crossing at a larger radius is a near-threshold decision in one form keeps the J_21
            # of a smaller radius in the other: at most 1e-4 of the cells may differ so, the rest
            # agree to 1e-5
            off = np.abs(av - bv) > 1e-4 * np.maximum(np.abs(bv), 1e-30)
            assert off.sum() <= 1e-4 * n ** 3
            av, bv = av[~off], bv[~off]
        assert rel_l2(av, bv) <= 1e-5, k
    assert np.max(np.abs(a.get("xH")[same] - b.get("xH")[same])) <= 1e-3
    da, db = oa.as_dict(), ob.as_dict()
    for k in da:
        assert da[k] == pytest.approx(db[k], rel=1e-5, abs=1e-12), k
    return oa


def test_plain_mode_matches_fused():
    compare_modes(64, 64.0, 8.0, 5)


def test_plain_mode_matches_fused_sharp_k():
    # the fused pass applies the sharp-k window as the step n2 <= cutoff, the plain pass reads
    # the window table: both are the same window
    compare_modes(128, 128.0, 8.0, 8, ftype=1)


@pytest.mark.parametrize("n,box", [(192, 190.0), (256, 250.0), (512, 500.0)])
def test_plain_mode_matches_fused_large(n, box):
    oa = compare_modes(n, box, 8.0, 6)
    assert 0.0 < oa.volume_weighted_global_xH < 1.0


@pytest.mark.parametrize("mode,spin", [(rg.RG_MODE_FUSED, False), (rg.RG_MODE_PLAIN, False), (rg.RG_MODE_FUSED, True)])
def test_host_entry_point_matches_device(mode, spin):
    """The host-buffer entry point (uploads on the copy stream, gated per stage) gives the device
    entry point's grids and scalars bit for bit."""
    n, box, z = 32, 32.0, 8.0
    src = wl.make_sources(n, box, seed=11)
    rng = np.random.default_rng(5)
    npad = n * n * 2 * (n // 2 + 1)
    xe = (rng.random(npad) * 0.05).astype(np.float32)
    tk = (20.0 + 10.0 * rng.random(n ** 3)).astype(np.float32)
    kw = {"Flag_IncludeSpinTemp": 1} if spin else {}
    p = rg.make_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=50.0, ReionEfficiency=4000.0, **kw)
    zz, snap = wl.snapshot_redshifts(z)
    s = rg.snapshot(zz, snap)
    dg = DeviceGrids(n, spin=spin)
    dg.put("deltax", src.deltax)
    dg.put("stars", src.stars)
    dg.put("weighted_sfr", src.sfr)
    if spin:
        dg.put("x_e_box", xe)
        dg.put("Tk_box", tk)
    ctx = rg.Context(n)
    ctx.call("rg_set_mode", mode)
    out = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out))
    ctx.close()
    h = {k: np.zeros(n ** 3, np.float32) for k in ("xH", "r_bubble", "J_21_at_ionization", "temp_kinetic_all_gas")}
    h["r_bubble"][:] = 7.0   # overwritten with zeros
    h["z_at_ionization"] = np.full(n ** 3, -1.0, np.float32)
    keep = {"deltax": np.ascontiguousarray(src.deltax), "stars": np.ascontiguousarray(src.stars),
            "weighted_sfr": np.ascontiguousarray(src.sfr)}
    if spin:
        keep.update(x_e_box=xe, Tk_box=tk)
    keep.update(h)
    g = rg.rg_grids()
    for k, v in keep.items():
        setattr(g, k, v.ctypes.data)
    ctx = rg.Context(n)
    ctx.call("rg_set_mode", mode)
    o2 = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles_host", C.byref(p), C.byref(s), C.byref(g), C.byref(o2))
    ctx.close()
    for k in ("xH", "z_at_ionization", "J_21_at_ionization", "temp_kinetic_all_gas", "r_bubble"):
        assert np.array_equal(h[k].reshape(n, n, n), dg.get(k)), k
    assert o2.as_dict() == out.as_dict()


def test_persistent_state_across_snapshots():
    """Two snapshots in a row: z_at_ionization keeps the earlier redshift of cells ionized first."""
    n, box = 32, 32.0
    src = wl.make_sources(n, box, seed=3)
    zz, _ = wl.snapshot_redshifts(8.0)
    z1, z2 = 9.0, 8.0
    st_o = ro.HIIState.fresh(n)
    dg, o1, p = run_gpu_hii(n, box, z1, src, 2000.0)
    op = oracle_params(p)
    ro.find_hii_bubbles(op, z1, src.deltax, src.stars, src.sfr, st_o, "fp64")
    st_g = ro.HIIState(dg.get("z_at_ionization").copy(), dg.get("J_21_at_ionization").copy(),
                       dg.get("temp_kinetic_all_gas").copy())
    dg2, o2, _ = run_gpu_hii(n, box, z2, src, 4000.0, state=st_g)
    op.ReionEfficiency = 4000.0
    xH_o, _, s_o, diag = ro.find_hii_bubbles(op, z2, src.deltax, src.stars, src.sfr, st_o, "fp64",
                                             record_margins=True)
    zin = dg2.get("z_at_ionization")
    assert np.any(zin == np.float32(z1)) and np.any(zin == np.float32(z2))
    agree = (zin == st_o.z_at_ionization).mean()
    assert agree > 0.999
    assert abs(o2.volume_weighted_global_xH - s_o["volume_weighted_global_xH"]) <= 1e-4


def test_invalid_parameters_rejected():
    n = 16
    ctx = rg.Context(n)
    dg = DeviceGrids(n)
    zz, snap = wl.snapshot_redshifts(8.0)
    s = rg.snapshot(zz, snap)
    out = rg.rg_hii_scalars()
    lib = rg.load()
    for kw, status in [({"ReionFilterType": 3}, rg.RG_EINVAL), ({"Flag_IncludeRecombinations": 1}, rg.RG_EINVAL),
                       ({"ReionGridDim": 32}, rg.RG_EINVAL), ({"ReionDeltaRFactor": 0.9}, rg.RG_EINVAL)]:
        p = rg.make_params(n, 16.0, **kw)
        assert lib.rg_find_HII_bubbles(ctx.h, C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out)) == status, kw
    p = rg.make_params(n, 16.0)
    bad = rg.snapshot(zz, len(zz) + 3)
    assert lib.rg_find_HII_bubbles(ctx.h, C.byref(p), C.byref(bad), C.byref(dg.g), C.byref(out)) == rg.RG_EINVAL
    p.TablesForXHeatingDir = b"/nonexistent"
    assert lib.rg_find_HII_bubbles(ctx.h, C.byref(p), C.byref(s), C.byref(dg.g), C.byref(out)) == rg.RG_ETABLE
    ctx.close()
