"""The oracle against the reference's own C code (oracle/_ref), on the CPU.

oracle/_ref is find_HII_bubbles.c, ComputeTs.c, XRayHeatingFunctions.c, BrightnessTemperature.c,
reionization.c and their helpers compiled unmodified from the reference sources over in-tree
stand-ins for FFTW, GSL, MPI, HDF5 and mlog (oracle/build_ref.py); its arithmetic is the
reference's float arithmetic.  These tests pin the numpy oracle, which every GPU parity test
checks against, to it:

* find_HII_bubbles (filters 0, 1, 2; with the spin-temperature grids; with BH feedback; the
  USE_MINI_HALOS build with Pop III sources): ionised flags equal outside cells whose FP64 barrier
  margin is within 1e-4, xH of partly ionised cells within 1e-4, z_at_ionization equal outside
  those cells, J_21 and temp_kinetic_all_gas within 1e-5 relative L2, box averages within 1e-6
  (1e-4 absolute for <xH>);
* ComputeTs (heating filters 0, 1, 2; the homogeneous branch; both AGN X-ray bands): x_e, T_K and
  T_S within 1e-5 relative L2, box averages within 1e-5, the collapse fraction within 1e-9;
* delta_T after the chain ComputeTs -> find_HII_bubbles: within 1e-5 relative L2 outside the
  near-threshold cells, <T_b> within 1e-5.

The oracle's "fp32" form, which restates the reference's float arithmetic, is compared too where
it is the closer statement (find_HII_bubbles).  Recombinations are not pinned this way: the
reference builds its MHR tables from an HDF5 file (init_MHR) that the stand-ins cannot read.
"""

import os
import sys

import numpy as np
import pytest

import reion_oracle as ro
import ts_oracle as to
import workloads as wl
from helpers import install_recfast, rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import ref_lib  # noqa: E402

REFERENCE = "/root/reference"


@pytest.fixture(scope="module", autouse=True)
def _reference_library():
    if not (ref_lib.available(False) and ref_lib.available(True)):
        if not os.path.isdir(os.path.join(REFERENCE, "src", "core")):
            pytest.skip("oracle/_ref is not built and the reference sources are not here")
        import build_ref
        for v in ("default", "mini"):
            build_ref.build(REFERENCE, v, False)
    install_recfast()


def params(n, box, **kw):
    base = dict(ReionGridDim=n, BoxSize=box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=50.0)
    base.update(kw)
    return ro.Params(**base)


def hii_inputs(src, x_e=None, tk=None, bh=None, mini=None):
    d = {"deltax": src.deltax, "stars": src.stars, "weighted_sfr": src.sfr}
    if x_e is not None:
        d.update(x_e_box=x_e, Tk_box=tk)
    if bh is not None:
        d.update(effective_bhm=bh[0], effective_bhar=bh[1])
    if mini is not None:
        d.update(starsIII=mini[0], weighted_sfrIII=mini[1])
    return d


def check_hii(n, ref, want, tol_partial=1e-4):
    xH_o, _, s_o, diag = want[:4]
    st = want[4]
    xr = ref["xH"].reshape(n, n, n)
    near = diag["min_margin"] <= 1e-4
    ok = ~near
    ion_r, ion_o = xr < ro.REL_TOL, xH_o < ro.REL_TOL
    assert np.array_equal(ion_r[ok], ion_o[ok])
    part = ok & ~ion_o
    if part.any():
        assert np.max(np.abs(xr[part] - xH_o[part])) <= tol_partial
    assert np.array_equal(ref["z_at_ionization"].reshape(n, n, n)[ok], st.z_at_ionization[ok])
    fc = ok & (diag["first_cross"] >= 0)
    if fc.any():
        assert rel_l2(ref["J_21_at_ionization"].reshape(n, n, n)[fc], st.J_21_at_ionization[fc]) <= 1e-5
    assert rel_l2(ref["temp_kinetic_all_gas"].reshape(n, n, n)[ok], st.temp_kinetic_all_gas[ok]) <= 1e-5
    sr = ref["scalars"]
    assert abs(sr["volume_weighted_global_xH"] - s_o["volume_weighted_global_xH"]) <= 1e-4
    assert abs(sr["mass_weighted_global_xH"] - s_o["mass_weighted_global_xH"]) <= 1e-4
    for k in ("volume_weighted_global_temp_kinetic_all_gas", "mass_weighted_global_temp_kinetic_all_gas",
              "volume_weighted_global_weighted_sfr"):
        assert sr[k] == pytest.approx(s_o[k], rel=1e-6), k
    return int((ion_r != ion_o).sum())


def oracle_hii(p, z, src, precision, x_e=None, tk=None, bh=None, mini=None):
    st = ro.HIIState.fresh(p.ReionGridDim)
    kw = {}
    if bh is not None:
        kw.update(effective_bhm=bh[0], effective_bhar=bh[1])
    if mini is not None:
        kw.update(starsIII=mini[0], weighted_sfrIII=mini[1])
    out = ro.find_hii_bubbles(p, z, src.deltax, src.stars, src.sfr, st, precision, x_e_box=x_e, Tk_box=tk,
                              record_margins=True, **kw)
    return (*out, st)


@pytest.mark.parametrize("ftype,eff", [(0, 4000.0), (1, 4000.0), (2, 4000.0), (0, 1.0)])
def test_find_hii_bubbles_matches_reference(ftype, eff):
    n, box, z = 32, 32.0, 8.0
    src = wl.make_sources(n, box, 1809 + ftype)
    p = params(n, box, ReionEfficiency=eff, ReionFilterType=ftype)
    zz, snap = wl.snapshot_redshifts(z)
    ref = ref_lib.run_step(p, zz, snap, hii_inputs(src))
    check_hii(n, ref, oracle_hii(p, z, src, "fp64"))
    # the oracle's float form restates the reference's arithmetic: flags agree everywhere
    w32 = oracle_hii(p, z, src, "fp32")
    assert check_hii(n, ref, w32) == 0
    if eff > 1:
        assert 0.0 < ref["scalars"]["volume_weighted_global_xH"] < 1.0


def test_find_hii_bubbles_matches_reference_64():
    """The benchmark's smallest configuration (c0_64's grid, box and redshift) at an efficiency that
    ionises part of the box."""
    cfg = wl.CONFIGS["c0_64"]
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed)
    p = params(cfg.n, cfg.box, ReionEfficiency=4000.0)
    zz, snap = wl.snapshot_redshifts(cfg.z)
    ref = ref_lib.run_step(p, zz, snap, hii_inputs(src))
    check_hii(cfg.n, ref, oracle_hii(p, cfg.z, src, "fp64"))


def test_find_hii_bubbles_spin_temperature_matches_reference():
    n, box, z = 32, 32.0, 8.0
    src = wl.make_sources(n, box, 77)
    rng = np.random.default_rng(78)
    x_e = wl.to_padded((2e-4 + 0.3 * rng.random((n, n, n))).astype(np.float32))
    tk = (12.0 + 40.0 * rng.random((n, n, n))).astype(np.float32)
    p = params(n, box, ReionEfficiency=3000.0, Flag_IncludeSpinTemp=1)
    zz, snap = wl.snapshot_redshifts(z)
    ref = ref_lib.run_step(p, zz, snap, hii_inputs(src, x_e, tk))
    check_hii(n, ref, oracle_hii(p, z, src, "fp64", x_e=x_e, tk=tk))


def test_find_hii_bubbles_bh_feedback_matches_reference():
    n, box, z = 32, 32.0, 8.0
    src = wl.make_sources(n, box, 31)
    rng = np.random.default_rng(32)
    bhm = (src.stars * 0.05 * rng.random(src.stars.shape)).astype(np.float32)
    bhar = (bhm * 1e-3).astype(np.float32)
    p = params(n, box, ReionEfficiency=3000.0, Flag_BHFeedback=1)
    zz, snap = wl.snapshot_redshifts(z)
    ref = ref_lib.run_step(p, zz, snap, hii_inputs(src, bh=(bhm, bhar)))
    want = oracle_hii(p, z, src, "fp64", bh=(bhm, bhar))
    check_hii(n, ref, want)
    assert ref["scalars"]["volume_weighted_global_effective_bhar"] == pytest.approx(
        want[2]["volume_weighted_global_effective_bhar"], rel=1e-6)


def test_find_hii_bubbles_pop3_matches_reference():
    """The USE_MINI_HALOS build: Pop III stars and SFR as more filtered grids of the barrier."""
    n, box, z = 32, 32.0, 8.0
    src = wl.make_sources(n, box, 41)
    rng = np.random.default_rng(42)
    s3 = (src.stars * 0.2 * rng.random(src.stars.shape)).astype(np.float32)
    w3 = (src.sfr * 0.2 * rng.random(src.sfr.shape)).astype(np.float32)
    p = params(n, box, ReionEfficiency=3000.0, UseMiniHalos=1, ReionEfficiencyIII=2000.0,
               ReionNionPhotPerBaryIII=6000.0)
    zz, snap = wl.snapshot_redshifts(z)
    ref = ref_lib.run_step(p, zz, snap, hii_inputs(src, mini=(s3, w3)))
    check_hii(n, ref, oracle_hii(p, z, src, "fp64", mini=(s3, w3)))


# ---------------------------------------------------------------------------
# ComputeTs

def ts_case(n, box, z, seed, n_hist=None):
    zz, idx = wl.snapshot_redshifts(z)
    src = wl.make_sources(n, box, seed)
    ti = wl.make_ts_inputs(src, zz, idx, idx + 1 if n_hist is None else n_hist, seed + 1)
    return zz, idx, src, ti


def ts_inputs(src, ti, agn=None):
    d = dict(deltax=src.deltax, stars=src.stars, sfr=src.sfr, xray_luminosity=src.xray,
             x_e_box_prev=ti.x_e_box_prev, Tk_box=ti.Tk_box, sfr_histories=np.stack(ti.sfr_histories),
             xray_luminosity_histories=np.stack(ti.xray_histories))
    if agn is not None:
        for b in ("soft", "hard"):
            d["BHXrayEmissivity_" + b] = agn["bh_xray_" + b]
            d["bh_xray_histories_" + b] = np.stack(agn["bh_xray_histories_" + b])
    return d


def oracle_ts(p, zz, idx, src, ti, agn=None):
    U = wl.from_padded
    g = dict(deltax=U(src.deltax), stars=U(src.stars), x_e_box_prev=U(ti.x_e_box_prev).copy(),
             Tk_box=ti.Tk_box.copy(), sfr=U(src.sfr), xray_luminosity=U(src.xray),
             sfr_histories=[U(a) for a in ti.sfr_histories], xray_luminosity_histories=[U(a) for a in ti.xray_histories])
    if agn is not None:
        for b in ("soft", "hard"):
            g["bh_xray_" + b] = U(agn["bh_xray_" + b])
            g["bh_xray_histories_" + b] = [U(a) for a in agn["bh_xray_histories_" + b]]
    out = to.compute_ts(p, to.TsTables(), zz, idx, ti.stored_fcoll.copy(), g, "fp64")
    return out, g


def check_ts(n, ref, want, g, idx, tol=1e-5):
    U = wl.from_padded
    for k in ("x_e_box", "x_e_box_prev"):
        assert rel_l2(U(ref[k].reshape(n, n, -1)), g[k]) <= tol, k
    for k in ("Tk_box", "TS_box"):
        assert rel_l2(ref[k].reshape(n, n, n), g[k]) <= tol, k
    sr = ref["scalars"]
    for k in ("volume_ave_TS", "volume_ave_TK", "volume_ave_xe", "volume_ave_J_alpha", "volume_ave_xalpha",
              "volume_ave_Xheat", "volume_ave_Xion"):
        assert sr[k] == pytest.approx(want[k], rel=tol, abs=1e-300), k
    assert ref["stored_fcoll"][idx] == pytest.approx(want["collapse_fraction"], rel=1e-9)


TS_OUT = ("x_e_box", "x_e_box_prev", "Tk_box", "TS_box")


@pytest.mark.parametrize("ftype", [0, 1, 2])
def test_compute_ts_matches_reference(ftype):
    n, box = 32, 64.0
    zz, idx, src, ti = ts_case(n, box, 15.0, 400 + ftype)
    p = params(n, box, Flag_IncludeSpinTemp=1, TsHeatingFilterType=ftype)
    ref = ref_lib.run_step(p, zz, idx, ts_inputs(src, ti), stages=("ts",), n_hist=len(ti.sfr_histories),
                           stored_fcoll=ti.stored_fcoll, outputs=TS_OUT)
    want, g = oracle_ts(p, zz, idx, src, ti)
    check_ts(n, ref, want, g, idx)


def test_compute_ts_homogeneous_branch_matches_reference():
    n, box = 32, 64.0
    zz, idx, src, ti = ts_case(n, box, 32.0, 91, n_hist=1)
    p = params(n, box, Flag_IncludeSpinTemp=1)
    ref = ref_lib.run_step(p, zz, idx, ts_inputs(src, ti), stages=("ts",), n_hist=1, stored_fcoll=ti.stored_fcoll,
                           outputs=TS_OUT)
    want, g = oracle_ts(p, zz, idx, src, ti)
    assert want["homogeneous"] == 1
    U = wl.from_padded
    for k in ("Tk_box", "TS_box"):
        assert rel_l2(ref[k].reshape(n, n, n), g[k]) <= 1e-6, k
    assert rel_l2(U(ref["x_e_box"].reshape(n, n, -1)), g["x_e_box"]) <= 1e-6


def test_compute_ts_agn_bands_match_reference():
    import test_gpu_ts_agn as ta
    n, box = 32, 64.0
    zz, idx, src, ti = ts_case(n, box, 15.0, 500)
    agn = ta.agn_inputs(src, ti, 501)
    p = params(n, box, Flag_IncludeSpinTemp=1, Flag_IncludeAGNXray=1)
    ref = ref_lib.run_step(p, zz, idx, ts_inputs(src, ti, agn), stages=("ts",), n_hist=len(ti.sfr_histories),
                           stored_fcoll=ti.stored_fcoll, outputs=TS_OUT)
    want, g = oracle_ts(p, zz, idx, src, ti, agn)
    check_ts(n, ref, want, g, idx)
    for b in ("soft", "hard"):
        k = "volume_ave_Xheat_AGN_" + b
        assert want[k] != 0.0
        assert ref["scalars"][k] == pytest.approx(want[k], rel=1e-5), k


# ---------------------------------------------------------------------------
# the chain ComputeTs -> find_HII_bubbles -> delta_T

def test_step_chain_matches_reference():
    n, box, z = 32, 64.0, 13.0
    zz, idx, src, ti = ts_case(n, box, z, 600)
    p = params(n, box, Flag_IncludeSpinTemp=1, ReionEfficiency=3000.0)
    inputs = ts_inputs(src, ti)
    inputs["weighted_sfr"] = src.sfr
    ref = ref_lib.run_step(p, zz, idx, inputs, stages=("ts", "hii", "dT"), n_hist=len(ti.sfr_histories),
                           stored_fcoll=ti.stored_fcoll,
                           outputs=TS_OUT + ("xH", "z_at_ionization", "J_21_at_ionization", "temp_kinetic_all_gas",
                                             "delta_T"))
    want_ts, g = oracle_ts(p, zz, idx, src, ti)
    check_ts(n, ref, want_ts, g, idx)
    want = oracle_hii(p, zz[idx], src, "fp64", x_e=wl.to_padded(g["x_e_box"]), tk=g["Tk_box"])
    check_hii(n, ref, want)
    dT, tb = ro.delta_T(p, zz[idx], want[0], src.deltax, g["TS_box"])
    near = want[3]["min_margin"] <= 1e-4
    assert rel_l2(ref["delta_T"].reshape(n, n, n)[~near], dT[~near]) <= 1e-5
    assert ref["scalars"]["volume_ave_Tb"] == pytest.approx(tb, rel=1e-5)


def test_compute_ts_dense_snapshot_list_matches_reference():
    """400 snapshots before z = 15, so that shells combine up to 14 history snapshots."""
    n, box = 32, 64.0
    zz, idx = wl.snapshot_redshifts(15.0, n_before=400)
    src = wl.make_sources(n, box, 700)
    p = params(n, box, Flag_IncludeSpinTemp=1)
    sh, _ = to.shells_and_sources(p, zz, idx, None, None, None, None, want_grids=False)
    ti = wl.make_ts_inputs(src, zz, idx, sh.max_slot + 1, 701)
    ref = ref_lib.run_step(p, zz, idx, ts_inputs(src, ti), stages=("ts",), n_hist=len(ti.sfr_histories),
                           stored_fcoll=ti.stored_fcoll, outputs=TS_OUT)
    want, g = oracle_ts(p, zz, idx, src, ti)
    check_ts(n, ref, want, g, idx)
