"""The golden outputs of the reference's own compiled step (tests/golden, written by
tests/golden/make_golden.py from oracle/_ref) on the CPU: the files equal a fresh run of the
reference's code where it is built, and the numpy oracle meets the pin gates against them (so the
oracle stays pinned where the reference cannot be built).  The GPU tests compare the library with
the same files (tests/test_gpu_configs.py)."""

import numpy as np
import pytest

import ref_lib
import reion_oracle as ro
import rg_b200 as rg
import workloads as wl
from helpers import golden, install_recfast, oracle_params, rel_l2


def c0_64_case(ftype):
    cfg = wl.CONFIGS["c0_64"]
    p = rg.make_params(cfg.n, cfg.box, Flag_EvolvingReionRBubbleMax=cfg.evolving_rmax,
                       ReionRBubbleMax=cfg.r_bubble_max, ReionRBubbleMin=cfg.r_bubble_min,
                       ReionDeltaRFactor=cfg.delta_r_factor, ReionFilterType=ftype, ReionEfficiency=4000.0,
                       ReionUVBFlag=cfg.uvb_flag, Flag_IncludeSpinTemp=0, TsHeatingFilterType=cfg.ts_filter_type,
                       TsNumFilterSteps=cfg.ts_steps)
    src = wl.make_sources(cfg.n, cfg.box, cfg.seed, cfg.source_scale)
    return cfg, p, src


def test_golden_files_equal_the_reference_code():
    if not ref_lib.available(False):
        pytest.skip("oracle/_ref is not built")
    cfg, p, src = c0_64_case(0)
    zz, snap = wl.snapshot_redshifts(cfg.z)
    ref = ref_lib.run_step(oracle_params(p), zz, snap, {"deltax": src.deltax, "stars": src.stars,
                                                         "weighted_sfr": src.sfr})
    g = golden("c0_64_f0")
    n = cfg.n
    for k in ("xH", "z_at_ionization", "temp_kinetic_all_gas"):
        assert np.array_equal(g[k], ref[k].reshape(n, n, n).astype(np.float32)), k
    assert g["scalars"]["volume_weighted_global_xH"] == ref["scalars"]["volume_weighted_global_xH"]


@pytest.mark.parametrize("ftype", [0, 1, 2])
def test_oracle_meets_the_pin_gates_against_golden_c0_64(ftype):
    install_recfast()
    cfg, p, src = c0_64_case(ftype)
    n = cfg.n
    g = golden(f"c0_64_f{ftype}")
    st = ro.HIIState.fresh(n)
    xH_o, _, s_o, diag = ro.find_hii_bubbles(oracle_params(p), cfg.z, src.deltax, src.stars, src.sfr, st, "fp64",
                                             record_margins=True)
    ok = diag["min_margin"] > 1e-4
    ion_g, ion_o = g["xH"] < ro.REL_TOL, xH_o < ro.REL_TOL
    assert np.array_equal(ion_g[ok], ion_o[ok])
    part = ok & ~ion_o
    assert np.max(np.abs(g["xH"][part] - xH_o[part])) <= 1e-4
    assert np.array_equal(g["z_at_ionization"][ok], st.z_at_ionization[ok])
    assert rel_l2(g["temp_kinetic_all_gas"][ok], st.temp_kinetic_all_gas[ok]) <= 1e-5
    assert abs(g["scalars"]["volume_weighted_global_xH"] - s_o["volume_weighted_global_xH"]) <= 1e-4
    assert 0.0 < g["scalars"]["volume_weighted_global_xH"] < 1.0


def test_chain_golden_file_equals_the_reference_code():
    if not ref_lib.available(False):
        pytest.skip("oracle/_ref is not built")
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "make_golden.py"))
    make_golden = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(make_golden)
    n, z, zz, snap, src, ti, p = make_golden.chain_inputs()
    inputs = dict(deltax=src.deltax, stars=src.stars, weighted_sfr=src.sfr, sfr=src.sfr, xray_luminosity=src.xray,
                  x_e_box_prev=ti.x_e_box_prev, Tk_box=ti.Tk_box, sfr_histories=np.stack(ti.sfr_histories),
                  xray_luminosity_histories=np.stack(ti.xray_histories))
    ref = ref_lib.run_step(oracle_params(p), zz, snap, inputs, stages=("ts", "hii", "dT"),
                           n_hist=len(ti.sfr_histories), stored_fcoll=ti.stored_fcoll,
                           outputs=("x_e_box", "Tk_box", "TS_box", "xH", "delta_T"))
    g = golden("chain_32")
    assert np.array_equal(g["x_e_box"], ref["x_e_box"].reshape(n, n, -1).astype(np.float32))
    for k in ("Tk_box", "TS_box", "xH", "delta_T"):
        assert np.array_equal(g[k], ref[k].reshape(n, n, n).astype(np.float32)), k
    assert g["scalars"]["volume_ave_Tb"] == ref["scalars"]["volume_ave_Tb"]
