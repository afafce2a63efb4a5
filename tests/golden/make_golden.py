"""Write the golden outputs of the reference's own compiled step (oracle/_ref) for the cases the
GPU tests compare against it, so those comparisons (and the oracle's pin) also run where the
reference cannot be built.  TEST INFRASTRUCTURE.

    python tests/golden/make_golden.py        # needs oracle/_ref (python oracle/build_ref.py)

Cases (inputs from the seeded workload generators, parameters as in tests/test_gpu_configs.py):

* ``c0_64_f{0,1,2}.npz``: _find_HII_bubbles on c0_64's grid, box and redshift at ReionEfficiency
  4000 with ReionFilterType 0, 1, 2: xH, z_at_ionization, temp_kinetic_all_gas and <xH>;
* ``chain_32.npz``: _ComputeTs -> _find_HII_bubbles -> ComputeBrightnessTemperatureBox at 32^3
  (z = 13, the spin temperature, every history slot): x_e_box, Tk_box, TS_box, xH, delta_T,
  <xH> and <T_b>.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "meraxes-devs_qyxnew_b200"), os.path.join(ROOT, "oracle"), os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

import ref_lib  # noqa: E402
import rg_b200 as rg  # noqa: E402
import workloads as wl  # noqa: E402
from helpers import oracle_params  # noqa: E402


def c0_64_params(ftype):
    cfg = wl.CONFIGS["c0_64"]
    return cfg, rg.make_params(cfg.n, cfg.box, Flag_EvolvingReionRBubbleMax=cfg.evolving_rmax,
                               ReionRBubbleMax=cfg.r_bubble_max, ReionRBubbleMin=cfg.r_bubble_min,
                               ReionDeltaRFactor=cfg.delta_r_factor, ReionFilterType=ftype,
                               ReionEfficiency=4000.0, ReionUVBFlag=cfg.uvb_flag, Flag_IncludeSpinTemp=0,
                               TsHeatingFilterType=cfg.ts_filter_type, TsNumFilterSteps=cfg.ts_steps)


def chain_inputs():
    n, box, z = 32, 64.0, 13.0
    zz, snap = wl.snapshot_redshifts(z)
    src = wl.make_sources(n, box, 600)
    ti = wl.make_ts_inputs(src, zz, snap, snap + 1, 601)
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=50.0,
                       ReionEfficiency=3000.0)
    return n, z, zz, snap, src, ti, p


def main():
    if not ref_lib.available(False):
        sys.exit("oracle/_ref is not built: python oracle/build_ref.py")
    for ftype in (0, 1, 2):
        cfg, p = c0_64_params(ftype)
        src = wl.make_sources(cfg.n, cfg.box, cfg.seed, cfg.source_scale)
        zz, snap = wl.snapshot_redshifts(cfg.z)
        ref = ref_lib.run_step(oracle_params(p), zz, snap, {"deltax": src.deltax, "stars": src.stars,
                                                             "weighted_sfr": src.sfr})
        n = cfg.n
        np.savez_compressed(os.path.join(HERE, f"c0_64_f{ftype}.npz"),
                            xH=ref["xH"].reshape(n, n, n).astype(np.float32),
                            z_at_ionization=ref["z_at_ionization"].reshape(n, n, n).astype(np.float32),
                            temp_kinetic_all_gas=ref["temp_kinetic_all_gas"].reshape(n, n, n).astype(np.float32),
                            mean_xH=ref["scalars"]["volume_weighted_global_xH"])
    n, z, zz, snap, src, ti, p = chain_inputs()
    inputs = dict(deltax=src.deltax, stars=src.stars, weighted_sfr=src.sfr, sfr=src.sfr, xray_luminosity=src.xray,
                  x_e_box_prev=ti.x_e_box_prev, Tk_box=ti.Tk_box, sfr_histories=np.stack(ti.sfr_histories),
                  xray_luminosity_histories=np.stack(ti.xray_histories))
    ref = ref_lib.run_step(oracle_params(p), zz, snap, inputs, stages=("ts", "hii", "dT"),
                           n_hist=len(ti.sfr_histories), stored_fcoll=ti.stored_fcoll,
                           outputs=("x_e_box", "Tk_box", "TS_box", "xH", "delta_T"))
    np.savez_compressed(os.path.join(HERE, "chain_32.npz"),
                        x_e_box=ref["x_e_box"].reshape(n, n, -1).astype(np.float32),
                        Tk_box=ref["Tk_box"].reshape(n, n, n).astype(np.float32),
                        TS_box=ref["TS_box"].reshape(n, n, n).astype(np.float32),
                        xH=ref["xH"].reshape(n, n, n).astype(np.float32),
                        delta_T=ref["delta_T"].reshape(n, n, n).astype(np.float32),
                        mean_xH=ref["scalars"]["volume_weighted_global_xH"],
                        mean_Tb=ref["scalars"]["volume_ave_Tb"])
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
