"""Shared helpers for the tests: device grids from numpy, and oracle set-up."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

import rg_b200 as rg
import reion_oracle as ro
import tables


def oracle_params(p: rg.rg_params) -> ro.Params:
    """The oracle's Params from the ABI struct (same field names)."""
    kw = {}
    for f in ro.Params.__dataclass_fields__:
        if hasattr(p, f):
            kw[f] = getattr(p, f)
    return ro.Params(**kw)


_RECFAST = None


def install_recfast():
    global _RECFAST
    if _RECFAST is None:
        _RECFAST = tables.Recfast(tables.default_tables_dir())
        ro.set_recfast(_RECFAST.T)
    return _RECFAST


class DeviceGrids:
    """torch CUDA buffers for an rg_grids struct."""

    def __init__(self, n: int, spin: bool = False, bh: bool = False, rec: bool = False):
        import torch
        self.torch = torch
        self.n = n
        npad = n * n * 2 * (n // 2 + 1)
        nreal = n ** 3
        dev = "cuda:0"
        z = lambda k: torch.zeros(k, dtype=torch.float32, device=dev)
        self.t = {
            "deltax": z(npad), "stars": z(npad), "weighted_sfr": z(npad),
            "xH": z(nreal), "r_bubble": z(nreal), "z_at_ionization": torch.full((nreal,), -1.0, device=dev),
            "J_21_at_ionization": z(nreal), "temp_kinetic_all_gas": z(nreal), "delta_T": z(nreal),
        }
        if spin:
            self.t.update({"x_e_box": z(npad), "x_e_box_prev": z(npad), "Tk_box": z(nreal), "TS_box": z(nreal),
                           "sfr": z(npad), "xray_luminosity": z(npad)})
        if bh:
            self.t.update({"effective_bhm": z(npad), "effective_bhar": z(npad)})
        if rec:
            self.t.update({"Gamma12": z(nreal), "N_rec": z(npad), "residual_xH": z(nreal),
                           "clumping_factor": z(nreal), "t_resp": torch.full((nreal,), 1e30, device=dev)})
        self.g = rg.rg_grids()
        for k, v in self.t.items():
            setattr(self.g, k, v.data_ptr())

    def put(self, name: str, arr: np.ndarray):
        self.t[name].copy_(self.torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32).ravel()))

    def get(self, name: str, real: bool = True) -> np.ndarray:
        a = self.t[name].cpu().numpy()
        n = self.n
        if a.size == n ** 3:
            return a.reshape(n, n, n)
        return a.reshape(n, n, 2 * (n // 2 + 1))


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# Measured errors of the GPU outputs against FP64, collected by the configuration-level parity
# tests and written as a markdown table at the end of the session when RG_PARITY_TABLE names a
# file (tests/conftest.py).
PARITY_ROWS: list = []


def record(config: str, output: str, measure: str, value: float, gate: str):
    PARITY_ROWS.append((config, output, measure, float(value), gate))


GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name: str):
    """Outputs of the reference's own compiled step for a test case (tests/golden/make_golden.py),
    as ref_lib.run_step returns them (grids, and the box averages under "scalars"); None when the
    file is absent."""
    path = os.path.join(GOLDEN_DIR, name + ".npz")
    if not os.path.exists(path):
        return None
    with np.load(path) as f:
        d = {k: f[k] for k in f.files}
    scal = {"volume_weighted_global_xH": float(d.pop("mean_xH"))}
    if "mean_Tb" in d:
        scal["volume_ave_Tb"] = float(d.pop("mean_Tb"))
    d["scalars"] = scal
    return d
