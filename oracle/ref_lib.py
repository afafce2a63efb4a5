"""The reference's own reionization step, built by oracle/build_ref.py -- TEST INFRASTRUCTURE ONLY.

``run_step`` drives libmeraxes_ref.so (or libmeraxes_ref_mini.so for a USE_MINI_HALOS build):
parameters by name, Meraxes' start-up for one rank (units, redshifts, the reference's own
assign_slabs / malloc_reionization_grids / init_reion_grids), the inputs copied into
run_globals.reion_grids, then the reference's _ComputeTs, _find_HII_bubbles and
ComputeBrightnessTemperatureBox in the order of src/core/dracarys.c:383-391.  The library keeps
Meraxes' process-wide state (run_globals, the static spline caches), so every call runs in a
fresh process started with ``spawn``.

Its FFTs and GSL routines are the in-tree stand-ins of oracle/ref_shim (double-precision FFT
rounded to float per transform; QAG-61, Brent and the natural cubic spline restated from GSL);
everything else is the reference's compiled C.
"""

from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import multiprocessing as mp
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "_ref")
TABLES_DIR = os.path.join(os.path.dirname(HERE), "meraxes-devs_qyxnew_b200", "data", "21cmFAST-tables")

# ro.Params fields that are not run_globals.params entries: units go to rg_ref_setup, the
# mini-halo switch selects the library build
_NOT_PARAMS = {"UnitLength_in_cm", "UnitMass_in_g", "UnitVelocity_in_cm_per_s", "UseMiniHalos"}

HII_SCALARS = ["volume_weighted_global_xH", "volume_weighted_global_r_bubble", "volume_weighted_global_weighted_sfr",
               "volume_weighted_global_effective_bhar", "volume_weighted_global_temp_kinetic_all_gas",
               "mass_weighted_global_xH", "mass_weighted_global_r_bubble",
               "mass_weighted_global_temp_kinetic_all_gas"]
TS_SCALARS = ["volume_ave_J_alpha", "volume_ave_xalpha", "volume_ave_Xheat", "volume_ave_Xion", "volume_ave_TS",
              "volume_ave_TK", "volume_ave_xe", "volume_ave_Xheat_AGN_soft", "volume_ave_Xheat_AGN_hard"]


def library_path(mini: bool = False) -> str:
    return os.path.join(LIB_DIR, "libmeraxes_ref_mini.so" if mini else "libmeraxes_ref.so")


def available(mini: bool = False) -> bool:
    return os.path.exists(library_path(mini))


def _load(mini: bool):
    lib = C.CDLL(library_path(mini))
    lib.rg_ref_set_param.argtypes = [C.c_char_p, C.c_double]
    lib.rg_ref_set_string.argtypes = [C.c_char_p, C.c_char_p]
    lib.rg_ref_setup.argtypes = [C.c_int, C.POINTER(C.c_double), C.c_int, C.c_double, C.c_double, C.c_double]
    lib.rg_ref_grid.argtypes = [C.c_char_p]
    lib.rg_ref_grid.restype = C.POINTER(C.c_float)
    lib.rg_ref_scalar.argtypes = [C.c_char_p, C.POINTER(C.c_double)]
    lib.rg_ref_stored_fcoll.restype = C.POINTER(C.c_double)
    for f in ("rg_ref_find_HII_bubbles", "rg_ref_compute_Ts", "rg_ref_delta_T"):
        getattr(lib, f).argtypes = [C.c_int]
    return lib


def _grid(lib, name: str, count: int) -> np.ndarray:
    ptr = lib.rg_ref_grid(name.encode())
    if not ptr:
        raise KeyError(f"grid {name} is not allocated in this configuration")
    return np.ctypeslib.as_array(ptr, shape=(count,))


def _run(params: dict, zz, snap: int, n_hist: int, inputs: dict, stages, stored_fcoll, outputs):
    mini = bool(params.get("UseMiniHalos", 0))
    lib = _load(mini)
    for k, v in params.items():
        if k in _NOT_PARAMS:
            continue
        if lib.rg_ref_set_param(k.encode(), float(v)) != 0:
            raise KeyError(f"run_globals.params has no entry {k} in the driver's table")
    lib.rg_ref_set_param(b"Flag_PatchyReion", 1.0)
    if "dT" in stages:
        lib.rg_ref_set_param(b"Flag_Compute21cmBrightTemp", 1.0)   # allocates delta_T
    lib.rg_ref_set_string(b"TablesForXHeatingDir", (TABLES_DIR + "/").encode())
    zz = np.ascontiguousarray(zz, np.float64)
    rc = lib.rg_ref_setup(len(zz), zz.ctypes.data_as(C.POINTER(C.c_double)), n_hist,
                          params.get("UnitLength_in_cm", 3.08568e24), params.get("UnitMass_in_g", 1.989e43),
                          params.get("UnitVelocity_in_cm_per_s", 1.0e5))
    if rc != 0:
        raise RuntimeError(f"reference set-up failed ({rc})")
    n = int(params["ReionGridDim"])
    npad, nreal = n * n * 2 * (n // 2 + 1), n ** 3
    sizes = {}
    for name, arr in inputs.items():
        a = np.ascontiguousarray(arr, np.float32).ravel()
        _grid(lib, name, a.size)[:] = a
        sizes[name] = a.size
    if stored_fcoll is not None:
        np.ctypeslib.as_array(lib.rg_ref_stored_fcoll(), shape=(len(zz),))[:] = stored_fcoll
    for st in stages:
        fn = {"ts": lib.rg_ref_compute_Ts, "hii": lib.rg_ref_find_HII_bubbles, "dT": lib.rg_ref_delta_T}[st]
        rc = fn(snap)
        if rc != 0:
            raise RuntimeError(f"reference stage {st} aborted ({rc})")
    out = {}
    for name in outputs:
        count = sizes.get(name) or (npad if name in ("x_e_box", "x_e_box_prev", "N_rec", "deltax") else nreal)
        out[name] = _grid(lib, name, count).copy()
    sc = {}
    for name in HII_SCALARS + TS_SCALARS + ["volume_ave_Tb"]:
        v = C.c_double()
        if lib.rg_ref_scalar(name.encode(), C.byref(v)) == 0:
            sc[name] = v.value
    out["scalars"] = sc
    out["stored_fcoll"] = np.ctypeslib.as_array(lib.rg_ref_stored_fcoll(), shape=(len(zz),)).copy()
    return out


def run_step(params, zz, snap: int, inputs: dict, stages=("hii",), n_hist: int = 1, stored_fcoll=None,
             outputs=("xH", "r_bubble", "z_at_ionization", "J_21_at_ionization", "temp_kinetic_all_gas")):
    """Run the reference's stages ("ts", "hii", "dT", in that order) on one snapshot in a fresh
    process.  ``params``: an oracle Params (or a dict of run_globals.params names); ``inputs``:
    reion_grids arrays by name in the reference's layouts (padded source grids, real state grids,
    histories as [n_hist] x padded).  Returns the named grids (flat, the reference's layout), the
    box averages under "scalars" and stored_fcoll."""
    if not isinstance(params, dict):
        import dataclasses
        params = dataclasses.asdict(params)
    # a worker that dies (the reference aborted outside a guarded call) raises BrokenProcessPool
    with cf.ProcessPoolExecutor(max_workers=1, mp_context=mp.get_context("spawn")) as ex:
        fut = ex.submit(_run, params, np.asarray(zz, np.float64), snap, n_hist, dict(inputs), tuple(stages),
                        None if stored_fcoll is None else np.asarray(stored_fcoll, np.float64), tuple(outputs))
        return fut.result()
