"""ctypes binding of librg_b200.so (include/rg_b200.h) for tests and the benchmark.

The library is the product; this module only mirrors its C structs and loads it.
Loading fails loudly when the shared library has not been built.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librg_b200.so")
TABLES_DIR = os.path.join(HERE, "data", "21cmFAST-tables")

RG_OK, RG_EINVAL, RG_ENOMEM, RG_ECUDA, RG_EUNSUPPORTED, RG_ETABLE, RG_ENODEV, RG_ETIMEDOUT = range(8)
RG_MODE_FUSED, RG_MODE_PLAIN = 0, 1
RG_DFT_FP32, RG_DFT_TC_BF16X3 = 0, 1


class rg_params(C.Structure):
    _fields_ = [
        ("ReionGridDim", C.c_int),
        ("BoxSize", C.c_double),
        ("Hubble_h", C.c_double), ("OmegaM", C.c_double), ("OmegaK", C.c_double), ("OmegaLambda", C.c_double),
        ("OmegaR", C.c_double), ("BaryonFrac", C.c_double), ("wLambda", C.c_double),
        ("UnitLength_in_cm", C.c_double), ("UnitMass_in_g", C.c_double), ("UnitVelocity_in_cm_per_s", C.c_double),
        ("ReionDeltaRFactor", C.c_double), ("ReionRBubbleMax", C.c_double), ("ReionRBubbleMaxRecomb", C.c_double),
        ("ReionRBubbleMin", C.c_double),
        ("Flag_EvolvingReionRBubbleMax", C.c_int),
        ("ReionFilterType", C.c_int),
        ("ReionRtoMFilterType", C.c_int),
        ("ReionUVBFlag", C.c_int),
        ("ReionEfficiency", C.c_double), ("ReionNionPhotPerBary", C.c_double), ("ReionGammaHaloBias", C.c_double),
        ("ReionAlphaUV", C.c_double), ("ReionAlphaUVBH", C.c_double),
        ("ReionSfrTimescale", C.c_double), ("Y_He", C.c_double),
        ("Flag_IncludeSpinTemp", C.c_int), ("Flag_IncludeRecombinations", C.c_int), ("Flag_BHFeedback", C.c_int),
        ("TsHeatingFilterType", C.c_int), ("TsNumFilterSteps", C.c_int), ("Flag_IncludeAGNXray", C.c_int),
        ("ReionMaxHeatingRedshift", C.c_double),
        ("NuXrayThreshold", C.c_double), ("NuXraySoftCut", C.c_double), ("NuXrayMax", C.c_double),
        ("SpecIndexXrayGal", C.c_double),
        ("Flag_IncludePecVelsFor21cm", C.c_int),
        ("TablesForXHeatingDir", C.c_char_p),
        ("TreesID", C.c_int),
        ("Flag_TemperatureDependentRec", C.c_int),
        ("SpecIndexXrayAGNSoft", C.c_double), ("SpecIndexXrayAGNHard", C.c_double),
        ("UseMiniHalos", C.c_int), ("ReionEfficiencyIII", C.c_double), ("ReionNionPhotPerBaryIII", C.c_double),
    ]


_FP = C.POINTER(C.c_float)


class rg_grids(C.Structure):
    _fields_ = [
        ("deltax", C.c_void_p), ("stars", C.c_void_p), ("weighted_sfr", C.c_void_p),
        ("effective_bhm", C.c_void_p), ("effective_bhar", C.c_void_p),
        ("xH", C.c_void_p), ("r_bubble", C.c_void_p), ("z_at_ionization", C.c_void_p),
        ("J_21_at_ionization", C.c_void_p), ("temp_kinetic_all_gas", C.c_void_p),
        ("x_e_box_prev", C.c_void_p), ("x_e_box", C.c_void_p), ("Tk_box", C.c_void_p), ("TS_box", C.c_void_p),
        ("sfr", C.c_void_p), ("xray_luminosity", C.c_void_p),
        ("sfr_histories", C.c_void_p), ("xray_luminosity_histories", C.c_void_p),
        ("n_hist", C.c_int),
        ("delta_T", C.c_void_p),
        ("vel", C.c_void_p),
        ("Gamma12", C.c_void_p), ("N_rec", C.c_void_p), ("residual_xH", C.c_void_p),
        ("clumping_factor", C.c_void_p), ("t_resp", C.c_void_p),
        ("bh_xray_soft", C.c_void_p), ("bh_xray_hard", C.c_void_p), ("bh_xray_histories_soft", C.c_void_p),
        ("bh_xray_histories_hard", C.c_void_p),
        ("starsIII", C.c_void_p), ("weighted_sfrIII", C.c_void_p),
    ]


class rg_snapshot(C.Structure):
    _fields_ = [("snapshot", C.c_int), ("n_snapshots", C.c_int), ("ZZ", C.POINTER(C.c_double)),
                ("stored_fcoll", C.POINTER(C.c_double))]


class rg_hii_scalars(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "volume_weighted_global_xH", "volume_weighted_global_r_bubble", "volume_weighted_global_weighted_sfr",
        "volume_weighted_global_effective_bhar", "volume_weighted_global_temp_kinetic_all_gas",
        "mass_weighted_global_xH", "mass_weighted_global_r_bubble", "mass_weighted_global_temp_kinetic_all_gas")] + [
        ("n_radii", C.c_int)] + [(n, C.c_double) for n in (
        "volume_weighted_global_Gamma12", "volume_weighted_global_N_rec", "volume_weighted_global_residual_xH",
        "volume_weighted_global_clumping_factor", "mass_weighted_global_Gamma12", "mass_weighted_global_N_rec",
        "mass_weighted_global_residual_xH", "mass_weighted_global_clumping_factor",
        "volume_weighted_global_weighted_sfrIII")]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class rg_ts_scalars(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "volume_ave_J_alpha", "volume_ave_xalpha", "volume_ave_Xheat", "volume_ave_Xion",
        "volume_ave_TS", "volume_ave_TK", "volume_ave_xe", "collapse_fraction", "x_e_ave")] + [
        ("homogeneous", C.c_int), ("volume_ave_Xheat_AGN_soft", C.c_double), ("volume_ave_Xheat_AGN_hard", C.c_double)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class rg_kernel_stat(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_int), ("ms_total", C.c_double),
                ("alg_bytes_total", C.c_double)]


_P = C.POINTER
_SIGS = {
    "rg_profile_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "rg_profile_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, _P(C.c_int)]),
    "rg_params_default": (C.c_int, [_P(rg_params), C.c_int, C.c_double]),
    "rg_create": (C.c_int, [C.c_int, C.c_int, _P(C.c_void_p)]),
    "rg_destroy": (C.c_int, [C.c_void_p]),
    "rg_set_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "rg_set_radius_batch": (C.c_int, [C.c_void_p, C.c_int]),
    "rg_debug_set_wait_limits": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "rg_push_histories": (C.c_int, [C.c_void_p, _P(rg_params), _P(rg_grids)]),
    "rg_dft_y_pass": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "rg_find_HII_bubbles_batch": (C.c_int, [C.c_void_p, C.c_int, _P(rg_params), _P(rg_snapshot), _P(rg_grids),
                                            _P(rg_hii_scalars)]),
    "rg_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rg_last_error": (C.c_char_p, [C.c_void_p]),
    "rg_status_string": (C.c_char_p, [C.c_int]),
    "rg_alloc_grids": (C.c_int, [C.c_void_p, _P(rg_params), C.c_int, _P(rg_grids)]),
    "rg_init_reion_grids": (C.c_int, [C.c_void_p, _P(rg_params), _P(rg_grids)]),
    "rg_find_HII_bubbles": (C.c_int, [C.c_void_p, _P(rg_params), _P(rg_snapshot), _P(rg_grids), _P(rg_hii_scalars)]),
    "rg_compute_Ts": (C.c_int, [C.c_void_p, _P(rg_params), _P(rg_snapshot), _P(rg_grids), _P(rg_ts_scalars)]),
    "rg_delta_T": (C.c_int, [C.c_void_p, _P(rg_params), _P(rg_snapshot), _P(rg_grids), _P(C.c_double)]),
    "rg_find_HII_bubbles_host": (C.c_int, [C.c_void_p, _P(rg_params), _P(rg_snapshot), _P(rg_grids),
                                           _P(rg_hii_scalars)]),
    "rg_compute_Ts_host": (C.c_int, [C.c_void_p, _P(rg_params), _P(rg_snapshot), _P(rg_grids), _P(rg_ts_scalars)]),
    "rg_delta_T_host": (C.c_int, [C.c_void_p, _P(rg_params), _P(rg_snapshot), _P(rg_grids), _P(C.c_double)]),
    "rg_debug_filter_roundtrip": (C.c_int, [C.c_void_p, _P(rg_params), C.c_void_p, C.c_void_p, C.c_double, C.c_int]),
    "rg_reion_step_host": (C.c_int, [C.c_void_p, _P(rg_params), _P(rg_snapshot), _P(rg_grids), _P(rg_ts_scalars),
                                     _P(rg_hii_scalars), _P(C.c_double)]),
    "rg_power_spectrum_length": (C.c_int, [_P(rg_params), _P(C.c_int)]),
    "rg_power_spectrum": (C.c_int, [C.c_void_p, _P(rg_params), C.c_void_p, C.c_int, _P(C.c_float), _P(C.c_float),
                                    _P(C.c_float), _P(C.c_int)]),
    "rg_power_spectrum_host": (C.c_int, [C.c_void_p, _P(rg_params), C.c_void_p, C.c_int, _P(C.c_float),
                                         _P(C.c_float), _P(C.c_float), _P(C.c_int)]),
    "rg_smooth_grid": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_void_p]),
    "rg_set_recombination_tables": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                              C.c_void_p, C.c_void_p]),
    "rg_deposit_ngp": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                 C.POINTER(C.c_double), C.POINTER(C.c_void_p)]),
    "rg_radius_schedule": (C.c_int, [_P(rg_params), C.c_double, _P(C.c_double), C.c_int, _P(C.c_int)]),
    "rg_debug_ts_tables": (C.c_int, [_P(rg_params), _P(rg_snapshot), C.c_int, C.c_double, C.c_double, C.c_int,
                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    "rg_debug_ts_agn_tables": (C.c_int, [_P(rg_params), _P(rg_snapshot), C.c_int, C.c_double, C.c_double, C.c_int,
                                         C.c_void_p, C.c_void_p]),
    "rg_filter_roundtrip_noalloc": (C.c_int, [_P(rg_params), C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                              C.c_void_p, C.c_char_p, C.c_size_t]),
}

_lib = None


def load() -> C.CDLL:
    """Load librg_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class RGError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"status {status}: {msg}")
        self.status = status


def check(ctx, rc: int):
    if rc != RG_OK:
        lib = load()
        detail = lib.rg_last_error(ctx).decode() if ctx else ""
        raise RGError(rc, f"{lib.rg_status_string(rc).decode()} {detail}")


def make_params(n: int, box: float, **kw) -> rg_params:
    p = rg_params()
    check(None, load().rg_params_default(C.byref(p), n, box))
    p.TablesForXHeatingDir = TABLES_DIR.encode()
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def power_spectrum_length(p: rg_params) -> int:
    """PS_Length of Initialise_PowerSpectrum (host computation)."""
    n = C.c_int()
    check(None, load().rg_power_spectrum_length(C.byref(p), C.byref(n)))
    return n.value


def radius_schedule(p: rg_params, redshift: float, max_r: int = 4096):
    """The filter radii of find_HII_bubbles at this redshift (host computation)."""
    import numpy as np
    radii = np.zeros(max_r)
    n = C.c_int()
    check(None, load().rg_radius_schedule(C.byref(p), redshift, radii.ctypes.data_as(C.POINTER(C.c_double)), max_r,
                                          C.byref(n)))
    return radii[: n.value].copy()


def ts_tables(p: rg_params, zz, snap: int, n_hist: int, x_e_ave: float, collapse_fraction: float,
              stored_fcoll=None, with_freq: bool = True):
    """The host coefficient engine of the spin-temperature step (no device work): returns
    (shells[6][nS], freq[3][14][nS] or None, coef[nS][1 + n_hist])."""
    import numpy as np
    ns = p.TsNumFilterSteps
    shells = np.zeros((6, ns))
    freq = np.zeros((3, 14, ns)) if with_freq else None
    coef = np.zeros((ns, 1 + n_hist), np.float32)
    s = snapshot(zz, snap, stored_fcoll)
    check(None, load().rg_debug_ts_tables(C.byref(p), C.byref(s), n_hist, x_e_ave, collapse_fraction, ns,
                                          shells.ctypes.data, freq.ctypes.data if with_freq else None,
                                          coef.ctypes.data))
    return shells, freq, coef


def ts_agn_tables(p: rg_params, zz, snap: int, n_hist: int, x_e_ave: float, collapse_fraction: float,
                  stored_fcoll=None):
    """The AGN band tables [2][3][14][nS] and (const_zp GAL, AGN soft, AGN hard) of the host
    coefficient engine (no device work)."""
    import numpy as np
    ns = p.TsNumFilterSteps
    agn = np.zeros((2, 3, 14, ns))
    cz = np.zeros(3)
    s = snapshot(zz, snap, stored_fcoll)
    check(None, load().rg_debug_ts_agn_tables(C.byref(p), C.byref(s), n_hist, x_e_ave, collapse_fraction, ns,
                                              agn.ctypes.data, cz.ctypes.data))
    return agn, cz


def snapshot(zz, snap: int, stored_fcoll=None):
    import numpy as np
    zz = np.ascontiguousarray(zz, dtype=np.float64)
    s = rg_snapshot()
    s.snapshot = snap
    s.n_snapshots = len(zz)
    s.ZZ = zz.ctypes.data_as(C.POINTER(C.c_double))
    keep = [zz]
    if stored_fcoll is not None:
        sf = np.ascontiguousarray(stored_fcoll, dtype=np.float64)
        s.stored_fcoll = sf.ctypes.data_as(C.POINTER(C.c_double))
        keep.append(sf)
    s._keep = keep
    return s


class Context:
    """Owns an rg_context."""

    def __init__(self, n: int, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        check(None, self.lib.rg_create(device, n, C.byref(h)))
        self.h = h
        self.n = n

    def close(self):
        if self.h:
            self.lib.rg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def call(self, name, *args):
        check(self.h, getattr(self.lib, name)(self.h, *args))

    def find_hii_batch(self, ps, ss, gs):
        """rg_find_HII_bubbles_batch over the units (params, snapshots, grids); returns their
        rg_hii_scalars.  The snapshots' redshift arrays stay owned by the rg_snapshot objects."""
        n = len(ps)
        pa, sa, ga = (rg_params * n)(*ps), (rg_snapshot * n)(*ss), (rg_grids * n)(*gs)
        oa = (rg_hii_scalars * n)()
        self.call("rg_find_HII_bubbles_batch", n, pa, sa, ga, oa)
        return [rg_hii_scalars.from_buffer_copy(oa[i]) for i in range(n)]

    def power_spectrum(self, p: rg_params, delta_T_ptr: int, host: bool = False, max_bins: int = 64):
        """Compute_PS of delta_T (a device pointer, or a host pointer with host=True): returns
        (PS_k, PS_data, PS_error) as float32 arrays."""
        import numpy as np
        k, d, e = (C.c_float * max_bins)(), (C.c_float * max_bins)(), (C.c_float * max_bins)()
        n = C.c_int()
        self.call("rg_power_spectrum_host" if host else "rg_power_spectrum", C.byref(p), C.c_void_p(delta_T_ptr),
                  max_bins, k, d, e, C.byref(n))
        m = n.value
        return (np.frombuffer(k, np.float32)[:m].copy(), np.frombuffer(d, np.float32)[:m].copy(),
                np.frombuffer(e, np.float32)[:m].copy())

    def set_recombination_tables(self, lnGamma, RR, CF, RNH):
        """The MHR tables (RR and RNH as natural logs), each [nz][nt][ng] float64."""
        import numpy as np
        k = np.ascontiguousarray(lnGamma, np.float64)
        tabs = [np.ascontiguousarray(a, np.float64) for a in (RR, CF, RNH)]
        nz, nt, ng = tabs[0].shape
        self.call("rg_set_recombination_tables", k.ctypes.data, nz, nt, ng, *(a.ctypes.data for a in tabs))

    def deposit_ngp(self, box_size: float, n_gal: int, pos_ptr: int, values_ptr: int, grid_ptrs, divisors=None):
        """Nearest-grid-point deposit of n_gal galaxies (device positions [n_gal][3] and values
        [n_prop][n_gal]) into the padded device grids grid_ptrs (overwritten)."""
        n_prop = len(grid_ptrs)
        grids = (C.c_void_p * n_prop)(*grid_ptrs)
        div = (C.c_double * n_prop)(*divisors) if divisors is not None else None
        self.call("rg_deposit_ngp", box_size, n_gal, C.c_void_p(pos_ptr), n_prop, C.c_void_p(values_ptr),
                  div, grids)

    def profile(self, on: bool):
        self.call("rg_profile_enable", int(on))

    def kernel_stats(self):
        arr = (rg_kernel_stat * 64)()
        n = C.c_int()
        self.call("rg_profile_read", arr, 64, C.byref(n))
        return [{"name": arr[i].name.decode(), "launches": arr[i].launches, "ms_total": arr[i].ms_total,
                 "alg_bytes_total": arr[i].alg_bytes_total} for i in range(min(n.value, 64))]
