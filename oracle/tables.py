"""Readers for the 21cmFAST data tables -- TEST INFRASTRUCTURE ONLY (the oracle's side).

Restates the file parsing of T_RECFAST / xion_RECFAST
(src/core/XRayHeatingFunctions.c:134-252), kappa_10_elec / kappa_10_pH
(:1827-1966), spectral_emissivity (:643-728) and initialize_interp_arrays
(:861-960).  GSL's ``gsl_interp_cspline`` is a natural cubic spline; the oracle
uses ``scipy.interpolate.CubicSpline(bc_type="natural")`` for it.
"""

from __future__ import annotations

import os

import numpy as np
from scipy.interpolate import CubicSpline

RECFAST_NPTS = 501
KAPPA_10_elec_NPTS = 20
KAPPA_10_pH_NPTS = 17
NSPEC_MAX = 23
x_int_NXHII = 14
x_int_NENERGY = 258

# x_int_XHII (XRayHeatingFunctions.c:878-891), stored as float in the C
X_INT_XHII = np.array([1.0e-4, 2.318e-4, 4.677e-4, 1.0e-3, 2.318e-3, 4.677e-3, 1.0e-2, 2.318e-2,
                       4.677e-2, 1.0e-1, 0.5, 0.9, 0.99, 0.999], dtype=np.float32)


def default_tables_dir() -> str:
    here = os.path.dirname(os.path.abspath(__file__))
    return os.path.join(os.path.dirname(here), "meraxes-devs_qyxnew_b200", "data", "21cmFAST-tables")


class Recfast:
    """Natural cubic splines of T_K(z) and x_e(z) from recfast_LCDM.dat."""

    def __init__(self, tables_dir: str):
        rows = np.loadtxt(os.path.join(tables_dir, "recfast_LCDM.dat"), dtype=np.float64, max_rows=RECFAST_NPTS)
        rows = rows.astype(np.float32).astype(np.float64)       # read with %f / %E into floats
        rows = rows[::-1]                                      # stored reversed: zt[i] ascending
        self.z = rows[:, 0]
        self.xion = rows[:, 1]
        self.tk = rows[:, 3]
        self._t = CubicSpline(self.z, self.tk, bc_type="natural")
        self._x = CubicSpline(self.z, self.xion, bc_type="natural")

    def T(self, z: float) -> float:
        z = float(np.float32(z))
        if z > self.z[-1]:
            return -1.0
        return float(self._t(z))

    def xe(self, z: float) -> float:
        z = float(np.float32(z))
        if z > self.z[-1]:
            return -1.0
        return float(self._x(z))


def read_kappa(tables_dir: str, name: str, npts: int) -> tuple[np.ndarray, np.ndarray]:
    d = np.loadtxt(os.path.join(tables_dir, name), dtype=np.float64, max_rows=npts).astype(np.float32).astype(np.float64)
    return np.log(d[:, 0]), np.log(d[:, 1])


def read_stellar_spectra(tables_dir: str):
    d = np.loadtxt(os.path.join(tables_dir, "stellar_spectra.dat"), dtype=np.float64, max_rows=NSPEC_MAX - 1)
    return d.astype(np.float32)


def read_x_int_tables(tables_dir: str):
    """x_int_Energy[258], and [14][258] fheat, n_Lya, nion_HI, nion_HeI, nion_HeII (float)."""
    energy = None
    fheat = np.zeros((x_int_NXHII, x_int_NENERGY), np.float32)
    nlya = np.zeros_like(fheat)
    nhi = np.zeros_like(fheat)
    nhei = np.zeros_like(fheat)
    nheii = np.zeros_like(fheat)
    for i, x in enumerate(X_INT_XHII):
        if x < 0.3:
            fname = "log_xi_%1.1f.dat" % np.log10(float(x))
        else:
            fname = "xi_%1.3f.dat" % float(x)
        with open(os.path.join(tables_dir, "x_int_tables", fname)) as fh:
            tok = fh.read().split()
        # 5 labels, 5 numbers, 11 column labels, then 258 rows of 9 numbers
        data = np.array(tok[21:21 + 9 * x_int_NENERGY], dtype=np.float64).astype(np.float32).reshape(x_int_NENERGY, 9)
        energy = data[:, 0]
        fheat[i] = data[:, 2]
        nlya[i] = data[:, 4]
        nhi[i] = data[:, 5]
        nhei[i] = data[:, 6]
        nheii[i] = data[:, 7]
    return energy, fheat, nlya, nhi, nhei, nheii
