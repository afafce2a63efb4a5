"""CPU oracle for the recombination tables' interpolation -- TEST INFRASTRUCTURE ONLY.

Restates ``splined_recombination`` (src/core/recombinations.c:35-84) on the tables that
``init_MHR`` (:208-373) holds: the (z, T) row by rounding to the nearest sample (spacings the
float constants of recombinations.h:17-34), then the natural cubic spline (what
``gsl_interp_cspline`` builds) of that row in ln Gamma12, vectorised over cells.  Used only by
``tests/`` as the checker; the product never imports it.

The spline's second derivatives come from a banded solve of the natural-spline system (scipy),
not from the library's Thomas sweep, so the two are independent restatements.

Parity status: **parity unpinned** (the reference's tests hold no vectors for this path); the
restatement is pinned by known answers in ``tests/test_rec_oracle.py`` (cubic reproduction,
knot interpolation, the out-of-table branches).
"""

from __future__ import annotations

import numpy as np
from scipy.linalg import solve_banded

F32 = np.float32
Z_DEL = float(F32(0.2))        # RR_DEL_Z
T_STA = float(F32(2.0))        # RR_T_STA
T_DEL = float(F32(0.03))       # RR_DEL_T
LNG_MIN = float(F32(-10.0))    # RR_lnGamma_min
LNG_DEL = F32(0.1)             # RR_DEL_lnGamma
FRACT_FLOAT_ERR = 1e-7


def knots(ng: int = 150) -> np.ndarray:
    """lnGamma_values of init_MHR (recombinations.c:255-256): float sums stored as double."""
    return np.array([F32(F32(-10.0) + F32(LNG_DEL * F32(i))) for i in range(ng)], np.float64)


def natural_half_curvature(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """c = y''/2 of the natural cubic spline through (x, y[..., :]) along the last axis."""
    x = np.asarray(x, np.float64)
    n = x.size
    h = np.diff(x)
    flat = np.asarray(y, np.float64).reshape(-1, n)
    s = np.diff(flat, axis=1) / h                      # slopes [K][n-1]
    rhs = 3.0 * (s[:, 1:] - s[:, :-1])                 # [K][n-2]
    ab = np.zeros((3, n - 2))
    ab[0, 1:] = h[1:-1]                                # super-diagonal
    ab[1, :] = 2.0 * (h[:-1] + h[1:])
    ab[2, :-1] = h[1:-1]                               # sub-diagonal
    inner = solve_banded((1, 1), ab, rhs.T)            # [n-2][K]
    c = np.zeros_like(flat)
    c[:, 1:-1] = inner.T
    return c.reshape(np.shape(y))


class RecTables:
    """RR (ln rate), CF and RNH (ln residual xH), each [nz][nt][ng], and their splines."""

    def __init__(self, lnGamma, RR, CF, RNH):
        self.knots = np.asarray(lnGamma, np.float64)
        self.nz, self.nt, self.ng = np.shape(RR)
        self.y = np.stack([np.asarray(a, np.float64).reshape(self.nz * self.nt, self.ng) for a in (RR, CF, RNH)])
        self.c = natural_half_curvature(self.knots, self.y)
        self.lng_hi = float(F32(F32(-10.0) + F32(LNG_DEL * F32(self.ng - 1))))

    def splined(self, z_eff, gamma12, temp):
        """(rate, residual_xH, clumping_factor) per cell (recombinations.c:35-84)."""
        z_eff = np.asarray(z_eff, np.float64)
        temp = np.broadcast_to(np.asarray(temp, np.float64), z_eff.shape)
        gamma12 = np.asarray(gamma12, np.float64)
        z_ct = np.trunc((z_eff - 0.0) / Z_DEL + 0.5).astype(np.int64)
        with np.errstate(divide="ignore", invalid="ignore"):
            t_ct = np.trunc((np.log10(temp) - T_STA) / T_DEL + 0.5)
            lng = np.log(gamma12)
        t_ct = np.where(np.isfinite(t_ct), t_ct, -1).astype(np.int64)
        z_ct = np.clip(z_ct, 0, self.nz - 1)
        zero = (t_ct < 0) | ~(lng >= LNG_MIN)
        t_ct = np.clip(t_ct, 0, self.nt - 1)
        lng = np.where(lng >= self.lng_hi, self.lng_hi - FRACT_FLOAT_ERR, lng)
        lng = np.where(zero, self.knots[0], lng)
        lo = np.clip(np.searchsorted(self.knots, lng, side="right") - 1, 0, self.ng - 2)
        row = z_ct * self.nt + t_ct
        xlo = self.knots[lo]
        h = self.knots[lo + 1] - xlo
        dx = lng - xlo
        out = []
        for k in range(3):
            yl, yh = self.y[k, row, lo], self.y[k, row, lo + 1]
            cl, ch = self.c[k, row, lo], self.c[k, row, lo + 1]
            b = (yh - yl) / h - h * (ch + 2.0 * cl) / 3.0
            d = (ch - cl) / (3.0 * h)
            out.append(yl + dx * (b + dx * (cl + dx * d)))
        rate = np.where(zero, 0.0, np.exp(out[0]))
        cf = np.where(zero, 1.0, out[1])
        rnh = np.where(zero, 1e4, np.exp(out[2]))
        return rate, rnh, cf


def synthetic_tables(nz: int = 200, nt: int = 100, ng: int = 150) -> RecTables:
    """The stand-in tables of the test inputs (``workloads.rec_stand_in_tables``) with their splines."""
    import workloads
    return RecTables(*workloads.rec_stand_in_tables(nz, nt, ng))
