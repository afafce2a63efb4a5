"""CPU oracle for the nearest-grid-point source deposit -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy, the per-property grid construction of ``construct_baryon_grids``
(src/core/reionization.c:2025-2592) for one rank holding the whole grid:

* ``pos_to_ngp`` (src/core/misc_tools.c:207-217): ``nearbyint(x / side * nx)`` in double (the
  default rounding, ties to even), an index above ``nx - 1`` wrapped to 0, a negative one an
  assertion failure;
* the rank's galaxies added to a float32 buffer in galaxy order (reionization.c:2236-2300);
* each cell read back in double, clamped at zero (``CLAMP_NEGATIVE``, src/core/misc_tools.h:7),
  divided by the SFR timescale for the sfr grids (reionization.c:2500-2510) and stored as float
  in the padded layout (reionization.c:2440-2520).

Used only by ``tests/`` as the checker; the product never imports it.

Parity status: **parity unpinned** (the reference's tests hold no vectors for this path); the
restatement is pinned by known answers in ``tests/test_grid_oracle.py``.
"""

from __future__ import annotations

import numpy as np


def pos_to_ngp(x, side: float, nx: int) -> np.ndarray:
    """pos_to_ngp of float positions (misc_tools.c:207-217); raises on an index below 0."""
    ind = np.rint(np.asarray(x, np.float32).astype(np.float64) / side * float(nx)).astype(np.int64)
    ind[ind > nx - 1] = 0
    if np.any(ind < 0):
        raise ValueError("position below the box (pos_to_ngp asserts)")
    return ind


def deposit_ngp(n: int, box_size: float, pos, values, divisors=None) -> np.ndarray:
    """Grids [n_prop][n][n][2(n/2+1)] (float32, padded layout) of the deposit.

    ``pos`` is (n_gal, 3) float32 in box units, ``values`` (n_prop, n_gal) float32 and
    ``divisors`` n_prop positive doubles (None for none).
    """
    pos = np.asarray(pos, np.float32).reshape(-1, 3)
    values = np.asarray(values, np.float32).reshape(-1, pos.shape[0])
    n_prop = values.shape[0]
    ix, iy, iz = (pos_to_ngp(pos[:, a], box_size, n) for a in range(3))
    cell = (ix * n + iy) * n + iz
    padw = 2 * (n // 2 + 1)
    out = np.zeros((n_prop, n, n, padw), np.float32)
    for p in range(n_prop):
        buf = np.zeros(n ** 3, np.float32)
        np.add.at(buf, cell, values[p])  # unbuffered float32 adds in galaxy order
        val = buf.astype(np.float64)
        val[val < 0] = 0.0
        if divisors is not None:
            val = val / float(divisors[p])
        out[p, :, :, :n] = val.astype(np.float32).reshape(n, n, n)
    return out
