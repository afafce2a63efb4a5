"""CPU oracle for the 21-cm power spectrum -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy, ``Initialise_PowerSpectrum`` and ``Compute_PS``
(src/core/ComputePowerSpectrum.c:18-42 and 44-255, the Pop II channel): the volume average of
delta_T, the padded field ((delta_T / ave - 1) V / N^3) ave, its unnormalised r2c transform, and
the log-spaced k bins (first upper edge 2 pi / L, factor 1.35, up to 2 pi N / L) holding
k^3 |delta_k|^2 / (2 pi^2 V), k and the mode count over the Hermitian half-space.  Used only by
``tests/`` as the checker; the product never imports it.

The bin edges and every mode's |k| are formed in float32 as the C code forms them (float
components, float squares and sums, the square root in double, rounded to float), so the bin of
each mode is the reference's; the transform is numpy's FP64 FFT (FFTW is not available here).

Parity status: **parity unpinned** (no golden vectors exist for this path); the restatement is
pinned by known answers in ``tests/test_ps_oracle.py`` (a single cosine mode, Parseval).
"""

from __future__ import annotations

import numpy as np


def bins(n: int, box_size: float, hubble_h: float):
    """(delta_k, upper edges) of Initialise_PowerSpectrum (ComputePowerSpectrum.c:21-39)."""
    box = box_size / hubble_h
    f = np.float32
    dk = f(2.0 * np.pi / box)
    k_max = f(dk * f(n))
    edges = []
    k_ceil = dk
    while k_ceil < k_max:
        edges.append(k_ceil)
        k_ceil = f(k_ceil * f(1.35))
    return dk, np.array(edges, dtype=np.float32)


def kmag(n: int, dk: np.float32) -> np.ndarray:
    """|k| of the Hermitian modes [x][y][z <= n/2] (ComputePowerSpectrum.c:170-189)."""
    f = np.float32
    idx = np.arange(n)
    signed = np.where(idx > n // 2, idx - n, idx).astype(np.float32)
    kx = (signed * dk).astype(np.float32)
    kz = (np.arange(n // 2 + 1).astype(np.float32) * dk).astype(np.float32)
    s = (kx[:, None, None] * kx[:, None, None]).astype(f) + (kx[None, :, None] * kx[None, :, None]).astype(f)
    s = s.astype(f) + (kz[None, None, :] * kz[None, None, :]).astype(f)
    return np.sqrt(s.astype(np.float32).astype(np.float64)).astype(np.float32)


def power_spectrum(delta_T: np.ndarray, box_size: float, hubble_h: float):
    """PS_k, PS_data, PS_error (float32) of Compute_PS for a real grid delta_T [n][n][n]."""
    n = delta_T.shape[0]
    box = box_size / hubble_h
    volume = np.float32(float(np.float32(box)) ** 3)
    n3 = float(n) ** 3
    d = delta_T.astype(np.float64)
    ave = d.sum() / n3
    field = ((d / ave - 1) * float(volume) / float(np.float32(n3))).astype(np.float32)
    field = (field.astype(np.float64) * ave).astype(np.float32)
    spec = np.fft.rfftn(field.astype(np.float64))
    dk, edges = bins(n, box_size, hubble_h)
    km = kmag(n, dk)
    b = np.searchsorted(edges, km, side="right")      # first edge above |k|
    inside = b < len(edges)
    kd = km.astype(np.float64)
    pw = kd ** 3 * (spec.real ** 2 + spec.imag ** 2) / (2.0 * np.pi * np.pi * float(volume))
    nb = len(edges)
    cnt = np.bincount(b[inside], minlength=nb).astype(np.float64)
    pbox = np.bincount(b[inside], weights=pw[inside], minlength=nb)
    kave = np.bincount(b[inside], weights=kd[inside], minlength=nb)
    with np.errstate(invalid="ignore", divide="ignore"):
        ps_k = (kave / cnt).astype(np.float32)
        ps = (pbox / cnt).astype(np.float32)
        err = ((pbox / cnt) / np.sqrt(cnt)).astype(np.float32)
    return ps_k, ps, err, cnt
