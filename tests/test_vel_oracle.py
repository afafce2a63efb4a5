"""CPU checks of the peculiar-velocity oracle (BrightnessTemperature.c velocity block).
Known answers: no velocity leaves the re-binning an identity and the gradient zero; a uniform
displacement of one cell moves every line by one cell; the re-binning conserves each line's sum."""

import numpy as np
import pytest

import reion_oracle as ro
import vel_oracle as vo


def _line_case(n=16, seed=0):
    rng = np.random.default_rng(seed)
    dT = (5.0 + rng.random((n, n, n))).astype(np.float32)
    xH = np.ones((n, n, n), np.float32)
    return dT, xH


def test_rsd_identity_without_velocity():
    n, box = 16, 32.0
    dT, xH = _line_case(n)
    out = vo.rsd(dT, xH, np.zeros((n, n, n), np.float32), 1e-17, box)
    assert np.allclose(out, dT, rtol=1e-6, atol=0)


def test_rsd_shift_by_one_cell():
    n, box = 16, 32.0
    dT, xH = _line_case(n, 1)
    H = 2e-17
    cell = box / n
    vc = np.full((n, n, n), np.float32(cell * H), np.float32)
    out = vo.rsd(dT, xH, vc, H, box)
    assert np.allclose(out, np.roll(dT, 1, axis=2), rtol=1e-5, atol=0)


def test_rsd_conserves_line_sums():
    n, box = 16, 32.0
    dT, xH = _line_case(n, 2)
    rng = np.random.default_rng(9)
    H = 2e-17
    vc = (rng.standard_normal((n, n, n)) * 1.5 * (box / n) * H).astype(np.float32)
    xH[0, 0, 3] = 0.0           # a fully ionised cell contributes nothing
    out = vo.rsd(dT, xH, vc, H, box)
    keep = dT.astype(np.float64) * (xH >= 1e-7)
    assert np.allclose(out.sum(axis=2), keep.sum(axis=2), rtol=1e-9)


def test_gradient_of_a_sine():
    n, L, h = 32, 40.0, 0.7
    z = np.arange(n)
    v = np.broadcast_to(np.sin(2 * np.pi * 3 * z / n)[None, None, :], (n, n, n)).astype(np.float32)
    g = vo.z_gradient(v, L, h)
    dk = float(np.float32(2 * np.pi / float(np.float32(L))))
    want = h * 3 * dk * np.cos(2 * np.pi * 3 * z / n)
    assert np.allclose(g[0, 0], want, rtol=1e-6, atol=1e-9)


def test_flag1_zero_gradient_keeps_delta_T():
    n = 8
    p = ro.Params(ReionGridDim=n, BoxSize=16.0)
    p.Flag_IncludeSpinTemp = 1
    p.Flag_IncludePecVelsFor21cm = 1
    p.TreesID = 0
    rng = np.random.default_rng(4)
    xH = rng.random((n, n, n)).astype(np.float32)
    deltax = np.zeros((n, n, 2 * (n // 2 + 1)), np.float32)
    TS = np.full((n, n, n), 50.0, np.float32)
    vel = np.zeros((n, n, 2 * (n // 2 + 1)), np.float32)
    got, ave = vo.delta_T_velocity(p, 8.0, xH, deltax, TS, vel)
    base = vo.base_delta_T(p, 8.0, xH, deltax, TS)
    assert np.allclose(got, base, rtol=1e-7)
