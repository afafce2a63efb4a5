"""CPU checks of the nearest-grid-point deposit oracle (construct_baryon_grids restatement).
Known answers: pos_to_ngp's rounding, wrap and assertion; galaxies in one cell add up; the
clamp at zero and the SFR-timescale division; the padding columns stay zero."""

import numpy as np
import pytest

import grid_oracle as go


def test_pos_to_ngp_rounding_and_wrap():
    n, box = 8, 16.0  # cell side 2
    x = np.array([0.0, 0.99, 1.0, 1.01, 3.0, 5.0, 14.99, 15.0, 15.5, -0.9], np.float32)
    # x / 2: 0, 0.495, 0.5 (tie, even 0), 0.505, 1.5 (tie, even 2), 2.5 (tie, even 2),
    # 7.495, 7.5 (tie to 8 -> wrapped 0), 7.75 (8 -> 0), -0.45 (-0 -> 0)
    assert list(go.pos_to_ngp(x, box, n)) == [0, 0, 0, 1, 2, 2, 7, 0, 0, 0]
    with pytest.raises(ValueError):
        go.pos_to_ngp(np.array([-1.1], np.float32), box, n)


def test_deposit_sums_clamps_and_divides():
    n, box = 4, 4.0
    pos = np.array([[0.1, 0.2, 0.3], [0.4, 0.0, 0.2], [1.0, 2.0, 3.0], [3.9, 3.9, 3.9]], np.float32)
    vals = np.array([[1.0, 2.0, 5.0, 7.0], [1.0, -3.0, 4.0, 0.5]], np.float32)
    g = go.deposit_ngp(n, box, pos, vals, divisors=[1.0, 2.0])
    assert g.shape == (2, n, n, 2 * (n // 2 + 1))
    assert g[0, 0, 0, 0] == 3.0 + 7.0  # two galaxies in cell 0, and (3.9 -> 4 -> 0) wraps into it
    assert g[0, 1, 2, 3] == 5.0
    assert g[1, 0, 0, 0] == np.float32((max(1.0 - 3.0 + 0.5, 0.0)) / 2.0)
    assert g[1, 1, 2, 3] == 2.0
    assert np.count_nonzero(g[0]) == 2 and np.all(g[:, :, :, n:] == 0)


def test_deposit_clamps_negative_sums():
    n, box = 4, 4.0
    pos = np.array([[1.0, 1.0, 1.0], [1.2, 0.9, 1.1]], np.float32)
    vals = np.array([[-2.0, 1.0]], np.float32)
    g = go.deposit_ngp(n, box, pos, vals)
    assert np.all(g == 0)


def test_deposit_total_is_preserved():
    rng = np.random.default_rng(5)
    n, box, ng = 16, 25.0, 5000
    pos = (rng.random((ng, 3)) * box).astype(np.float32)
    vals = rng.random((3, ng)).astype(np.float32)
    g = go.deposit_ngp(n, box, pos, vals, divisors=[1.0, 3.0, 0.5])
    for p, d in enumerate([1.0, 3.0, 0.5]):
        assert g[p].sum(dtype=np.float64) == pytest.approx(vals[p].sum(dtype=np.float64) / d, rel=1e-5)
