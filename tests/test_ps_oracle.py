"""CPU checks of the power-spectrum oracle (Compute_PS restatement) and of the library's bin
count.  Known answers: a single cosine mode puts all its power, with the reference's
normalisation, into the bin of its |k|; a uniform field has no power."""

import numpy as np
import pytest

import ps_oracle as po
import rg_b200 as rg


@pytest.mark.parametrize("n,box,h", [(16, 20.0, 0.678), (64, 64.0, 0.7), (128, 100.0, 0.678), (512, 500.0, 0.678)])
def test_bin_count_matches_library(n, box, h):
    dk, edges = po.bins(n, box, h)
    assert edges[0] == dk and np.all(np.diff(edges) > 0) and edges[-1] < np.float32(dk * np.float32(n))
    p = rg.make_params(n, box, Hubble_h=h)
    assert rg.power_spectrum_length(p) == len(edges)


def test_single_cosine_mode():
    n, box, h = 32, 40.0, 0.7
    amp, mean, n0 = 3.0, 20.0, 5
    x = np.arange(n)
    field = mean + amp * np.cos(2 * np.pi * n0 * x / n)
    dT = np.broadcast_to(field[:, None, None], (n, n, n)).astype(np.float32)
    ps_k, ps, err, cnt = po.power_spectrum(dT, box, h)
    dk, edges = po.bins(n, box, h)
    k0 = float(np.sqrt(np.float64(np.float32(np.float32(n0) * dk)) ** 2))
    k0 = float(np.float32(k0))
    b = int(np.searchsorted(edges, np.float32(k0), side="right"))
    vol = float(np.float32(float(np.float32(box / h)) ** 3))
    # modes (n0, 0, 0) and (n - n0, 0, 0), each |delta_k| = amp V / 2
    want = 2 * k0 ** 3 * (amp * vol / 2) ** 2 / (2 * np.pi ** 2 * vol) / cnt[b]
    assert ps[b] == pytest.approx(want, rel=1e-5)
    others = np.delete(ps, b)
    assert np.all(np.abs(others[np.isfinite(others)]) <= 1e-8 * ps[b])
    # the bin's k average and the Poisson error
    assert err[b] == pytest.approx(ps[b] / np.sqrt(cnt[b]), rel=1e-6)
    assert cnt.sum() <= n * n * (n // 2 + 1) and cnt[0] == 1


def test_uniform_field_has_no_power():
    n = 16
    dT = np.full((n, n, n), 7.5, np.float32)
    ps_k, ps, err, cnt = po.power_spectrum(dT, 20.0, 0.7)
    assert np.all(np.abs(ps[np.isfinite(ps)]) <= 1e-20)
