"""GPU parity of the callers next to the step, through the C ABI:

* the 21-cm power spectrum (Compute_PS) against the oracle restatement: PS_k to 1e-6 relative
  (every mode in the reference's bin), PS_data and PS_error to 1e-5 relative (FP32 transform
  against the FP64 oracle), empty bins NaN in both;
* smooth_grid against the FP64 filter round trip: relative L2 <= 1e-5.
"""

import numpy as np
import pytest

import ps_oracle as po
import reion_oracle as ro
import rg_b200 as rg
import workloads as wl
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def close(got, want, rel):
    both_nan = np.isnan(got) & np.isnan(want)
    ok = both_nan | (np.abs(got - want) <= rel * np.abs(want) + 1e-30)
    return bool(np.all(ok))


@pytest.mark.parametrize("n,box,h", [(32, 40.0, 0.7), (64, 64.0, 0.678), (128, 100.0, 0.678)])
def test_power_spectrum_matches_oracle(n, box, h):
    import torch
    rng = np.random.default_rng(n + 3)
    dT = (15.0 + 4.0 * rng.standard_normal((n, n, n))).astype(np.float32)
    p = rg.make_params(n, box, Hubble_h=h)
    ctx = rg.Context(n)
    d = torch.from_numpy(dT.ravel()).cuda()
    k, ps, err = ctx.power_spectrum(p, d.data_ptr())
    k2, ps2, err2 = ctx.power_spectrum(p, dT.ctypes.data, host=True)
    ctx.close()
    wk, wps, werr, cnt = po.power_spectrum(dT, box, h)
    assert len(k) == len(wk)
    assert close(k, wk, 1e-6)
    assert close(ps, wps, 1e-5)
    assert close(err, werr, 1e-5)
    # the host-buffer form is the same computation
    assert np.array_equal(k, k2, equal_nan=True) and np.array_equal(ps, ps2, equal_nan=True)
    assert np.array_equal(err, err2, equal_nan=True)


def test_power_spectrum_single_mode():
    import torch
    n, box, h = 64, 80.0, 0.7
    x = np.arange(n)
    field = 20.0 + 3.0 * np.cos(2 * np.pi * 7 * x / n)
    dT = np.broadcast_to(field[None, :, None], (n, n, n)).astype(np.float32).copy()
    p = rg.make_params(n, box, Hubble_h=h)
    ctx = rg.Context(n)
    d = torch.from_numpy(dT.ravel()).cuda()
    k, ps, err = ctx.power_spectrum(p, d.data_ptr())
    ctx.close()
    wk, wps, werr, cnt = po.power_spectrum(dT, box, h)
    b = int(np.nanargmax(wps))
    assert int(np.nanargmax(ps)) == b
    assert ps[b] == pytest.approx(wps[b], rel=1e-5)
    rest = np.delete(ps, b)
    assert np.all(np.abs(rest[np.isfinite(rest)]) <= 1e-6 * ps[b])


@pytest.mark.parametrize("n,box,dim", [(64, 64.0, 32), (128, 100.0, 32)])
def test_smooth_grid_matches_fp64(n, box, dim):
    import torch
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n)).astype(np.float32)
    d_in = torch.from_numpy(wl.to_padded(x).ravel()).cuda()
    d_out = torch.zeros_like(d_in)
    ctx = rg.Context(n)
    ctx.call("rg_smooth_grid", box, dim, d_in.data_ptr(), d_out.data_ptr())
    ctx.close()
    got = d_out.cpu().numpy().reshape(n, n, -1)[:, :, :n]
    R = float(np.float32(box / dim / 2.0))
    want = ro.inverse(ro.forward(x.astype(np.float64), "fp64") * ro.window(n, box, R, 0, "fp64"), n)
    assert rel_l2(got, want) <= 1e-5
