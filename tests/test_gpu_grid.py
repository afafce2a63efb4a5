"""GPU parity of the nearest-grid-point source deposit (construct_baryon_grids, one rank holding
the whole grid) against the oracle, through the C ABI.

The device adds the galaxies of a cell in any order (float atomics), the reference in galaxy
order, so a cell may differ by float rounding of its sum: the bound is 1e-5 of the sum of the
absolute values that went into the cell (divided like the cell).  Every cell index is exact
(positions that round differently would leave a whole galaxy's value in the wrong cell)."""

import numpy as np
import pytest

import grid_oracle as go
import rg_b200 as rg

pytestmark = pytest.mark.gpu


def run_deposit(n, box, pos, vals, divisors=None):
    import torch
    ctx = rg.Context(n)
    padw = 2 * (n // 2 + 1)
    n_prop = vals.shape[0]
    grids = [torch.full((n * n * padw,), 7.0, dtype=torch.float32, device="cuda") for _ in range(n_prop)]
    dpos = torch.from_numpy(np.ascontiguousarray(pos, np.float32).ravel()).cuda()
    dval = torch.from_numpy(np.ascontiguousarray(vals, np.float32).ravel()).cuda()
    ctx.deposit_ngp(box, pos.shape[0], dpos.data_ptr(), dval.data_ptr(), [g.data_ptr() for g in grids], divisors)
    out = np.stack([g.cpu().numpy().reshape(n, n, padw) for g in grids])
    ctx.close()
    return out


def bound(n, box, pos, vals, divisors):
    absg = go.deposit_ngp(n, box, pos, np.abs(vals), divisors)
    return 1e-5 * absg + 1e-30


@pytest.mark.parametrize("n,box,ng,n_prop", [(32, 40.0, 100_000, 3), (64, 67.8, 400_000, 5), (128, 100.0, 50_000, 8)])
def test_deposit_matches_oracle(n, box, ng, n_prop):
    rng = np.random.default_rng(n + ng)
    # clustered positions (many galaxies per cell), a few on the top edge (wrap to 0) and just
    # below 0 (round to cell 0)
    centres = rng.random((64, 3)) * box
    pos = (centres[rng.integers(0, 64, ng)] + rng.normal(0, box / n, (ng, 3))) % box
    pos[:50] = box
    pos[50:100] = -0.2 * box / n
    pos = pos.astype(np.float32)
    vals = rng.lognormal(0, 1, (n_prop, ng)).astype(np.float32)
    vals[n_prop - 1] -= 1.0  # a signed property: some cells sum below zero and clamp
    divisors = [1.0] * (n_prop - 1) + [3.7e-2]
    got = run_deposit(n, box, pos, vals, divisors)
    want = go.deposit_ngp(n, box, pos, vals, divisors)
    assert np.all(np.abs(got - want) <= bound(n, box, pos, vals, divisors))
    assert np.all(got[:, :, :, n:] == 0)  # padding overwritten with zeros
    assert np.count_nonzero(want[-1]) < np.count_nonzero(want[0])  # the clamp was exercised


def test_deposit_no_galaxies_zeroes_grids():
    n = 32
    got = run_deposit(n, 40.0, np.zeros((0, 3), np.float32), np.zeros((2, 0), np.float32))
    assert np.all(got == 0)


def test_deposit_rejects_positions_below_box_and_stays_usable():
    import torch
    n, box = 32, 40.0
    ctx = rg.Context(n)
    padw = 2 * (n // 2 + 1)
    g = torch.zeros(n * n * padw, dtype=torch.float32, device="cuda")
    pos = torch.tensor([[1.0, 2.0, 3.0], [1.0, -2.0, 3.0]], dtype=torch.float32, device="cuda")
    val = torch.ones(2, dtype=torch.float32, device="cuda")
    with pytest.raises(rg.RGError) as e:
        ctx.deposit_ngp(box, 2, pos.data_ptr(), val.data_ptr(), [g.data_ptr()])
    assert e.value.status == rg.RG_EINVAL
    with pytest.raises(rg.RGError):
        ctx.deposit_ngp(box, 2, pos.data_ptr(), val.data_ptr(), [g.data_ptr()], divisors=[0.0])
    ctx.deposit_ngp(box, 1, pos.data_ptr(), val.data_ptr(), [g.data_ptr()])
    h = g.cpu().numpy().reshape(n, n, padw)
    ix, iy, iz = go.pos_to_ngp(np.array([1.0, 2.0, 3.0], np.float32), box, n)
    assert h[ix, iy, iz] == 1.0 and h.sum() == 1.0
    ctx.close()
