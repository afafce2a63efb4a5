"""GPU parity of the nearest-grid-point source deposit (construct_baryon_grids, one rank holding
the whole grid) against the oracle, through the C ABI.

The device adds the galaxies of a cell in any order (float atomics), the reference in galaxy
order, so a cell may differ by float rounding of its sum: the bound is 1e-5 of the sum of the
absolute values that went into the cell (divided like the cell).  Every cell index is exact
(positions that round differently would leave a whole galaxy's value in the wrong cell)."""

import ctypes as C

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


@pytest.mark.parametrize("agn", [0, 1])
def test_push_histories_matches_reference_shift(agn):
    """rg_push_histories: the slot shift of construct_baryon_grids (reionization.c:2105-2140) and
    the snapshot's grid into slot 0 (:2470-2500), for sfr, xray_luminosity and the AGN bands."""
    import torch
    n, nh = 16, 5
    npad = n * n * 2 * (n // 2 + 1)
    rng = np.random.default_rng(5 + agn)
    names = ["sfr", "xray_luminosity"] + (["bh_xray_soft", "bh_xray_hard"] if agn else [])
    hists = {"sfr": "sfr_histories", "xray_luminosity": "xray_luminosity_histories",
             "bh_xray_soft": "bh_xray_histories_soft", "bh_xray_hard": "bh_xray_histories_hard"}
    cur = {k: rng.random(npad).astype(np.float32) for k in names}
    hist = {k: rng.random(nh * npad).astype(np.float32) for k in names}
    dcur = {k: torch.from_numpy(v).cuda() for k, v in cur.items()}
    dhist = {k: torch.from_numpy(v).cuda() for k, v in hist.items()}
    g = rg.rg_grids()
    for k in names:
        setattr(g, k, dcur[k].data_ptr())
        setattr(g, hists[k], dhist[k].data_ptr())
    g.n_hist = nh
    p = rg.make_params(n, 20.0, Flag_IncludeSpinTemp=1, Flag_IncludeAGNXray=agn)
    ctx = rg.Context(n)
    assert ctx.lib.rg_push_histories(ctx.h, C.byref(p), C.byref(g)) == rg.RG_OK
    torch.cuda.synchronize()
    ctx.close()
    for k in names:
        want = hist[k].reshape(nh, npad).copy()
        for s in range(nh - 2, -1, -1):       # the reference's loop, slot s + 1 <- slot s
            want[s + 1] = want[s]
        want[0] = cur[k]
        assert np.array_equal(dhist[k].cpu().numpy().reshape(nh, npad), want), k
