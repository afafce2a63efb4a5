"""GPU parity of the brightness temperature with peculiar velocities (Flag_IncludePecVelsFor21cm
1, 2 and 3, spin temperature on) against the oracle, through the C ABI.  Tolerances: delta_T
relative L2 <= 1e-5 against the FP64 oracle (FP32 transform of the velocity; for flag 3 the
sub-cell shares reach each cell in any order, in float), the volume average to 1e-5."""

import ctypes as C

import numpy as np
import pytest

import rg_b200 as rg
import vel_oracle as vo
import workloads as wl
from helpers import DeviceGrids, oracle_params, rel_l2

pytestmark = pytest.mark.gpu


def run_case(n, box, flag, trees, seed, host=False):
    import torch
    rng = np.random.default_rng(seed)
    npad = 2 * (n // 2 + 1)
    xH = rng.random((n, n, n)).astype(np.float32)
    xH[rng.random((n, n, n)) < 0.2] = 0.0
    deltax = (0.3 * rng.standard_normal((n, n, npad))).astype(np.float32)
    TS = (20.0 + 80.0 * rng.random((n, n, n))).astype(np.float32)
    # a smooth velocity field (correlation length ~3 cells) with displacements of about one cell:
    # raw velocities of order 20 (VELOCIraptor units) at z = 8; |dv/dz| / H stays well below 1, as
    # in a cosmological field (near dv/dz = -H the optical depth is ill-conditioned in any precision)
    k = np.fft.fftfreq(n) * n
    kz = np.arange(n // 2 + 1)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2
    sm = np.fft.irfftn(np.fft.rfftn(rng.standard_normal((n, n, n))) * np.exp(-k2 * (3.0 * 2 * np.pi / n) ** 2 / 2),
                       s=(n, n, n), axes=(0, 1, 2))
    sm *= 20.0 / sm.std()
    vel = np.zeros((n, n, npad), np.float32)
    vel[:, :, :n] = sm
    if trees == 1:
        vel *= 3000.0
    p = rg.make_params(n, box, Flag_IncludeSpinTemp=1, Flag_IncludePecVelsFor21cm=flag, TreesID=trees)
    zz, snap = wl.snapshot_redshifts(8.0)
    s = rg.snapshot(zz, snap)
    ctx = rg.Context(n)
    tb = C.c_double()
    if host:
        h = {"deltax": deltax, "xH": xH, "TS_box": TS, "vel": vel, "delta_T": np.zeros((n, n, n), np.float32)}
        g = rg.rg_grids()
        for k, v in h.items():
            setattr(g, k, v.ctypes.data)
        ctx.call("rg_delta_T_host", C.byref(p), C.byref(s), C.byref(g), C.byref(tb))
        got = h["delta_T"]
    else:
        dg = DeviceGrids(n, spin=True)
        dg.put("deltax", deltax)
        dg.put("xH", xH)
        dg.put("TS_box", TS)
        dv = torch.from_numpy(vel.ravel()).cuda()
        dg.g.vel = dv.data_ptr()
        ctx.call("rg_delta_T", C.byref(p), C.byref(s), C.byref(dg.g), C.byref(tb))
        got = dg.get("delta_T")
    ctx.close()
    op = oracle_params(p)
    op.Flag_IncludeSpinTemp = 1
    op.Flag_IncludePecVelsFor21cm = flag
    op.TreesID = trees
    want, ave = vo.delta_T_velocity(op, float(zz[snap]), xH, deltax, TS, vel)
    return got, tb.value, want, ave


@pytest.mark.parametrize("flag", [1, 2, 3])
@pytest.mark.parametrize("n,box", [(32, 40.0), (64, 64.0)])
def test_velocity_modes_match_oracle(n, box, flag):
    got, tb, want, ave = run_case(n, box, flag, 0, 100 * flag + n)
    assert rel_l2(got, want) <= 1e-5
    assert tb == pytest.approx(ave, rel=1e-5)


def test_velocity_modes_gbptrees_units_and_host_entry():
    got, tb, want, ave = run_case(32, 40.0, 3, 1, 7)
    assert rel_l2(got, want) <= 1e-5
    got_h, tb_h, _, _ = run_case(32, 40.0, 3, 1, 7, host=True)
    # the host form is the same computation (shares of one cell meet in any order: float level)
    assert rel_l2(got_h, got) <= 1e-6
    assert tb_h == pytest.approx(tb, rel=1e-6)
