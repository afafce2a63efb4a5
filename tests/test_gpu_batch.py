"""rg_find_HII_bubbles_batch: several snapshots of one size in one call (shared forward and x/y
launches, per-snapshot z passes) give every snapshot exactly what rg_find_HII_bubbles gives it:
the same kernels do the same arithmetic on each snapshot's grids, so the grids and box averages
are compared for equality.  Units with different radii or sizes are refused."""

import ctypes as C

import numpy as np
import pytest

import rg_b200 as rg
import workloads as wl

pytestmark = pytest.mark.gpu


def make_unit(n, box, z, eff, seed, spin, torch):
    src = wl.make_sources(n, box, seed)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32).ravel()).cuda()
    b = {"deltax": t(src.deltax), "stars": t(src.stars), "weighted_sfr": t(src.sfr)}
    for k in ("xH", "r_bubble", "J_21_at_ionization", "temp_kinetic_all_gas"):
        b[k] = torch.zeros(n ** 3, device="cuda")
    b["z_at_ionization"] = torch.full((n ** 3,), -1.0, device="cuda")
    if spin:
        rng = np.random.default_rng(seed + 1)
        b["x_e_box"] = t(np.abs(rng.normal(2e-3, 1e-3, src.deltax.shape)))
        b["Tk_box"] = torch.full((n ** 3,), 30.0, device="cuda")
    g = rg.rg_grids()
    for k, v in b.items():
        setattr(g, k, v.data_ptr())
    p = rg.make_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=20.0, ReionEfficiency=eff,
                       Flag_IncludeSpinTemp=int(spin), ReionUVBFlag=1)
    zz, idx = wl.snapshot_redshifts(z)
    return dict(b=b, g=g, p=p, s=rg.snapshot(zz, idx))


def fresh(units, torch):
    return [make_unit(*u, torch) for u in units]


@pytest.mark.parametrize("n,spin,kb", [(64, False, 8), (96, True, 5), (128, False, 16)])
def test_batch_equals_one_at_a_time(n, spin, kb):
    import torch
    units = [(n, float(n), z, eff, 100 + i, spin) for i, (z, eff) in
             enumerate([(12.0, 3000.0), (9.5, 60.0), (8.0, 40000.0), (7.0, 900.0)])]
    ctx = rg.Context(n)
    ctx.call("rg_set_radius_batch", kb)
    one = fresh(units, torch)
    outs1 = []
    for u in one:
        o = rg.rg_hii_scalars()
        ctx.call("rg_find_HII_bubbles", C.byref(u["p"]), C.byref(u["s"]), C.byref(u["g"]), C.byref(o))
        outs1.append(o)
    many = fresh(units, torch)
    outs2 = ctx.find_hii_batch([u["p"] for u in many], [u["s"] for u in many], [u["g"] for u in many])
    torch.cuda.synchronize()
    ctx.close()
    xh = []
    for a, b, oa, ob in zip(one, many, outs1, outs2):
        for k in ("xH", "z_at_ionization", "J_21_at_ionization", "temp_kinetic_all_gas", "r_bubble"):
            assert torch.equal(a["b"][k], b["b"][k]), k
        for f, _ in rg.rg_hii_scalars._fields_:
            assert getattr(oa, f) == getattr(ob, f), f
        xh.append(oa.volume_weighted_global_xH)
    assert min(xh) < 0.9 and max(xh) > 0.99   # partly ionised and nearly neutral units both covered


def test_batch_refuses_different_sizes_and_radii():
    import torch
    ctx = rg.Context(64)
    a = make_unit(64, 64.0, 8.0, 100.0, 1, False, torch)
    b = make_unit(64, 64.0, 8.0, 100.0, 2, False, torch)
    b["p"].BoxSize = 80.0
    with pytest.raises(rg.RGError) as e:
        ctx.find_hii_batch([a["p"], b["p"]], [a["s"], b["s"]], [a["g"], b["g"]])
    assert e.value.status == rg.RG_EINVAL
    c = make_unit(64, 64.0, 8.0, 100.0, 3, False, torch)
    c["p"].ReionRBubbleMax = 10.0
    with pytest.raises(rg.RGError) as e:
        ctx.find_hii_batch([a["p"], c["p"]], [a["s"], c["s"]], [a["g"], c["g"]])
    assert e.value.status == rg.RG_EINVAL
    ctx.close()
