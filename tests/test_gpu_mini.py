"""GPU parity of the Pop III (mini-halo) sources of find_HII_bubbles (UseMiniHalos, the
USE_MINI_HALOS build of the reference) against the oracle, through the C ABI: starsIII in the
barrier with its own efficiency, in J_21 and in the partial xH; with recombinations also
weighted_sfrIII in Gamma12.  Tolerances as in the find_HII parity tests (ionized flags outside
the 1e-4 barrier margin equal; partial xH within 1e-4; J_21, Gamma12 relative L2 <= 1e-4;
temperatures <= 1e-5)."""

import ctypes as C

import numpy as np
import pytest

import reion_oracle as ro
import rg_b200 as rg
import test_gpu_rec as tr
import workloads as wl
from helpers import DeviceGrids, install_recfast, oracle_params, rel_l2

pytestmark = pytest.mark.gpu


def pop3_inputs(src, seed, frac=0.3):
    rng = np.random.default_rng(seed)
    s3 = (src.stars * frac * rng.random(src.stars.shape)).astype(np.float32)
    w3 = (src.sfr * 0.3 * rng.random(src.sfr.shape)).astype(np.float32)
    return s3, w3


def pop3_params(n, box, **kw):
    """Pop III with five times the photons per baryon (J_21, Gamma12) and twice the efficiency of
    Pop II (set directly, so the two populations' barrier terms are of one size)."""
    p = rg.make_params(n, box, UseMiniHalos=1, **kw)
    p.ReionNionPhotPerBaryIII = 5.0 * p.ReionNionPhotPerBary
    p.ReionEfficiencyIII = 2.0 * p.ReionEfficiency
    return p


@pytest.mark.parametrize("n,box,ftype,bh,rec,uvb,eff,frac", [
    (32, 32.0, 0, 0, 0, 1, 8000.0, 0.3),
    (64, 64.0, 1, 1, 0, 1, 4000.0, 0.3),
    (32, 32.0, 2, 1, 1, 2, 8000.0, 0.3),
    (48, 40.0, 0, 0, 1, 1, 6000.0, 0.3),
])
def test_pop3_matches_oracle(n, box, ftype, bh, rec, uvb, eff, frac):
    install_recfast()
    zz, snap = wl.snapshot_redshifts(8.0)
    z = float(zz[snap])
    src = wl.make_sources(n, box, seed=800 + n + ftype)
    s3, w3 = pop3_inputs(src, 801 + n, frac)
    rng = np.random.default_rng(802)
    p = pop3_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=20.0, ReionRBubbleMaxRecomb=20.0,
                    ReionEfficiency=eff, ReionFilterType=ftype, Flag_BHFeedback=bh, Flag_IncludeRecombinations=rec,
                    ReionUVBFlag=uvb)
    dg = DeviceGrids(n, bh=bool(bh), rec=bool(rec))
    dg.t["starsIII"] = dg.torch.zeros_like(dg.t["stars"])
    dg.t["weighted_sfrIII"] = dg.torch.zeros_like(dg.t["stars"])
    dg.g.starsIII = dg.t["starsIII"].data_ptr()
    dg.g.weighted_sfrIII = dg.t["weighted_sfrIII"].data_ptr()
    for k, v in (("deltax", src.deltax), ("stars", src.stars), ("weighted_sfr", src.sfr), ("starsIII", s3),
                 ("weighted_sfrIII", w3)):
        dg.put(k, v)
    kw = {"starsIII": s3, "weighted_sfrIII": w3}
    if bh:
        bhm = (src.stars * 0.05 * rng.random(src.stars.shape)).astype(np.float32)
        bhar = (src.sfr * 0.3 * rng.random(src.sfr.shape)).astype(np.float32)
        dg.put("effective_bhm", bhm)
        dg.put("effective_bhar", bhar)
        kw.update(effective_bhm=bhm, effective_bhar=bhar)
    st = ro.HIIState.fresh(n, rec=bool(rec))
    ctx = rg.Context(n)
    if rec:
        tr.set_tables(ctx)
        kw.update(rec_tables=tr.tables(), prev_z=float(zz[snap - 1]))
    out = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(rg.snapshot(zz, snap)), C.byref(dg.g), C.byref(out))
    ctx.close()
    xH_o, rb_o, s_o, diag = ro.find_hii_bubbles(oracle_params(p), z, src.deltax, src.stars, src.sfr, st, "fp64",
                                                record_margins=True, **kw)
    xH = dg.get("xH")
    ion_g, ion_o = xH < ro.REL_TOL, xH_o < ro.REL_TOL
    ok = diag["min_margin"] > 1e-4
    assert 0.02 < ion_o.mean() < 0.98
    assert (ion_g != ion_o).mean() <= 1e-4
    assert np.array_equal(ion_g[ok], ion_o[ok])
    part = ok & ~ion_o
    assert part.any() and np.max(np.abs(xH[part] - xH_o[part])) <= 1e-4
    assert abs(out.volume_weighted_global_xH - s_o["volume_weighted_global_xH"]) <= 1e-4
    same_first = ok & (diag["first_cross"] >= 0)
    assert rel_l2(dg.get("J_21_at_ionization")[same_first], st.J_21_at_ionization[same_first]) <= 1e-4
    assert rel_l2(dg.get("temp_kinetic_all_gas")[ok], st.temp_kinetic_all_gas[ok]) <= 1e-5
    assert out.volume_weighted_global_weighted_sfrIII == pytest.approx(s_o["volume_weighted_global_weighted_sfrIII"],
                                                                        rel=1e-5)
    if rec:
        crossed = ok & (rb_o > 0)
        assert rel_l2(dg.get("Gamma12")[crossed], st.Gamma12[crossed]) <= 1e-4
    # Pop III sources ionize: without them fewer cells cross
    p0 = rg.rg_params.from_buffer_copy(p)
    p0.ReionEfficiencyIII = 0.0
    st0 = ro.HIIState.fresh(n, rec=bool(rec))
    x0, _, _, _ = ro.find_hii_bubbles(oracle_params(p0), z, src.deltax, src.stars, src.sfr, st0, "fp64", **kw)
    assert (x0 < ro.REL_TOL).sum() < ion_o.sum()


def test_pop3_host_entry_point_matches_device():
    install_recfast()
    n, box = 32, 32.0
    zz, snap = wl.snapshot_redshifts(8.0)
    src = wl.make_sources(n, box, seed=901)
    s3, w3 = pop3_inputs(src, 902)
    p = pop3_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMaxRecomb=20.0, ReionEfficiency=3000.0,
                    Flag_IncludeRecombinations=1, ReionUVBFlag=2)
    ctx = rg.Context(n)
    tr.set_tables(ctx)
    dg = DeviceGrids(n, rec=True)
    dg.t["starsIII"] = dg.torch.zeros_like(dg.t["stars"])
    dg.t["weighted_sfrIII"] = dg.torch.zeros_like(dg.t["stars"])
    dg.g.starsIII = dg.t["starsIII"].data_ptr()
    dg.g.weighted_sfrIII = dg.t["weighted_sfrIII"].data_ptr()
    for k, v in (("deltax", src.deltax), ("stars", src.stars), ("weighted_sfr", src.sfr), ("starsIII", s3),
                 ("weighted_sfrIII", w3)):
        dg.put(k, v)
    sn = rg.snapshot(zz, snap)
    o1 = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(sn), C.byref(dg.g), C.byref(o1))
    z = lambda: np.zeros(n ** 3, np.float32)
    h = dict(deltax=src.deltax.ravel().copy(), stars=src.stars.ravel().copy(), weighted_sfr=src.sfr.ravel().copy(),
             starsIII=s3.ravel().copy(), weighted_sfrIII=w3.ravel().copy(),
             N_rec=np.zeros(n * n * 2 * (n // 2 + 1), np.float32), Gamma12=z(), xH=z(), r_bubble=z(),
             z_at_ionization=np.full(n ** 3, -1.0, np.float32), J_21_at_ionization=z(), temp_kinetic_all_gas=z(),
             residual_xH=z(), clumping_factor=z(), t_resp=z())
    g = rg.rg_grids()
    for k, v in h.items():
        setattr(g, k, v.ctypes.data)
    o2 = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles_host", C.byref(p), C.byref(sn), C.byref(g), C.byref(o2))
    ctx.close()
    for k in ("xH", "r_bubble", "Gamma12", "J_21_at_ionization", "temp_kinetic_all_gas", "t_resp"):
        assert np.array_equal(h[k].reshape(n, n, n), dg.get(k)), k
    assert o1.as_dict() == o2.as_dict()
    assert o2.volume_weighted_global_weighted_sfrIII > 0


def test_pop3_limits_and_unbuilt_channels():
    n = 16
    zz, snap = wl.snapshot_redshifts(8.0)
    sn = rg.snapshot(zz, snap, np.zeros(len(zz)))
    lib = rg.load()
    ctx = rg.Context(n)
    dg = DeviceGrids(n, spin=True)
    p = pop3_params(n, 20.0, Flag_IncludeSpinTemp=1)
    out = rg.rg_hii_scalars()
    # the grids are required; ComputeTs and delta_T have no Pop III channels
    assert lib.rg_find_HII_bubbles(ctx.h, C.byref(p), C.byref(sn), C.byref(dg.g), C.byref(out)) == rg.RG_EINVAL
    ts = rg.rg_ts_scalars()
    assert lib.rg_compute_Ts(ctx.h, C.byref(p), C.byref(sn), C.byref(dg.g), C.byref(ts)) == rg.RG_EUNSUPPORTED
    tb = C.c_double()
    assert lib.rg_delta_T(ctx.h, C.byref(p), C.byref(sn), C.byref(dg.g), C.byref(tb)) == rg.RG_EUNSUPPORTED
    ctx.close()
    # at 192^3 one z pass holds 8 grids: spin + BH + Pop III + recombinations (9) is refused
    n = 192
    ctx = rg.Context(n)
    set_tables = tr.set_tables
    set_tables(ctx)
    dg = DeviceGrids(n, spin=True, bh=True, rec=True)
    dg.t["starsIII"] = dg.torch.zeros_like(dg.t["stars"])
    dg.g.starsIII = dg.t["starsIII"].data_ptr()
    dg.g.weighted_sfrIII = dg.t["starsIII"].data_ptr()
    p = pop3_params(n, 190.0, Flag_IncludeSpinTemp=1, Flag_BHFeedback=1, Flag_IncludeRecombinations=1)
    assert lib.rg_find_HII_bubbles(ctx.h, C.byref(p), C.byref(sn), C.byref(dg.g), C.byref(out)) == rg.RG_EUNSUPPORTED
    assert "row buffers" in lib.rg_last_error(ctx.h).decode()
    ctx.close()
