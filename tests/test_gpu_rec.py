"""GPU parity of the recombination branch of find_HII_bubbles (Flag_IncludeRecombinations) against
the oracle, through the C ABI, on smooth stand-in MHR tables with the real tables' ranges.

Two consecutive snapshots run on the device with the state carried on the device.  Before each
snapshot the oracle takes the device's state (z_at_ionization, J_21, temperature, Gamma12,
N_rec), so the second snapshot tests the barrier against a non-zero N_rec.  Tolerances (FP32
transforms against the FP64 oracle):
* ionized flags as in the find_HII parity tests (disagreements only within 1e-4 of the barrier,
  at most 0.01% of cells); r_bubble equal outside those cells;
* Gamma12 and J_21 (ReionUVBFlag 2): relative L2 <= 1e-4 over the cells that crossed;
* N_rec, residual_xH, clumping_factor, t_resp: relative L2 <= 1e-4 over the cells away from the
  barrier whose (z, T) table row is the same on both sides (a temperature within an ulp of a
  half-sample boundary may pick the neighbouring row);
* the recombination averages: 1e-4 relative.
"""

import ctypes as C

import numpy as np
import pytest

import rec_oracle as rco
import reion_oracle as ro
import rg_b200 as rg
import workloads as wl
from helpers import DeviceGrids, install_recfast, oracle_params, rel_l2

pytestmark = pytest.mark.gpu

TABLES = None


def tables():
    global TABLES
    if TABLES is None:
        TABLES = rco.synthetic_tables()
    return TABLES


def table_row(z, deltax, temp, temp_dep):
    dom = 1.0 + deltax.astype(np.float64)
    z_eff = (1.0 + z) * dom ** (1.0 / 3.0) - 1.0
    z_ct = np.clip(np.trunc(z_eff / rco.Z_DEL + 0.5), 0, 199)
    if not temp_dep:
        return z_ct
    with np.errstate(divide="ignore"):
        t_ct = np.trunc((np.log10(temp.astype(np.float64)) - rco.T_STA) / rco.T_DEL + 0.5)
    return z_ct * 1000 + np.clip(t_ct, -1, 99)


def set_tables(ctx):
    t = tables()
    ctx.set_recombination_tables(t.knots, *(t.y[k].reshape(t.nz, t.nt, t.ng) for k in range(3)))


def check_snapshot(n, z, prev_z, src, p, dg, out, st_o, extra, temp_dep):
    op = oracle_params(p)
    kw = {"rec_tables": tables(), "prev_z": prev_z, "record_margins": True}
    kw.update(extra)
    xH_o, rb_o, s_o, diag = ro.find_hii_bubbles(op, z, src.deltax, src.stars, src.sfr, st_o, "fp64", **kw)
    xH = dg.get("xH")
    ion_g, ion_o = xH < ro.REL_TOL, xH_o < ro.REL_TOL
    dis = ion_g != ion_o
    assert dis.mean() <= 1e-4, dis.mean()
    if dis.any():
        assert np.all(diag["min_margin"][dis] <= 1e-4)
    ok = diag["min_margin"] > 1e-4
    assert ion_o.mean() > 0.02 and (~ion_o).mean() > 0.02   # both branches exercised
    rb = dg.get("r_bubble")
    assert np.array_equal(rb[ok], rb_o[ok])
    crossed = ok & (rb_o > 0)
    assert crossed.sum() > 50
    assert rel_l2(dg.get("Gamma12")[crossed], st_o.Gamma12[crossed]) <= 1e-4
    assert np.array_equal(dg.get("Gamma12")[ok & ~crossed], st_o.Gamma12[ok & ~crossed])
    if p.ReionUVBFlag == 2:
        assert rel_l2(dg.get("J_21_at_ionization")[crossed], st_o.J_21_at_ionization[crossed]) <= 1e-4
    dxu = wl.from_padded(src.deltax)
    same_row = table_row(z, dxu, dg.get("temp_kinetic_all_gas"), temp_dep) == \
        table_row(z, dxu, st_o.temp_kinetic_all_gas, temp_dep)
    assert same_row.mean() > 0.999
    cmp = ok & same_row
    nrec = dg.get("N_rec")[:, :, :n]
    assert rel_l2(nrec[cmp], st_o.N_rec[cmp]) <= 1e-4
    rec = diag["rec"]
    for name in ("residual_xH", "clumping_factor", "t_resp"):
        assert rel_l2(dg.get(name)[cmp], rec[name][cmp]) <= 1e-4, name
    # the no-recombination branch (Gamma12 = 0) is exact
    zero = cmp & (st_o.Gamma12 == 0)
    assert zero.sum() > 0
    assert np.all(dg.get("residual_xH")[zero] == np.float32(1e4)) and np.all(dg.get("t_resp")[zero] == np.float32(1e30))
    for k in ("Gamma12", "N_rec", "residual_xH", "clumping_factor"):
        for w in ("volume", "mass"):
            key = f"{w}_weighted_global_{k}"
            assert getattr(out, key) == pytest.approx(s_o[key], rel=1e-4, abs=1e-12), key
    assert out.volume_weighted_global_r_bubble == pytest.approx(s_o["volume_weighted_global_r_bubble"], rel=1e-3)
    assert abs(out.volume_weighted_global_xH - s_o["volume_weighted_global_xH"]) <= 1e-4
    return xH_o


def load_state(dg, n, spin):
    st = ro.HIIState.fresh(n, rec=True)
    st.z_at_ionization[:] = dg.get("z_at_ionization")
    st.J_21_at_ionization[:] = dg.get("J_21_at_ionization")
    st.temp_kinetic_all_gas[:] = dg.get("temp_kinetic_all_gas")
    st.Gamma12[:] = dg.get("Gamma12")
    st.N_rec[:] = dg.get("N_rec")[:, :, :n]
    return st


@pytest.mark.parametrize("n,box,ftype,spin,bh,uvb,temp_dep,eff", [
    (32, 32.0, 0, 0, 0, 1, 1, 20000.0),
    (32, 32.0, 1, 0, 1, 2, 1, 4000.0),
    (64, 64.0, 0, 1, 0, 2, 0, 10000.0),
    (64, 64.0, 2, 1, 1, 1, 1, 10000.0),
    (48, 40.0, 0, 0, 1, 2, 0, 8000.0),
])
def test_recombinations_match_oracle(n, box, ftype, spin, bh, uvb, temp_dep, eff):
    install_recfast()
    zz, snap = wl.snapshot_redshifts(8.0)
    rng = np.random.default_rng(n + 10 * ftype + spin)
    dg = DeviceGrids(n, spin=bool(spin), bh=bool(bh), rec=True)
    p = rg.make_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMaxRecomb=30.0, ReionEfficiency=eff,
                       ReionFilterType=ftype, Flag_IncludeSpinTemp=spin, Flag_BHFeedback=bh, ReionUVBFlag=uvb,
                       Flag_IncludeRecombinations=1, Flag_TemperatureDependentRec=temp_dep)
    ctx = rg.Context(n)
    set_tables(ctx)
    for k, s in enumerate((snap - 1, snap)):
        src = wl.make_sources(n, box, seed=400 + n + k)
        dg.put("deltax", src.deltax)
        dg.put("stars", src.stars)
        dg.put("weighted_sfr", src.sfr)
        extra = {}
        if spin:
            xe = wl.to_padded((0.2 * rng.random((n, n, n))).astype(np.float32))
            tk = (10.0 + 990.0 * rng.random((n, n, n))).astype(np.float32)
            dg.put("x_e_box", xe)
            dg.put("Tk_box", tk)
            extra.update(x_e_box=xe, Tk_box=tk)
        if bh:
            bhm = (src.stars * 0.05 * rng.random(src.stars.shape)).astype(np.float32)
            bhar = (src.sfr * 0.3 * rng.random(src.sfr.shape)).astype(np.float32)
            dg.put("effective_bhm", bhm)
            dg.put("effective_bhar", bhar)
            extra.update(effective_bhm=bhm, effective_bhar=bhar)
        st_o = load_state(dg, n, spin)
        sn = rg.snapshot(zz, s)
        out = rg.rg_hii_scalars()
        ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(sn), C.byref(dg.g), C.byref(out))
        check_snapshot(n, float(zz[s]), float(zz[s - 1]), src, p, dg, out, st_o, extra, temp_dep)
        if k == 1:
            assert dg.get("N_rec").max() > 0.1   # the second snapshot read a non-zero N_rec
    ctx.close()


def test_recombination_host_entry_point_matches_device():
    """rg_find_HII_bubbles_host stages N_rec, Gamma12 and the recombination outputs through host
    arrays; its results equal the device-pointer call's bit for bit."""
    install_recfast()
    n, box = 32, 32.0
    zz, snap = wl.snapshot_redshifts(8.0)
    src = wl.make_sources(n, box, seed=91)
    p = rg.make_params(n, box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMaxRecomb=30.0, ReionEfficiency=20000.0,
                       Flag_IncludeRecombinations=1, ReionUVBFlag=2)
    rng = np.random.default_rng(5)
    n_rec0 = wl.to_padded((0.3 * rng.random((n, n, n))).astype(np.float32))
    g12 = (0.5 * rng.random(n ** 3)).astype(np.float32)
    ctx = rg.Context(n)
    set_tables(ctx)
    dg = DeviceGrids(n, rec=True)
    for k, v in (("deltax", src.deltax), ("stars", src.stars), ("weighted_sfr", src.sfr), ("N_rec", n_rec0),
                 ("Gamma12", g12)):
        dg.put(k, v)
    sn = rg.snapshot(zz, snap)
    o1 = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles", C.byref(p), C.byref(sn), C.byref(dg.g), C.byref(o1))
    npad = n * n * 2 * (n // 2 + 1)
    h = dict(deltax=src.deltax.ravel().copy(), stars=src.stars.ravel().copy(), weighted_sfr=src.sfr.ravel().copy(),
             N_rec=n_rec0.ravel().copy(), Gamma12=g12.copy(), xH=np.zeros(n ** 3, np.float32),
             r_bubble=np.zeros(n ** 3, np.float32), z_at_ionization=np.full(n ** 3, -1.0, np.float32),
             J_21_at_ionization=np.zeros(n ** 3, np.float32), temp_kinetic_all_gas=np.zeros(n ** 3, np.float32),
             residual_xH=np.zeros(n ** 3, np.float32), clumping_factor=np.zeros(n ** 3, np.float32),
             t_resp=np.zeros(n ** 3, np.float32))
    assert h["N_rec"].size == npad
    g = rg.rg_grids()
    for k, v in h.items():
        setattr(g, k, v.ctypes.data)
    o2 = rg.rg_hii_scalars()
    ctx.call("rg_find_HII_bubbles_host", C.byref(p), C.byref(sn), C.byref(g), C.byref(o2))
    ctx.close()
    for k in ("xH", "r_bubble", "Gamma12", "residual_xH", "clumping_factor", "t_resp", "J_21_at_ionization"):
        assert np.array_equal(h[k].reshape(n, n, n), dg.get(k)), k
    assert np.array_equal(h["N_rec"].reshape(n, n, -1)[:, :, :n], dg.get("N_rec")[:, :, :n])
    assert o1.as_dict() == o2.as_dict()
    assert o2.volume_weighted_global_N_rec > 0
