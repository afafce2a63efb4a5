"""CPU checks of the spin-temperature oracle and of the library's host coefficient engine.

The oracle's quadrature, root finder and rule are pinned by known answers; the host
engine (shells, history weights, frequency tables, Lyman-n sums; no device work) must
agree with the oracle: shells to 1e-12, frequency tables to 1e-6 relative (both run
the same adaptive QAG, so only rounding differs), history weights to float rounding.
"""

import math
import os
import re

import numpy as np
import pytest

import gk61
import reion_oracle as ro
import rg_b200 as rg
import ts_oracle as to
import workloads as wl
from helpers import oracle_params

HERE = os.path.dirname(os.path.abspath(__file__))


def test_gk61_rule_exact_to_degree_91():
    x, wk, wg = gk61.rule()
    assert x[30] == 0.0 and np.all(np.diff(x) < 0)
    for k in range(0, 92, 2):
        got = 2 * np.sum(wk[:30] * x[:30] ** k) + (wk[30] if k == 0 else 0.0)
        assert abs(got - 2.0 / (k + 1)) <= 2e-15
    for k in range(0, 60, 2):   # the embedded 30-point Gauss rule
        got = 2 * np.sum(wg * x[:30] ** k)
        assert abs(got - 2.0 / (k + 1)) <= 2e-15


def test_gk61_header_matches_oracle_rule():
    path = os.path.join(HERE, "..", "meraxes-devs_qyxnew_b200", "csrc", "rg_gk61.h")
    text = open(path).read()

    def arr(name):
        body = re.search(name + r"\[31\] = \{([^}]*)\}", text).group(1)
        return np.array([float(v) for v in body.split(",") if v.strip()])

    x, wk, wg = gk61.rule()
    assert np.allclose(arr("GK61_X"), x, rtol=0, atol=1e-16)
    assert np.allclose(arr("GK61_WK"), wk, rtol=0, atol=1e-16)
    assert np.allclose(arr("GK61_WG")[:30], wg, rtol=0, atol=1e-16)


def test_qag61_known_integrals():
    st, r, e = to.qag61(lambda x: x ** 5, 0.0, 1.0, 0, 1e-10)
    assert st == 0 and abs(r - 1 / 6) < 1e-15
    st, r, e = to.qag61(np.sin, 0.0, math.pi, 0, 1e-12)
    assert st == 0 and abs(r - 2.0) < 1e-14
    # a sharp peak needs bisection
    st, r, e = to.qag61(lambda x: 1.0 / (x * x + 1e-4), -1.0, 1.0, 0, 1e-10)
    assert st == 0 and abs(r - 200.0 * math.atan(100.0)) <= 1e-9 * r
    # iteration limit reached -> non-zero status, as GSL reports it
    st, r, e = to.qag61(lambda x: 1.0 / np.sqrt(np.abs(x - 0.3)), 0.0, 1.0, 0, 1e-14, limit=3)
    assert st != 0


def test_brent_known_roots():
    r, st = to.brent(lambda x: x ** 3 - 2.0, 0.0, 2.0, 0, 1e-12, 100)
    assert st == 0 and abs(r - 2 ** (1 / 3)) < 1e-11
    r, st = to.brent(lambda x: math.cos(x) - x, 0.0, 1.0, 0, 1e-12, 100)
    assert st == 0 and abs(r - 0.7390851332151607) < 1e-11
    r, st = to.brent(lambda x: x * x + 1, 0.0, 1.0, 0, 1e-12, 100)
    assert st == 1           # the end points do not straddle a root


def test_homogeneous_branch_uniform_box():
    # deltax = 0: T_K = T_RECFAST(z), x_e = xion_RECFAST(z), T_S from collisional coupling only
    n = 8
    p = ro.Params(ReionGridDim=n, BoxSize=16.0)
    T = to.TsTables()
    zz, idx = wl.snapshot_redshifts(33.0)
    z = zz[idx]
    g = dict(deltax=np.zeros((n, n, n), np.float32), stars=np.zeros((n, n, n), np.float32),
             x_e_box_prev=np.zeros((n, n, n), np.float32), Tk_box=np.zeros((n, n, n), np.float32))
    out = to.compute_ts(p, T, zz, idx, None, g)
    assert out["homogeneous"] == 1 and out["collapse_fraction"] == 0.0
    tk = np.float32(T.recfast.T(z))
    xe = np.float32(T.recfast.xe(z))
    assert np.all(g["Tk_box"] == tk) and np.all(g["x_e_box"] == xe)
    cm = to.Cosmo(p)
    zf = float(np.float32(z))
    trad = to.TCMB * (1 + zf)
    nh = (1 - float(xe)) * cm.No * (1 + zf) ** 3
    ne = float(xe) * cm.N_b0 * (1 + zf) ** 3
    npr = float(xe) * cm.No * (1 + zf) ** 3
    t = float(tk)
    xc = to.T21 / trad / to.A10_HYPERFINE * (nh * T.kappa_10(t) + ne * T.kappa_elec(t) + npr * T.kappa_pH(t))
    ts = 1.0 / ((1.0 / trad + xc / t) / (1.0 + xc))
    assert np.allclose(g["TS_box"], ts, rtol=1e-6)
    assert 10.0 < t < 100.0 and trad > ts > t


@pytest.fixture(scope="module")
def engine_case():
    n = 32
    p = rg.make_params(n, 64.0, Flag_IncludeSpinTemp=1)
    zz, idx = wl.snapshot_redshifts(15.0)
    sf = np.zeros(len(zz))
    sf[idx - 1] = 2e-4
    return p, zz, idx, sf


def test_engine_shells_and_history_weights_match_oracle(engine_case):
    p, zz, idx, sf = engine_case
    nh = idx + 1
    shells, _, coef = rg.ts_tables(p, zz, idx, nh, 3e-4, 2.5e-4, sf, with_freq=False)
    rng = np.random.default_rng(3)
    hs = [rng.random((4, 4, 4)).astype(np.float32) for _ in range(nh)]
    sh, grids = to.shells_and_sources(oracle_params(p), zz, idx, hs[0], hs[0], hs, hs)
    assert np.allclose(sh.R, shells[0], rtol=1e-12, atol=0)
    assert np.allclose(sh.zpp_edge, shells[1], rtol=1e-12, atol=0)
    assert np.allclose(sh.zpp, shells[2], rtol=1e-12, atol=0)
    assert np.allclose(sh.dzpp, shells[3], rtol=1e-10, atol=0)
    assert np.allclose(sh.dt_dzpp, shells[4], rtol=1e-12, atol=0)
    used = 0
    for r in range(len(sh.R)):
        comb = sum(float(coef[r, k]) * hs[0 if k == 0 else k - 1].astype(np.float64) for k in range(nh + 1))
        want = grids[r][0].astype(np.float64)
        assert np.max(np.abs(comb - want)) <= 2e-6 * max(np.max(np.abs(want)), 1e-30), r
        used = max(used, int(np.max(np.nonzero(coef[r])[0], initial=0)))
    assert used >= 2          # the 40 shells reach back over several snapshots


def test_engine_frequency_tables_match_oracle(engine_case):
    p, zz, idx, sf = engine_case
    x_e_ave, cf = 3e-4, 2.5e-4
    shells, freq, _ = rg.ts_tables(p, zz, idx, idx + 1, x_e_ave, cf, sf)
    op = oracle_params(p)
    T = to.TsTables()
    sh, _ = to.shells_and_sources(op, zz, idx, None, None, [0] * (idx + 1), [0] * (idx + 1), want_grids=False)
    heat, ion, lya, sum_lyn = to.freq_tables(op, T, sh, zz[idx], x_e_ave, cf, zz, sf, idx)
    for got, want in ((freq[0], heat), (freq[1], ion), (freq[2], lya)):
        assert np.all(np.abs(got - want) <= 1e-6 * np.abs(want) + 1e-300)
    assert np.allclose(shells[5], sum_lyn, rtol=1e-12, atol=0)
    assert np.all(heat > 0) and np.all(lya > 0)


@pytest.mark.parametrize("flag", [1, 2, 3])
def test_engine_agn_tables_match_oracle(engine_case, flag):
    """The AGN X-ray band integrals (limits redshifted from zpp to zp, the band's spectral index)
    and the band prefactors of the library's host engine against the oracle."""
    p, zz, idx, sf = engine_case
    p = rg.rg_params.from_buffer_copy(p)
    p.Flag_IncludeAGNXray = flag
    p.TablesForXHeatingDir = rg.TABLES_DIR.encode()
    x_e_ave, cf = 3e-4, 2.5e-4
    agn, cz = rg.ts_agn_tables(p, zz, idx, idx + 1, x_e_ave, cf, sf)
    op = oracle_params(p)
    T = to.TsTables()
    sh, _ = to.shells_and_sources(op, zz, idx, None, None, [0] * (idx + 1), [0] * (idx + 1), want_grids=False)
    bands = [b for b, on in ((0, flag in (1, 3)), (1, flag in (1, 2))) if on]
    ft = to.freq_tables(op, T, sh, zz[idx], x_e_ave, cf, zz, sf, idx, agn_bands=tuple(bands))
    for b in (0, 1):
        for k in range(3):
            if b in bands:
                want = ft[4][b][k]
                assert np.all(np.abs(agn[b, k] - want) <= 1e-6 * np.abs(want) + 1e-300), (b, k)
                assert np.any(want != 0)
            else:
                assert np.all(agn[b, k] == 0)
    pf = to.prefactors(op, float(zz[idx]))
    assert cz[0] == pytest.approx(pf["const_zp"], rel=1e-12)
    assert cz[1] == pytest.approx(pf["const_agn"][0], rel=1e-12)
    assert cz[2] == pytest.approx(pf["const_agn"][1], rel=1e-12)

