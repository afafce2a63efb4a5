"""CPU checks of the recombination-table oracle (splined_recombination restatement) and of the
recombination branch of the find_HII_bubbles oracle.  Known answers: the natural spline
interpolates its knots, reproduces straight lines, matches scipy's natural CubicSpline and an
independent dense solve; the out-of-table branches return the reference's constants; a box
without sources keeps N_rec and Gamma12 at zero."""

import numpy as np
import pytest
from scipy.interpolate import CubicSpline

import reion_oracle as ro
import rec_oracle as rco
import workloads as wl
from helpers import install_recfast


def test_knots_are_float_sums():
    k = rco.knots()
    assert k.size == 150 and k[0] == -10.0
    assert k[1] == float(np.float32(-9.9)) and np.all(np.diff(k) > 0)
    t = rco.synthetic_tables(4, 3, 150)
    assert t.lng_hi == k[-1]


def test_natural_spline_matches_dense_solve_and_scipy():
    rng = np.random.default_rng(3)
    x = np.sort(rng.random(12)) * 5
    y = rng.standard_normal((4, 12))
    c = rco.natural_half_curvature(x, y)
    n = x.size
    h = np.diff(x)
    A = np.zeros((n, n))
    rhs = np.zeros((4, n))
    A[0, 0] = A[-1, -1] = 1.0
    for i in range(1, n - 1):
        A[i, i - 1], A[i, i], A[i, i + 1] = h[i - 1], 2 * (h[i - 1] + h[i]), h[i]
        rhs[:, i] = 3 * ((y[:, i + 1] - y[:, i]) / h[i] - (y[:, i] - y[:, i - 1]) / h[i - 1])
    dense = np.linalg.solve(A, rhs.T).T
    assert np.allclose(c, dense, rtol=1e-12, atol=1e-12)
    sp = CubicSpline(x, y[0], bc_type="natural")
    assert np.allclose(2 * c[0], sp(x, 2), rtol=1e-10, atol=1e-10)


def test_splined_values_match_scipy_and_knots():
    t = rco.synthetic_tables(10, 8, 150)
    z_ct, t_ct = 7, 5
    z_eff = np.full(50, z_ct * rco.Z_DEL + 0.03)
    temp = np.full(50, 10 ** (rco.T_STA + t_ct * rco.T_DEL + 0.004))
    lng = np.linspace(-9.95, 4.8, 50)
    rate, rnh, cf = t.splined(z_eff, np.exp(lng), temp)
    row = z_ct * t.nt + t_ct
    for k, got in ((0, np.log(rate)), (1, cf), (2, np.log(rnh))):
        want = CubicSpline(t.knots, t.y[k, row], bc_type="natural")(lng)
        assert np.allclose(got, want, rtol=1e-12, atol=1e-10)
    # at the knots the spline returns the table
    r2, n2, c2 = t.splined(z_eff[:20], np.exp(t.knots[3:23]), temp[:20])
    assert np.allclose(c2, t.y[1, row, 3:23], rtol=1e-13)


def test_splined_out_of_table_branches():
    t = rco.synthetic_tables(10, 8, 150)
    # Gamma12 = 0 (log -inf) and below the table, temperature below 10^2 K: the no-recombination values
    rate, rnh, cf = t.splined(np.array([5.0, 5.0, 5.0]), np.array([0.0, np.exp(-10.5), 1.0]),
                              np.array([1e4, 1e4, 50.0]))
    assert np.all(rate == 0) and np.all(rnh == 1e4) and np.all(cf == 1.0)
    # above the table in Gamma12, z and T: clamped to the last sample
    r1, _, c1 = t.splined(np.array([1e3]), np.array([np.exp(9.0)]), np.array([1e9]))
    r2, _, c2 = t.splined(np.array([(t.nz - 1) * rco.Z_DEL]), np.array([np.exp(t.lng_hi - 1e-7)]),
                          np.array([10 ** (rco.T_STA + (t.nt - 1) * rco.T_DEL)]))
    assert r1 == pytest.approx(r2[0], rel=1e-12) and c1 == pytest.approx(c2[0], rel=1e-12)
    # negative effective redshift rounds into the first row
    r3, _, _ = t.splined(np.array([-0.3]), np.array([1.0]), np.array([1e4]))
    r4, _, _ = t.splined(np.array([0.0]), np.array([1.0]), np.array([1e4]))
    assert r3[0] == r4[0]


def test_find_hii_without_sources_keeps_recombination_state():
    install_recfast()
    n, box = 16, 20.0
    src = wl.make_sources(n, box, seed=5)
    zero = np.zeros_like(src.stars)
    p = ro.Params(ReionGridDim=n, BoxSize=box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=10.0,
                  ReionEfficiency=4000.0, Flag_IncludeRecombinations=1)
    st = ro.HIIState.fresh(n, rec=True)
    xH, rb, s, d = ro.find_hii_bubbles(p, 8.0, src.deltax, zero, zero, st, "fp64", rec_tables=rco.synthetic_tables(),
                                       prev_z=8.3)
    assert np.all(xH == 1) and np.all(rb == 0) and np.all(st.Gamma12 == 0) and np.all(st.N_rec == 0)
    assert np.all(d["rec"]["residual_xH"] == np.float32(1e4)) and np.all(d["rec"]["clumping_factor"] == 1)
    assert np.all(d["rec"]["t_resp"] == np.float32(1e30))
    assert s["volume_weighted_global_N_rec"] == 0 and s["volume_weighted_global_clumping_factor"] == 1


def test_find_hii_recombinations_raise_the_barrier():
    """N_rec > 0 from a previous snapshot can only keep cells neutral (the barrier is 1 + N_rec)."""
    install_recfast()
    n, box = 32, 32.0
    src = wl.make_sources(n, box, seed=77)
    tabs = rco.synthetic_tables()
    p = ro.Params(ReionGridDim=n, BoxSize=box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=50.0,
                  ReionEfficiency=20000.0, Flag_IncludeRecombinations=1)
    st0 = ro.HIIState.fresh(n, rec=True)
    xa, _, _, _ = ro.find_hii_bubbles(p, 8.0, src.deltax, src.stars, src.sfr, st0.copy(), "fp64", rec_tables=tabs,
                                      prev_z=8.0)
    st1 = st0.copy()
    st1.N_rec[:] = 0.5
    xb, _, _, _ = ro.find_hii_bubbles(p, 8.0, src.deltax, src.stars, src.sfr, st1, "fp64", rec_tables=tabs,
                                      prev_z=8.0)
    ion_a, ion_b = xa < ro.REL_TOL, xb < ro.REL_TOL
    assert ion_a.sum() > ion_b.sum() > 0 and not np.any(ion_b & ~ion_a)
