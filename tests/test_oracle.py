"""CPU tests of the oracle: known answers derived from the reference code.

The reference has no golden vectors for this path (its regression tests need a
dataset that is not available), so the restatement is pinned here by
closed-form and code-derived answers.
"""

import math

import numpy as np
import pytest

import reion_oracle as ro
import tables
import workloads as wl
from helpers import install_recfast


def test_radius_schedule_counts():
    # counts re-derived from find_HII_bubbles.c:279-285,546 for the benchmark configurations
    cases = [(64, 64.0, 8.0, 50.0, 44), (256, 250.0, 7.0, 50.0, 42), (512, 500.0, 8.0, 1000.0, 61),
             (96, 96.0, 8.0, 50.0, 47), (128, 128.0, 8.0, 50.0, 47), (192, 192.0, 8.0, 50.0, 47)]
    for n, box, z, rmax, want in cases:
        p = ro.Params(ReionGridDim=n, BoxSize=box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=rmax)
        s = ro.radius_schedule(p, z)
        assert len(s) == want, (n, len(s))
        assert s[-1][1] and not any(last for _, last in s[:-1])
        # last radius is the cell size times L_FACTOR, or the cell size when cells are < 1 Mpc/h
        cell = box / n
        assert s[-1][0] == pytest.approx((1.0 if cell < 1.0 else ro.L_FACTOR) * cell)
        # radii decrease by ReionDeltaRFactor
        for (r0, _), (r1, _) in zip(s[:-2], s[1:-1]):
            assert r1 == pytest.approx(r0 / 1.1)


def test_radius_schedule_evolving_rmax():
    p = ro.Params(ReionGridDim=64, BoxSize=500.0, Flag_EvolvingReionRBubbleMax=1)
    assert ro.radius_schedule(p, 8.0)[0][0] == pytest.approx(25.483241248322766)
    assert ro.radius_schedule(p, 5.0)[0][0] == pytest.approx(112.0 * (6.0 / 5.0) ** -4.4)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_window_closed_forms(precision):
    n, box, R = 16, 20.0, 3.0
    k = ro.kmag(n, box, precision).astype(np.float64)
    w0 = ro.window(n, box, R, 0, precision)
    assert w0[0, 0, 0] == 1.0
    kr = k * R
    m = kr > 1e-3
    ref = 3.0 * (np.sin(kr[m]) / kr[m] ** 3 - np.cos(kr[m]) / kr[m] ** 2)
    tol = 2e-5 if precision == "fp32" else 1e-12
    assert np.max(np.abs(w0[m] - ref)) < tol
    w1 = ro.window(n, box, R, 1, precision)
    assert set(np.unique(w1)) <= {0.0, 1.0}
    assert np.all(w1[kr * 0.413566994 < 0.999] == 1.0) and np.all(w1[kr * 0.413566994 > 1.001] == 0.0)
    w2 = ro.window(n, box, R, 2, precision)
    assert np.max(np.abs(w2 - np.exp(-(0.643 * kr) ** 2 / 2))) < (1e-6 if precision == "fp32" else 1e-14)
    with pytest.raises(ValueError):
        ro.window(n, box, R, 3, precision)


def test_fft_roundtrip():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((24, 24, 24))
    for prec, tol in (("fp64", 1e-13), ("fp32", 2e-6)):
        back = ro.inverse(ro.forward(x, prec), 24)
        assert np.max(np.abs(back - x)) < tol * 10


def test_uniform_field_known_answer():
    """A uniform box: every filtered field equals the mean, so the answer is analytic."""
    install_recfast()
    n, box, z = 16, 32.0, 8.0
    p = ro.Params(ReionGridDim=n, BoxSize=box, Flag_EvolvingReionRBubbleMax=0, ReionRBubbleMax=20.0)
    u = ro.run_units(p)
    cell_mass = p.OmegaM * u.RhoCrit * (box / n) ** 3
    # f_coll_prefactor * stars = eff * stars / (V_cell * OmegaM * RhoCrit) for the top-hat RtoM
    for frac, ionized in ((0.5, False), (2.0, True)):
        stars = np.full((n, n, n), frac * cell_mass / 100.0, np.float64)
        p.ReionEfficiency = 100.0
        st = ro.HIIState.fresh(n)
        xH, rb, s, _ = ro.find_hii_bubbles(p, z, wl.to_padded(np.zeros((n, n, n))), wl.to_padded(stars),
                                          wl.to_padded(np.zeros((n, n, n))), st, "fp64")
        if ionized:
            assert np.all(xH == 0) and np.all(st.z_at_ionization == np.float32(z))
        else:
            assert np.allclose(xH, 1.0 - frac, atol=1e-6)
            assert np.all(st.z_at_ionization == -1)
        assert np.all(rb == 0)           # r_bubble is only written with recombinations on
        assert s["volume_weighted_global_xH"] == pytest.approx(0.0 if ionized else 1.0 - frac, abs=1e-6)


def test_fully_ionized_temperature_same_redshift():
    # z_re == z: result = (1 * T_RE^1.7 + (1e4 (1+z)/4)^1.7 (1+delta))^0.5882
    z, d = 8.0, 0.3
    want = (1e4 ** 1.7 + (1e4 * (1 + z) / 4) ** 1.7 * (1 + d)) ** 0.5882
    got = ro.fully_ionized_temperature(np.array([z], np.float32), z, np.array([d], np.float32))[0]
    assert got == pytest.approx(want, rel=1e-6)


def test_delta_T_uniform_neutral_box():
    n = 8
    p = ro.Params(ReionGridDim=n, BoxSize=8.0)
    dT, ave = ro.delta_T(p, 10.0, np.ones((n, n, n), np.float32), wl.to_padded(np.zeros((n, n, n))))
    ob = p.OmegaM * p.BaryonFrac
    cf = 27.0 * (ob * p.Hubble_h ** 2 / 0.023) * math.sqrt(0.15 / p.OmegaM / p.Hubble_h ** 2 * 11.0 / 10.0)
    assert ave == pytest.approx(cf, rel=1e-6)
    assert np.allclose(dT, cf, rtol=1e-6)


def test_tables_and_recfast_spline():
    r = tables.Recfast(tables.default_tables_dir())
    # the spline passes through the knots and is monotone between low-z knots
    assert r.T(float(r.z[100])) == pytest.approx(r.tk[100], rel=1e-6)
    assert r.T(501.0) == -1.0
    e, fheat, nlya, nhi, nhei, nheii = tables.read_x_int_tables(tables.default_tables_dir())
    assert e.shape == (258,) and fheat.shape == (14, 258)
    assert e[0] == np.float32(10.0)
    lt, lk = tables.read_kappa(tables.default_tables_dir(), "kappa_eH_table.dat", 20)
    assert lt[0] == pytest.approx(0.0)
