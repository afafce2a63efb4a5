"""The 61-point Gauss-Kronrod rule on [-1, 1] -- TEST INFRASTRUCTURE ONLY (the oracle's side).

The reference integrates with GSL's QAG and the GSL_INTEG_GAUSS61 rule
(src/core/XRayHeatingFunctions.c:400, 846).  The rule is a mathematical object:
the 30-point Gauss-Legendre rule plus the 31 Kronrod nodes that make the 61-node
rule exact for polynomials of degree 3*30 + 1 = 91.  This module computes it
from that definition in 80-digit arithmetic, working in monomials of y = x^2
(the rule is symmetric):

* Gauss nodes: roots of P_30, a degree-15 polynomial in y;
* Kronrod nodes: 0 and the roots of the Stieltjes polynomial E_31(x) = x Q(x^2),
  Q monic of degree 15 with integral(E_31 P_30 x^k) = 0 for k = 1, 3, ..., 29;
* weights: the symmetric moment equations (exactness for x^0, x^2, ...).

It is independent of the product's generator (which works in the Legendre
basis); a CPU test compares the two tables.
"""

from __future__ import annotations

import functools

import mpmath as mp
import numpy as np

N = 30


def _legendre_coeffs(n: int) -> list:
    """Monomial coefficients c[k] of P_n (exact rationals via the three-term recurrence)."""
    p0 = [mp.mpf(1)]
    p1 = [mp.mpf(0), mp.mpf(1)]
    if n == 0:
        return p0
    for k in range(1, n):
        nxt = [mp.mpf(0)] * (k + 2)
        for i, c in enumerate(p1):
            nxt[i + 1] += (2 * k + 1) * c / (k + 1)
        for i, c in enumerate(p0):
            nxt[i] -= k * c / (k + 1)
        p0, p1 = p1, nxt
    return p1


def _moment(k: int):
    """integral_{-1}^{1} x^k dx."""
    return mp.mpf(0) if k % 2 else mp.mpf(2) / (k + 1)


def _even_roots(coeffs_y: list) -> list:
    """Roots in (0, 1) of the polynomial sum c[j] y^j, as positive x = sqrt(y), descending."""
    roots = mp.polyroots(list(reversed(coeffs_y)), maxsteps=400, extraprec=400)
    xs = sorted((mp.sqrt(mp.re(r)) for r in roots), reverse=True)
    return xs


@functools.lru_cache(maxsize=1)
def rule():
    """(xgk[31], wgk[31], wg[30]) in QUADPACK's order: xgk descending with xgk[30] = 0;
    wg[k] is the Gauss weight of node xgk[k] (zero for Kronrod-only nodes)."""
    with mp.workdps(80):
        P = _legendre_coeffs(N)                       # degree 30, even
        gauss = _even_roots([P[2 * j] for j in range(N // 2 + 1)])
        # Q(y) = y^15 + sum_{j<15} q_j y^j ; E(x) = x Q(x^2) = sum q_j x^{2j+1}
        m = N // 2
        A = mp.matrix(m, m)
        rhs = mp.matrix(m, 1)
        for a, k in enumerate(range(1, N, 2)):
            # integral(x^{2j+1} P_30(x) x^k) = sum_i P[i] moment(2j+1+i+k)
            def pint(power):
                return mp.fsum(P[i] * _moment(power + i) for i in range(len(P)))
            for j in range(m):
                A[a, j] = pint(2 * j + 1 + k)
            rhs[a] = -pint(2 * m + 1 + k)
        q = mp.lu_solve(A, rhs)
        kron = _even_roots([q[j] for j in range(m)] + [mp.mpf(1)])
        nodes = sorted(gauss + kron, reverse=True) + [mp.mpf(0)]     # 30 positive + centre
        # Kronrod weights: sum_i w_i * 2 x_i^{2e} + w_c [e == 0] = 2 / (2e + 1), e = 0..30
        M = mp.matrix(N + 1, N + 1)
        b = mp.matrix(N + 1, 1)
        for e in range(N + 1):
            for i, x in enumerate(nodes):
                M[e, i] = (x ** (2 * e)) * (1 if i == N else 2)
            b[e] = mp.mpf(2) / (2 * e + 1)
        wk = mp.lu_solve(M, b)
        # Gauss weights: 15 positive nodes, exact for y^e, e = 0..14
        G = mp.matrix(m, m)
        gb = mp.matrix(m, 1)
        for e in range(m):
            for i, x in enumerate(gauss):
                G[e, i] = 2 * x ** (2 * e)
            gb[e] = mp.mpf(2) / (2 * e + 1)
        wgs = mp.lu_solve(G, gb)
        gmap = {float(x): float(w) for x, w in zip(gauss, wgs)}
        xgk = np.array([float(x) for x in nodes])
        wgk = np.array([float(w) for w in wk])
        wg = np.array([gmap.get(float(x), 0.0) for x in nodes[:N]])
    return xgk, wgk, wg
