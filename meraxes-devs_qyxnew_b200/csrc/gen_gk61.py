"""Generate rg_gk61.h: the 61-point Gauss-Kronrod rule (Kronrod extension of the
30-point Gauss-Legendre rule) on [-1, 1], computed here in 60-digit arithmetic.

The reference integrates with GSL's QAG using the GSL_INTEG_GAUSS61 rule
(src/core/XRayHeatingFunctions.c:400,846).  The rule's nodes and weights are a
mathematical object; this script derives them instead of copying a table:

* the Gauss nodes are the roots of P_30, with weights 2 / ((1 - x^2) P_30'(x)^2);
* the 31 added Kronrod nodes are the roots of the Stieltjes polynomial E_31, the
  degree-31 polynomial orthogonal to x^k P_30(x) for k = 0..30 (found from its
  Legendre expansion, whose coefficients solve a linear system);
* the Kronrod weights make the 61-node rule exact for P_0 .. P_60, and the check
  below confirms exactness up to degree 91 = 3n + 1.

Run:  python gen_gk61.py   (writes rg_gk61.h next to this file)
"""

import os

import mpmath as mp

mp.mp.dps = 60
N = 30


def legendre_all(x, nmax):
    p = [mp.mpf(1), x]
    for k in range(1, nmax):
        p.append(((2 * k + 1) * x * p[k] - k * p[k - 1]) / (k + 1))
    return p[: nmax + 1]


def gauss_legendre(n):
    nodes, weights = [], []
    for i in range(1, n + 1):
        x = mp.cos(mp.pi * (i - mp.mpf(1) / 4) / (n + mp.mpf(1) / 2))
        for _ in range(100):
            p = legendre_all(x, n)
            dp = n * (x * p[n] - p[n - 1]) / (x * x - 1)
            dx = p[n] / dp
            x -= dx
            if abs(dx) < mp.mpf(10) ** (-mp.mp.dps + 5):
                break
        p = legendre_all(x, n)
        dp = n * (x * p[n] - p[n - 1]) / (x * x - 1)
        nodes.append(x)
        weights.append(2 / ((1 - x * x) * dp * dp))
    return nodes, weights


def main():
    # exact integration helper: a 64-point Gauss-Legendre rule (exact to degree 127)
    qx, qw = gauss_legendre(64)

    def integ(f):
        return mp.fsum(w * f(x) for x, w in zip(qx, qw))

    # E_31 = P_31 + sum_{j = 29, 27, ..., 1} c_j P_j ; orthogonal to x^k P_30, k = 0..30.
    # By parity only odd k give nontrivial conditions: k = 1, 3, ..., 29 (15 equations)
    js = list(range(N - 1, 0, -2))          # 29, 27, ..., 1  (15 unknowns)
    ks = list(range(1, N, 2))               # 1, 3, ..., 29
    A = mp.matrix(len(ks), len(js))
    rhs = mp.matrix(len(ks), 1)
    cache = {}

    def leg(x):
        if x not in cache:
            cache[x] = legendre_all(x, N + 1)
        return cache[x]

    for a, k in enumerate(ks):
        for b, j in enumerate(js):
            A[a, b] = integ(lambda x: leg(x)[j] * leg(x)[N] * x ** k)
        rhs[a] = -integ(lambda x: leg(x)[N + 1] * leg(x)[N] * x ** k)
    c = mp.lu_solve(A, rhs)
    coef = {N + 1: mp.mpf(1)}
    for b, j in enumerate(js):
        coef[j] = c[b]

    def E(x):
        p = legendre_all(x, N + 1)
        return mp.fsum(cj * p[j] for j, cj in coef.items())

    gx, gw = gauss_legendre(N)
    gx = sorted(gx)
    # Kronrod nodes interlace with the Gauss nodes: one in each gap and one outside each end
    brackets = [(mp.mpf(-1), gx[0])] + [(gx[i], gx[i + 1]) for i in range(N - 1)] + [(gx[-1], mp.mpf(1))]
    kx = []
    for lo, hi in brackets:
        flo, fhi = E(lo), E(hi)
        assert flo * fhi < 0, "Stieltjes root not bracketed"
        for _ in range(250):
            mid = (lo + hi) / 2
            fm = E(mid)
            if fm * flo <= 0:
                hi = mid
            else:
                lo, flo = mid, fm
        kx.append((lo + hi) / 2)
    # E_31 is odd, so its middle root is exactly 0
    kx = [mp.mpf(0) if abs(v) < mp.mpf(10) ** -40 else v for v in kx]
    nodes = sorted(gx + kx)
    assert len(nodes) == 2 * N + 1 and nodes[N] == 0
    # weights: exact for P_0 .. P_60
    M = mp.matrix(2 * N + 1, 2 * N + 1)
    b = mp.matrix(2 * N + 1, 1)
    for i in range(2 * N + 1):
        for jx, x in enumerate(nodes):
            M[i, jx] = leg_any(x, i)
        b[i] = 2 if i == 0 else 0
    w = mp.lu_solve(M, b)
    # exactness check up to degree 3N + 1 = 91
    for deg in range(0, 3 * N + 2):
        exact = mp.mpf(2) / (deg + 1) if deg % 2 == 0 else mp.mpf(0)
        got = mp.fsum(w[i] * nodes[i] ** deg for i in range(2 * N + 1))
        assert abs(got - exact) < mp.mpf(10) ** -40, deg
    # Gauss weights on the Gauss nodes (for the embedded error estimate)
    gmap = {str(x): wt for x, wt in zip(*gauss_legendre(N))}
    # positive half, decreasing abscissa, with the centre last
    half = [i for i in range(2 * N + 1) if nodes[i] >= 0]
    half.sort(key=lambda i: -nodes[i])
    lines = []
    lines.append("// Generated by gen_gk61.py: 61-point Gauss-Kronrod rule on [-1, 1] (see that script).")
    lines.append("#pragma once")
    lines.append("namespace rg {")
    lines.append("// abscissae x_k >= 0 in decreasing order (x_30 = 0), Kronrod weights wk_k, and the Gauss")
    lines.append("// weight wg_k of the same node (0 for the nodes only the Kronrod rule has)")
    xs, wks, wgs = [], [], []
    gsorted = sorted(gauss_legendre(N)[0])
    for i in half:
        x = nodes[i]
        xs.append(x)
        wks.append(w[i])
        g = 0
        for gxv, gwv in zip(*gauss_legendre(N)):
            if abs(gxv - x) < mp.mpf(10) ** -40:
                g = gwv
        wgs.append(g)
    fmt = lambda v: mp.nstr(v, 25, min_fixed=-1, max_fixed=-1) if v != 0 else "0.0"
    lines.append("constexpr int GK61_HALF = %d;" % len(xs))
    lines.append("constexpr double GK61_X[%d] = {%s};" % (len(xs), ", ".join(fmt(v) for v in xs)))
    lines.append("constexpr double GK61_WK[%d] = {%s};" % (len(xs), ", ".join(fmt(v) for v in wks)))
    lines.append("constexpr double GK61_WG[%d] = {%s};" % (len(xs), ", ".join(fmt(v) for v in wgs)))
    lines.append("}  // namespace rg")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rg_gk61.h")
    open(out, "w").write("\n".join(lines) + "\n")
    print("wrote", out)


def leg_any(x, n):
    return legendre_all(x, max(n, 1))[n]


if __name__ == "__main__":
    main()
