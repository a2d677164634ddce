"""t-quadrature rules for the ERI t-integral (2/sqrt(pi)) int_0^inf f(t) dt.

Every rule lives on u in [0,1] and is mapped by t = s u/(1-u), dt = s/(1-u)^2 du,
the map of the reference's fast_quad rule (precompute_t.f90:906-942, s = 0.6).

* mapped_gauss_legendre(n, s): the reference rule for s = 0.6.
* gauss_kronrod(n): the (2n+1)-point Kronrod extension of the n-point
  Gauss-Legendre rule on [0,1] with the embedded Gauss weights, built from the
  definition: the extension nodes are the zeros of the Stieltjes polynomial
  E_{n+1} (monic, int_{-1}^{1} P_n E_{n+1} x^k dx = 0 for k = 0..n), solved
  exactly in rational arithmetic; the weights make the rule exact for every
  polynomial of degree <= 2n (then it is exact to 3n+1).  Roots and weights
  are computed with 60 significant digits and rounded to double.
* mapped_rule(x, wk, wg, s, a, b): a [0,1] rule placed on the panel [a,b] of u
  and mapped to t, giving t nodes, Kronrod weights and Gauss weights.

The rule dictionary of the learned grid is the set of mapped Kronrod rules
over scales s_j = 0.6 * 2^(j/2) and orders n (RULE_SCALES, RULE_ORDERS).
"""
from __future__ import annotations

import functools
from fractions import Fraction
from typing import List, Tuple

import numpy as np

RULE_ORDERS = (7, 10, 15, 20, 30)      # K15, K21, K31, K41, K61
RULE_SCALES = tuple(0.6 * 2.0 ** (j / 2.0) for j in range(-18, 3))


def mapped_gauss_legendre(n: int, s: float = 0.6) -> Tuple[np.ndarray, np.ndarray]:
    x, w = np.polynomial.legendre.leggauss(n)
    u = 0.5 * (x[::-1] * -1 + 1)        # ascending u
    u = np.sort(0.5 * (1 + x))
    wu = 0.5 * w[np.argsort(0.5 * (1 + x))]
    return s * u / (1 - u), wu * s / (1 - u) ** 2


def _legendre_coeffs(n: int) -> List[Fraction]:
    """Monomial coefficients (ascending) of P_n, Bonnet recurrence in rationals."""
    p0, p1 = [Fraction(1)], [Fraction(0), Fraction(1)]
    if n == 0:
        return p0
    for k in range(1, n):
        nxt = [Fraction(0)] * (k + 2)
        for i, c in enumerate(p1):
            nxt[i + 1] += Fraction(2 * k + 1, k + 1) * c
        for i, c in enumerate(p0):
            nxt[i] -= Fraction(k, k + 1) * c
        p0, p1 = p1, nxt
    return p1


def _moment(m: int) -> Fraction:
    return Fraction(2, m + 1) if m % 2 == 0 else Fraction(0)


def _solve_rational(A: List[List[Fraction]], b: List[Fraction]) -> List[Fraction]:
    n = len(b)
    M = [row[:] + [bi] for row, bi in zip(A, b)]
    for col in range(n):
        piv = next(r for r in range(col, n) if M[r][col] != 0)
        M[col], M[piv] = M[piv], M[col]
        for r in range(n):
            if r != col and M[r][col] != 0:
                f = M[r][col] / M[col][col]
                M[r] = [x - f * y for x, y in zip(M[r], M[col])]
    return [M[i][n] / M[i][i] for i in range(n)]


@functools.lru_cache(maxsize=None)
def gauss_kronrod(n: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(2n+1) nodes on [0,1] (ascending), Kronrod weights, Gauss weights (0 off the Gauss nodes)."""
    import mpmath as mp
    mp.mp.dps = 60
    P = _legendre_coeffs(n)
    # E_{n+1} = x^{n+1} + sum_{j<=n} e_j x^j with int P_n E x^k = 0, k = 0..n
    def ipx(m):    # int_{-1}^{1} P_n(x) x^m dx
        return sum(c * _moment(i + m) for i, c in enumerate(P))
    A = [[ipx(j + k) for j in range(n + 1)] for k in range(n + 1)]
    b = [-ipx(n + 1 + k) for k in range(n + 1)]
    e = _solve_rational(A, b) + [Fraction(1)]
    to_mp = lambda q: mp.mpf(q.numerator) / q.denominator  # noqa: E731
    xs_e = mp.polyroots([to_mp(c) for c in reversed(e)], maxsteps=400, extraprec=400)
    xs_g = mp.polyroots([to_mp(c) for c in reversed(P)], maxsteps=400, extraprec=400)
    xs_e = [mp.re(x) for x in xs_e]
    xs_g = [mp.re(x) for x in xs_g]
    nodes = sorted(xs_g + xs_e)
    N = len(nodes)
    # Kronrod weights: exact for x^k, k = 0..2n
    V = mp.matrix(N, N)
    rhs = mp.matrix(N, 1)
    for k in range(N):
        for i, x in enumerate(nodes):
            V[k, i] = x ** k
        rhs[k] = to_mp(_moment(k))
    wk = mp.lu_solve(V, rhs)
    # Gauss weights 2 / ((1 - x^2) P_n'(x)^2)
    dP = [i * c for i, c in enumerate(P)][1:]
    wg = []
    for x in nodes:
        if any(abs(x - g) < mp.mpf(10) ** -40 for g in xs_g):
            d = sum(to_mp(c) * x ** i for i, c in enumerate(dP))
            wg.append(2 / ((1 - x * x) * d * d))
        else:
            wg.append(mp.mpf(0))
    u = np.array([float((x + 1) / 2) for x in nodes])
    return u, np.array([float(w / 2) for w in wk]), np.array([float(w / 2) for w in wg])


def mapped_rule(n: int, s: float, a: float = 0.0, b: float = 1.0):
    """Kronrod rule of order n on the u-panel [a,b], mapped by t = s u/(1-u)."""
    u, wk, wg = gauss_kronrod(n)
    uu = a + (b - a) * u
    jac = (b - a) * s / (1 - uu) ** 2
    return s * uu / (1 - uu), wk * jac, wg * jac


def rule_dictionary():
    """All (scale, order) rules of the learned grid: list of (s, n, t, wk, wg)."""
    out = []
    for n in RULE_ORDERS:
        for s in RULE_SCALES:
            t, wk, wg = mapped_rule(n, s)
            out.append((s, n, t, wk, wg))
    return out
