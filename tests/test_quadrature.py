"""CPU checks of the quadrature rules of the learned grid and of the network's
numpy restatement (no GPU)."""
import numpy as np
import pytest

import mlp_ref
from william_ci_b200 import quadrature as Q


@pytest.mark.parametrize("n", [7, 10, 15, 20, 30])
def test_gauss_kronrod_exactness(n):
    u, wk, wg = Q.gauss_kronrod(n)
    assert len(u) == 2 * n + 1 and np.all(np.diff(u) > 0) and u[0] > 0 and u[-1] < 1
    # Kronrod exact to degree 3n+1 on [0,1]; embedded Gauss (n nodes) to 2n-1
    for k in range(0, 3 * n + 2):
        assert abs(np.dot(wk, u ** k) - 1.0 / (k + 1)) < 1e-14
    for k in range(0, 2 * n):
        assert abs(np.dot(wg, u ** k) - 1.0 / (k + 1)) < 1e-14
    assert np.count_nonzero(wg) == n
    # the Gauss nodes are those of Gauss-Legendre and interlace with the extension nodes
    x, w = np.polynomial.legendre.leggauss(n)
    np.testing.assert_allclose(np.sort(u[wg != 0]), np.sort(0.5 * (x + 1)), atol=1e-15)
    np.testing.assert_allclose(wg[wg != 0], 0.5 * w[np.argsort(x)], atol=1e-15)
    assert np.all(wg[1::2] != 0) and np.all(wg[0::2] == 0)


def test_rule_dictionary_shape_and_mapping():
    d = Q.rule_dictionary()
    assert len(d) == len(Q.RULE_ORDERS) * len(Q.RULE_SCALES) == 105
    for s, n, t, wk, wg in d:
        assert len(t) == 2 * n + 1 <= 64
        # mapped rule integrates the t-space test function 1/(1+t)^2 exactly enough
        ref = 1.0
        val = np.dot(wk, 1.0 / (1.0 + t) ** 2)
        if 0.3 <= s <= 3.0 and n >= 10:
            assert abs(val - ref) < 1e-9
    # a panel rule is the [0,1] rule placed on [a,b]
    t, wk, wg = Q.mapped_rule(7, 0.6, 0.25, 0.5)
    u = t / (0.6 + t)
    assert np.all((u > 0.25) & (u < 0.5))
    assert abs(np.sum(wk * (0.6 / (0.6 + t) ** 2)) - 0.25) < 1e-14   # int of du over the panel


def test_mapped_gauss_legendre_matches_reference_map():
    t, w = Q.mapped_gauss_legendre(32, 0.6)
    assert np.all(np.diff(t) > 0)
    # int_0^inf dt/(1+t)^2 = 1 (a smooth rational function of u under the map)
    assert abs(np.dot(w, 1.0 / (1.0 + t) ** 2) - 1.0) < 1e-13
    # the same nodes as the oracle's fast_quad restatement
    import pyoracle
    to, wo = pyoracle.fast_quad(32)
    np.testing.assert_allclose(t, to, rtol=1e-13)
    np.testing.assert_allclose(w, wo, rtol=1e-12)


def test_judge_estimate_formula():
    from william_ci_b200.learned_grid import judge_estimate
    K = np.array([1.0, 2.0, 0.5, 1e-3])
    G = np.array([1.0 + 1e-9, 2.0, 0.5, 1e-3 + 1e-12])
    offs = np.array([0, 3, 4])
    est = judge_estimate(K, G, offs)
    assert est[0] == pytest.approx(2.0 * (200 * 1e-9 / 2.0) ** 1.5, rel=1e-6)
    assert est[1] == pytest.approx(1e-3 * (200 * 1e-12 / 1e-3) ** 1.5, rel=1e-3)
    # a rule that misses by more than the block scale estimates the scale itself
    assert judge_estimate(np.array([1.0]), np.array([0.0]), np.array([0, 1]))[0] == 1.0


def test_mlp_oracle_gradient_finite_differences():
    rng = np.random.default_rng(0)
    nf, nh, nc, B = 5, 7, 4, 11
    npar = nh * nf + nh + nh * nh + nh + nc * nh + nc
    p = rng.standard_normal(npar) * 0.5
    mu, sig = rng.standard_normal(nf), rng.random(nf) + 0.5
    X = rng.standard_normal((B, nf))
    Y = (rng.random((B, nc)) < 0.5).astype(float)
    L, g = mlp_ref.loss_grad(p, mu, sig, X, Y, nf, nh, nc)
    h = 1e-6
    for i in rng.choice(npar, 25, replace=False):
        e = np.zeros(npar)
        e[i] = h
        fd = (mlp_ref.loss_grad(p + e, mu, sig, X, Y, nf, nh, nc)[0] -
              mlp_ref.loss_grad(p - e, mu, sig, X, Y, nf, nh, nc)[0]) / (2 * h)
        assert abs(fd - g[i]) < 1e-6 * max(1.0, abs(g[i]))


def test_library_kronrod_rules_equal_the_exact_ones():
    """libtce's Gauss-Kronrod rules (Laurie's algorithm, extended precision,
    tce_gk_rule) against the ones built here from the definition in 60-digit
    arithmetic, and the dictionary tce_lg_setup loads against the host's."""
    from william_ci_b200 import engine as E
    from william_ci_b200 import learned_grid as LG
    for n in Q.RULE_ORDERS + (1, 3):
        u, wk, wg = E.gk_rule(n)
        u2, wk2, wg2 = Q.gauss_kronrod(n)
        assert np.abs(u - u2).max() < 1e-15 and np.abs(wk - wk2).max() < 1e-15 and np.abs(wg - wg2).max() < 1e-15
    lib_rules = E.lg_dictionary()
    host_rules, _ = LG.dictionary()
    assert len(lib_rules) == len(host_rules)
    for a, b in zip(lib_rules, host_rules):
        for x, y in zip(a, b):
            assert x.shape == y.shape
            assert np.abs(x - y).max() <= 1e-15 * np.abs(y).max()
