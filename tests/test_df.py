"""Density fitting for k-MP2 on the CPU: the product's k-space algebra
(william_ci_b200/df.py: fit_B, L_vectors, chol_factor) against the literal
restatement of df_init / df_L_kap (oracle/df_ref.py), both fed the C oracle's
3- and 2-index integrals on the orbital + auxiliary + dummy system; MP2 from
the L vectors with the numpy restatement of kMP2_calc."""
import numpy as np
import pytest

import df_ref
import mp2_ref
import pyoracle as po
from test_scf import dimer_chain, rhf_inputs


@pytest.fixture(scope="module")
def dimer_df():
    from william_ci_b200 import df, scf
    from william_ci_b200 import system as S
    ao = dimer_chain(4)
    cell = S.Cell("Tori1D", (4, 1, 1), 4.0, (16.0, 0.0, 0.0), [("H", (0.0, 0.0, 0.0)), ("H", (1.4, 0.0, 0.0))])
    aux = S.build_system(cell, df.even_tempered_aux(ao.charges))
    po.normalize(aux)
    dfs = df.df_system(ao, aux)
    orc = po.Oracle(dfs.sys)
    sh, nshuc, _ = orc.shells()
    Vm, T3 = df_ref.integrals(orc, dfs, sh, nshuc)
    o, St, Tt, Vt, en, nO = rhf_inputs(ao)
    r = scf.rhf_sao(St, Tt, Vt, en, nO, ao.nfuc, ao.ncell, lambda P: o.direct_jk(P)[:2])
    assert r.converged
    return dfs, Vm, T3, r


def test_chol_factor_whitens_the_metric():
    from william_ci_b200 import df
    rng = np.random.default_rng(1)
    A = rng.standard_normal((9, 6)) + 1j * rng.standard_normal((9, 6))
    V = A @ A.conj().T                                   # rank 6
    f, nd = df.chol_factor(V, 1e-10)
    assert nd == 3
    P = f.conj().T @ V @ f
    np.testing.assert_allclose(P[:6, :6], np.eye(6), atol=1e-10)
    np.testing.assert_allclose(f, df_ref.chol_f(V, 1e-10), atol=1e-12)


def test_fitted_vectors_and_L_match_the_restatement(dimer_df):
    from william_ci_b200 import df
    dfs, Vm, T3, r = dimer_df
    ncl = dfs.sys.ncell
    B, _ = df.fit_B(Vm, T3, ncl, dfs.nau)
    Bref = df_ref.fitted(Vm, T3, ncl, dfs.nau)
    # the inverse Cholesky factor of the metric amplifies the rounding of the two
    # summation orders (metric entries up to ~1e2, smallest pivots ~1e-6)
    assert np.abs(B - Bref).max() < 1e-9
    (p0, p1), (q0, q1) = df.band_ranges(r.occ_k)
    L = df.L_vectors(B, r.C_k, ncl, dfs.nfuc_ao, dfs.nau, (p0, p1), (q0, q1))
    Lref = df_ref.L_vectors(Bref, r.C_k, ncl, dfs.nfuc_ao, dfs.nau, p0, p1, q0, q1)
    assert np.abs(L - Lref).max() < 1e-9


def test_fit_reproduces_four_index_integrals(dimer_df):
    """sum_Q B B approximates (mu0 nu|la si) (the fitting error of this minimal
    auxiliary set), checked on the diagonal (mu0 nu|mu0 nu) = Q(mu,nu)^2."""
    from william_ci_b200 import df
    dfs, Vm, T3, r = dimer_df
    B, _ = df.fit_B(Vm, T3, dfs.sys.ncell, dfs.nau)
    o = po.Oracle(dimer_chain(4))
    Q = o.schwarz()
    nf, nb = B.shape[0], B.shape[1]
    fit = np.einsum("abq,abq->ab", B, B)
    exact = Q[:nf, :nb] ** 2
    big = exact > 1e-3
    assert np.all(fit[big] <= exact[big] * (1 + 1e-8))      # the fit never exceeds the exact value
    assert np.max(np.abs(fit[big] - exact[big]) / exact[big]) < 0.05


def test_mp2_energy_restatement_is_consistent(dimer_df):
    from william_ci_b200 import df
    dfs, Vm, T3, r = dimer_df
    ncl = dfs.sys.ncell
    Bref = df_ref.fitted(Vm, T3, ncl, dfs.nau)
    (p0, p1), (q0, q1) = df.band_ranges(r.occ_k)
    L = df_ref.L_vectors(Bref, r.C_k, ncl, dfs.nfuc_ao, dfs.nau, p0, p1, q0, q1)
    G = mp2_ref.ovov(L, ncl)
    e = mp2_ref.kmp2(G, ncl, r.eps_k[:, p0:p1], r.occ_k[:, p0:p1], r.eps_k[:, q0:q1], r.occ_k[:, q0:q1])
    assert e["nzero"] == 0
    assert -0.1 < e["emp2"] < 0.0                        # a small negative correlation energy per supercell


def tinv_density(nf, ncl, seed=3):
    """A symmetric, translation-invariant real-space density (block (r, c) = D(c - r))."""
    N = int(np.prod(ncl))
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((N, nf, nf)) * 0.1
    for d in range(N):
        md = df_ref.csub(ncl, 0, d)
        if md >= d:
            D[d] = 0.5 * (D[d] + D[md].T)
            D[md] = D[d].T
    P = np.zeros((nf * N, nf * N))
    for r in range(N):
        for c in range(N):
            P[r * nf:(r + 1) * nf, c * nf:(c + 1) * nf] = D[df_ref.csub(ncl, c, r)]
    return P


def test_k_space_B_and_df_jk_restatement(dimer_df):
    """The product's k-space Bh (fit_B, bh=True) against the restatement of
    df_init :660-678; the restated df_JK against the oracle's exact J/K (the
    fitting error of this auxiliary basis, not a parity bar)."""
    from william_ci_b200 import df
    from test_scf import dimer_chain
    dfs, Vm, T3, r = dimer_df
    ncl = dfs.sys.ncell
    B, _, Bh = df.fit_B(Vm, T3, ncl, dfs.nau, bh=True)
    Bref, Bhref = df_ref.fitted(Vm, T3, ncl, dfs.nau, bh=True)
    assert Bh.shape == Bhref.shape
    assert np.abs(Bh - Bhref).max() < 1e-9
    nf = dfs.nfuc_ao
    P = tinv_density(nf, ncl)
    J, K = df_ref.df_jk(Bref, Bhref, P, ncl, nf, dfs.nau)
    ao = dimer_chain(4)
    Je, Ke, _ = po.Oracle(ao).direct_jk(P)
    assert np.abs(J[nf:]).max() == 0.0 and np.abs(K[nf:]).max() == 0.0
    assert np.abs(J[:nf] - Je[:nf]).max() < 2e-2 * np.abs(Je[:nf]).max()
    assert np.abs(K[:nf] - Ke[:nf]).max() < 2e-2 * np.abs(Ke[:nf]).max()


@pytest.mark.parametrize("ncl", [(4, 1, 1), (5, 1, 1), (2, 3, 1), (2, 2, 2)])
def test_half_k_set_matches_the_restatement(ncl):
    """df_khalf (:103-114): the product's table against the restatement; every
    k is in the set or its -k is, never both unless k = -k."""
    from william_ci_b200 import df
    khi = df.khalf(ncl)
    assert np.array_equal(khi, df_ref.khalf(ncl))
    N = int(np.prod(ncl))
    for k in range(N):
        mk = df_ref.csub(ncl, 0, k)
        assert (khi[k] >= 0) or (khi[mk] >= 0)
        if mk != k:
            assert not (khi[k] >= 0 and khi[mk] >= 0)
