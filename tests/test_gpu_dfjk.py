"""Density-fitted J/K on the device (tce_dfjk) against the restatement of
df_JK (oracle/df_ref.py), both fed the same fitted coefficients (the C
oracle's 3- and 2-index integrals, fitted by the product's fit_B): J and K
within 1e-10 per element."""
import numpy as np
import pytest

import df_ref
import pyoracle as po

pytestmark = pytest.mark.gpu


def test_dfjk_vs_restatement():
    from william_ci_b200 import df
    from william_ci_b200 import system as S
    from test_df import tinv_density
    from test_scf import dimer_chain
    ao = dimer_chain(4)
    cell = S.Cell("Tori1D", (4, 1, 1), 4.0, (16.0, 0.0, 0.0), [("H", (0.0, 0.0, 0.0)), ("H", (1.4, 0.0, 0.0))])
    aux = S.build_system(cell, df.even_tempered_aux(ao.charges))
    po.normalize(aux)
    dfs = df.df_system(ao, aux)
    orc = po.Oracle(dfs.sys)
    sh, nshuc, _ = orc.shells()
    Vm, T3 = df_ref.integrals(orc, dfs, sh, nshuc)
    ncl = dfs.sys.ncell
    B, _, Bh = df.fit_B(Vm, T3, ncl, dfs.nau, bh=True)
    nf = dfs.nfuc_ao
    jk = df.DFJK(B, Bh, ncl, nf, dfs.nau)
    for seed in (3, 4):                       # two calls on one handle
        P = tinv_density(nf, ncl, seed)
        J, K = jk(P)
        Jr, Kr = df_ref.df_jk(B, Bh, P, ncl, nf, dfs.nau)
        assert np.abs(J - Jr).max() <= 1e-10, np.abs(J - Jr).max()
        assert np.abs(K - Kr).max() <= 1e-10, np.abs(K - Kr).max()
        assert np.abs(K[:nf]).max() > 1e-3
    jk.close()
