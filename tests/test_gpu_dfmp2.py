"""DF-MP2 end to end (row a13): device 3- and 2-index integrals with the
constant dummies, host fitting, device (ov|ov) contraction and energy, against
the oracle pipeline (C oracle integrals, oracle/df_ref.py, oracle/mp2_ref.py)
on the same RHF orbitals.  Integrals 1e-10 absolute; E_MP2 1e-10 Eh with the
FP64 contraction; the split-BF16 tensor-core contraction's error is stated and
bounded at 1e-5 relative."""
import numpy as np
import pytest

import df_ref
import mp2_ref
import pyoracle as po
from test_scf import dimer_chain, rhf_inputs

pytestmark = pytest.mark.gpu


def _df_pair(ao, cell):
    from william_ci_b200 import df
    from william_ci_b200 import system as S
    aux = S.build_system(cell, df.even_tempered_aux(ao.charges))
    po.normalize(aux)
    return df.df_system(ao, aux)


def _dimer_cell(n):
    from william_ci_b200 import system as S
    return S.Cell("Tori1D", (n, 1, 1), 4.0, (4.0 * n, 0.0, 0.0), [("H", (0.0, 0.0, 0.0)), ("H", (1.4, 0.0, 0.0))])


@pytest.mark.parametrize("which", ["dimer", "h_chain"])
def test_df_integrals_vs_oracle(which):
    from conftest import make_system
    from william_ci_b200 import df
    from william_ci_b200 import system as S
    if which == "dimer":
        ao, cell = dimer_chain(4), _dimer_cell(4)
    else:
        ao = make_system("h_chain64", (4, 1, 1))
        c0, _ = S.workload("h_chain64")
        cell = S.scaled_down(c0, (4, 1, 1))
    dfs = _df_pair(ao, cell)
    dfit = df.DensityFitting(dfs)
    Vm, T3 = dfit.metric(), dfit.three_index()
    orc = po.Oracle(dfs.sys)
    sh, nshuc, _ = orc.shells()
    Vr, Tr = df_ref.integrals(orc, dfs, sh, nshuc)
    assert np.abs(Vm - Vr).max() < 1e-10
    assert np.abs(T3 - Tr).max() < 1e-10


def test_dfmp2_energy_vs_oracle_pipeline():
    from william_ci_b200 import df, scf
    ao = dimer_chain(4)
    dfs = _df_pair(ao, _dimer_cell(4))
    o, St, Tt, Vt, en, nO = rhf_inputs(ao)
    r = scf.rhf_sao(St, Tt, Vt, en, nO, ao.nfuc, ao.ncell, lambda P: o.direct_jk(P)[:2])
    assert r.converged
    # oracle pipeline
    orc = po.Oracle(dfs.sys)
    sh, nshuc, _ = orc.shells()
    Vr, Tr = df_ref.integrals(orc, dfs, sh, nshuc)
    ncl = dfs.sys.ncell
    Bref = df_ref.fitted(Vr, Tr, ncl, dfs.nau)
    (p0, p1), (q0, q1) = df.band_ranges(r.occ_k)
    Lref = df_ref.L_vectors(Bref, r.C_k, ncl, dfs.nfuc_ao, dfs.nau, p0, p1, q0, q1)
    ref = mp2_ref.kmp2(mp2_ref.ovov(Lref, ncl), ncl, r.eps_k[:, p0:p1], r.occ_k[:, p0:p1],
                       r.eps_k[:, q0:q1], r.occ_k[:, q0:q1])
    # product: device integrals, host fitting, device contraction
    dfit = df.DensityFitting(dfs)
    B = dfit.fitted()
    e64 = df.dfmp2(dfit, r.C_k, r.eps_k, r.occ_k, mode=0, B=B)
    e16 = df.dfmp2(dfit, r.C_k, r.eps_k, r.occ_k, mode=1, B=B)
    print("E_MP2 oracle %.12f  FP64 %.12f  split-BF16 %.12f (rel err %.2e)" % (
        ref["emp2"], e64["emp2"], e16["emp2"], abs(e16["emp2"] - ref["emp2"]) / abs(ref["emp2"])))
    assert abs(e64["emp2"] - ref["emp2"]) < 1e-10
    assert abs(e16["emp2"] - ref["emp2"]) < 1e-5 * abs(ref["emp2"])
