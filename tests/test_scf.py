"""The SCF consumer (RHF_SAO mirror) on CPU with oracle J/K providers."""
import numpy as np
import pytest

import pyoracle as po
from conftest import make_system
from william_ci_b200 import scf
from william_ci_b200 import system as S


def dimer_chain(ncell=6):
    cell = S.Cell("Tori1D", (ncell, 1, 1), 4.0, (4.0 * ncell, 0.0, 0.0), [("H", (0.0, 0.0, 0.0)), ("H", (1.4, 0.0, 0.0))])
    sysm = S.build_system(cell, {1: [S.STO3G_H]})
    po.normalize(sysm)
    return sysm


def rhf_inputs(sysm):
    o = po.Oracle(sysm)
    St, Tt, Vt = o.one_electron()
    return o, St, Tt, Vt, po.nuclear_repulsion(sysm), scf.n_occupied(sysm)


def test_sao_round_trip_and_fill():
    sysm = make_system("h_chain64", (8, 1, 1))
    o, St, Tt, Vt, en, nO = rhf_inputs(sysm)
    sao = scf.SAO(sysm.nfuc, sysm.ncell)
    for M in (St, Tt, Vt):
        assert np.max(np.abs(sao.to_ao(sao.to_sao(M)) - M)) < 1e-13
        assert np.max(np.abs(scf.fill_with_symmetry(M[:sysm.nfuc], sysm.nfuc, sysm.ncell) - M)) == 0.0
    # S_k Hermitian positive definite for every k
    for Sk in sao.to_sao(St):
        assert np.max(np.abs(Sk - Sk.conj().T)) < 1e-13
        assert np.linalg.eigvalsh(Sk).min() > 0


def test_occupy_cut_fractional():
    e = np.array([-1.0, -0.5, -0.5, 0.3])
    c = np.eye(4)
    P = scf.guess_occupy_cut(2, e, c)
    np.testing.assert_allclose(np.diag(P), [2.0, 1.0, 1.0, 0.0])


@pytest.mark.parametrize("which", ["h2_ring", "dimer_chain"])
def test_direct_and_stored_jk_give_the_same_rhf_energy(which):
    sysm = make_system("h2_ring") if which == "h2_ring" else dimer_chain()
    o, St, Tt, Vt, en, nO = rhf_inputs(sysm)
    r1 = scf.rhf_sao(St, Tt, Vt, en, nO, sysm.nfuc, sysm.ncell, lambda P: o.direct_jk(P)[:2])
    E, _ = o.eri_stored()
    r2 = scf.rhf_sao(St, Tt, Vt, en, nO, sysm.nfuc, sysm.ncell, lambda P: po.hartree_exchange(sysm.nfuc, P, E))
    assert r1.converged and r2.converged
    assert abs(r1.energy - r2.energy) < 1e-10
    assert r1.iterations == r2.iterations
