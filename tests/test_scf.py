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


def test_trexio_chunks_follow_the_reference_writer():
    """eri_chunks cuts an entry stream into the reference's buffered writes:
    full buffers at offsets 0, B, 2B, ...; the last partial buffer passed with
    count B, its tail left from the buffer before (trexio_conv.f90:326-357)."""
    from william_ci_b200 import trexio_out as TX
    n, B = 25, 10
    idx = np.arange(4 * n, dtype=np.int32).reshape(n, 4)
    val = np.arange(n, dtype=np.float64) + 0.5
    calls = TX.eri_chunks(idx, val, bufsize=B)
    assert [c[0] for c in calls] == [0, 10, 20] and all(c[1] == B for c in calls)
    np.testing.assert_array_equal(calls[1][3], val[10:20])
    last = calls[2][3]
    np.testing.assert_array_equal(last[:5], val[20:25])
    np.testing.assert_array_equal(last[5:], val[15:20])     # stale entries of the previous buffer
    assert len(TX.eri_chunks(idx[:20], val[:20], bufsize=B)) == 2


def test_trexio_reference_stream_on_the_oracle_integrals():
    """The stream restatement on the oracle's full integrals of the 2-cell ring:
    the loop's conditions and order."""
    from william_ci_b200 import trexio_out as TX
    sysm = make_system("h2_ring")
    o = po.Oracle(sysm, sao=False)
    E, _ = o.eri_stored()
    idx, val = TX.reference_stream(E)
    n = sysm.nbas
    expect = []
    for l in range(n):
        for k in range(n):
            for j in range(n):
                for i in range(n):
                    if (i == j and k < l) or i < j or E[i, k, j, l] == 0.0:
                        continue
                    expect.append((i + 1, j + 1, k + 1, l + 1, E[i, k, j, l]))
    assert [tuple(r) for r in idx] == [e[:4] for e in expect]
    np.testing.assert_array_equal(val, [e[4] for e in expect])
