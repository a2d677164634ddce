"""The restatement of transform_ERI_AO_to_kMO (oracle/kmo_ref.py, the
reference's three steps) against the transform's definition summed directly,
    (p k1, q k2 | r k3, s k4) = 1/N sum_{R2 R3 R4} e^{i k2 R2 - i k3 R3 + i k4 R4}
        sum_{abcd} C1*(a,p) C2(b,q) C3*(c,r) C4(d,s) (a0 b R2 | c R3 d R4),
on the oracle's stored integrals of a 4-cell dimer chain with random unitary
k blocks (CPU)."""
import numpy as np

import df_ref
import kmo_ref
import pyoracle as po
from test_scf import dimer_chain


def test_kmo_steps_equal_the_definition():
    ao = dimer_chain(4)
    nf, ncl = ao.nfuc, tuple(ao.ncell)
    N = int(np.prod(ncl))
    n = ao.nbas
    eri, _ = po.Oracle(ao).eri_stored()
    rng = np.random.default_rng(5)
    coeff = np.zeros((n, n), dtype=np.complex128)
    for k in range(N):
        q, _ = np.linalg.qr(rng.standard_normal((nf, nf)) + 1j * rng.standard_normal((nf, nf)))
        coeff[k * nf:(k + 1) * nf, k * nf:(k + 1) * nf] = q
    got = kmo_ref.ao_to_kmo(eri, coeff, ncl, nf, 1, nf, 1, nf)
    ph = df_ref.phase(ncl)
    c = df_ref.coords(ncl)
    E = np.asarray(eri).reshape(nf, nf, N, nf, N, nf, N, order="F")       # (a, b, R2, c, R3, d, R4)
    Y = np.einsum("abxcydz,kx,ly,mz->abcdklm", E, ph, ph.conj(), ph) / N
    Ck = [coeff[k * nf:(k + 1) * nf, k * nf:(k + 1) * nf] for k in range(N)]
    worst = 0.0
    for k1 in range(N):
        for k2 in range(N):
            for k3 in range(N):
                k4 = sum(((c[k1][d] - c[k2][d] + c[k3][d]) % ncl[d]) * int(np.prod(ncl[:d])) for d in range(3))
                ref = np.einsum("ap,bq,cr,ds,abcd->pqrs", Ck[k1].conj(), Ck[k2], Ck[k3].conj(), Ck[k4],
                                Y[:, :, :, :, k2, k3, k4])
                worst = max(worst, np.abs(got[:, :, :, :, k1, k2, k3] - ref).max())
    assert worst < 1e-12, worst
    assert np.abs(got).max() > 1e-2
