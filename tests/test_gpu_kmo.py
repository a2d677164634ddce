"""k-space MO integrals on the device (tce_ao_to_kmo) against the restatement
of transform_ERI_AO_to_kMO (oracle/kmo_ref.py) fed the device's own stored
SAO integrals and the RHF orbitals of a 4-cell dimer chain: every element
within 1e-10, on the (ov|ov) ranges of MP2 and the full range of CCSD."""
import numpy as np
import pytest

import kmo_ref

pytestmark = pytest.mark.gpu


def test_ao_to_kmo_vs_restatement():
    from william_ci_b200 import df, scf
    from william_ci_b200.engine import Engine
    from test_scf import dimer_chain, rhf_inputs
    ao = dimer_chain(4)
    o, St, Tt, Vt, en, nO = rhf_inputs(ao)
    r = scf.rhf_sao(St, Tt, Vt, en, nO, ao.nfuc, ao.ncell, lambda P: o.direct_jk(P)[:2])
    assert r.converged
    nf, ncl = ao.nfuc, tuple(ao.ncell)
    N = int(np.prod(ncl))
    with Engine(ao) as eng:
        eri = eng.ERI_integral_toroidal()
        coeff = np.zeros((ao.nbas, ao.nbas), dtype=np.complex128)
        for k in range(N):
            coeff[k * nf:(k + 1) * nf, k * nf:(k + 1) * nf] = r.C_k[k]
        (p0, p1), (q0, q1) = df.band_ranges(r.occ_k)
        for pr, qr in (((p0, p1), (q0, q1)), ((0, nf), (0, nf))):
            got = eng.ao_to_kmo(r.C_k, pr, qr)
            ref = kmo_ref.ao_to_kmo(eri, coeff, ncl, nf, pr[0] + 1, pr[1], qr[0] + 1, qr[1])
            assert got.shape == ref.shape
            assert np.abs(got - ref).max() <= 1e-10, np.abs(got - ref).max()
            assert np.abs(ref).max() > 1e-2
