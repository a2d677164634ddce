"""CPU restatement of transform_ERI_AO_to_kMO (AO_to_MO_SAO.f90:34-393).

TEST INFRASTRUCTURE ONLY: the checker of tce_ao_to_kmo; the product never
imports it.  Same three steps as the reference, k4 by k4, with numpy
contractions (small systems only):
  1) X1(a, j2, j3, d)     = sum_R4 ERI(a, j2, j3, d R4) e^{+i k4 R4}
  2) X2(a, j2, c, d, k3)  = sum_R3 X1(a, j2, c R3, d) e^{-i k3 R3}
  3) per (k1, k2), k3 = k4 - k1 + k2:
     S(a, b, c, d)       = 1/N sum_R2 X2(a, b R2, c, d, k3) e^{+i k2 R2}
     ERI_out(p, q, r, s, k1, k2, k3) = sum C1*(a,p) C2(b,q) C3*(c,r) C4(d,s) S
with C_k(a, p) = coeff_SAO(k nfuc + a, k nfuc + p) and the phase
e^{2 pi i k.R / n} of the reference (:~60-70).  Band ranges 1-based, inclusive.
"""
import numpy as np

from df_ref import coords, phase


def ao_to_kmo(eri, coeff, ncl, nf, p_lo, p_hi, q_lo, q_hi):
    N = int(np.prod(ncl))
    nbas = nf * N
    ph = phase(ncl)
    c = coords(ncl)
    E = np.asarray(eri, dtype=np.float64).reshape(nf, nbas, nbas, nbas, order="F")
    p0, p1, q0, q1 = p_lo - 1, p_hi, q_lo - 1, q_hi
    no, nv = p1 - p0, q1 - q0
    out = np.zeros((no, nv, no, nv, N, N, N), dtype=np.complex128, order="F")
    Ck = [coeff[k * nf:(k + 1) * nf, k * nf:(k + 1) * nf] for k in range(N)]

    def cell(x, y, z):
        return (x % ncl[0]) + ncl[0] * ((y % ncl[1]) + ncl[1] * (z % ncl[2]))

    for k4 in range(N):
        Er = E.reshape(nf, nbas, nbas, nf, N, order="F")                  # d R4: d fastest
        X1 = np.einsum("abcdr,r->abcd", Er, ph[k4])
        X1r = X1.reshape(nf, nbas, nf, N, nf, order="F")                  # c R3
        X2 = np.einsum("abcrd,kr->abcdk", X1r, ph.conj())
        for k1 in range(N):
            for k2 in range(N):
                k3 = cell(c[k4][0] - c[k1][0] + c[k2][0], c[k4][1] - c[k1][1] + c[k2][1],
                          c[k4][2] - c[k1][2] + c[k2][2])
                X2r = X2[:, :, :, :, k3].reshape(nf, nf, N, nf, nf, order="F")   # b R2
                S = np.einsum("abrcd,r->abcd", X2r, ph[k2]) / N
                C1, C2, C3, C4 = Ck[k1][:, p0:p1], Ck[k2][:, q0:q1], Ck[k3][:, p0:p1], Ck[k4][:, q0:q1]
                out[:, :, :, :, k1, k2, k3] = np.einsum("ap,bq,cr,ds,abcd->pqrs", C1.conj(), C2, C3.conj(), C4, S)
    return out
