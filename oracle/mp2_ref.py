"""CPU restatement of the DF-MP2 (ov|ov) contraction and the k-MP2 energy.

TEST INFRASTRUCTURE ONLY: the checker of libtce's tce_dfmp2_energy.  The
product never imports it.  Follows, loop for loop:

* the (ov|ov) loop of df_kMO (df_toroidal.f90:1018-1035):
    ERI_out(:,:,:,:,k1,k2,k3) = 1/N L(:,:,:,k1,k2) L(:,:,:,k3,k4)^T,
    k4 = cadd(csub(k1,k2),k3) (cell coordinates modulo the lattice);
* kMP2_calc (MP2_SAO.f90:6-151): occupied i (occupation 2) in ki, j in kj,
  virtual a (occupation 0) in ka, b in kb = ki - ka + kj; D = e_a + e_b -
  e_i - e_j; terms with |D| < 1e-8 left out and counted;
  E2d -= |g_d|^2 / D, E2x -= Re(g_d conj g_x) / D, E_MP2 = 2 E2d - E2x.
"""
from __future__ import annotations

import numpy as np


def coords(ncl):
    nx, ny, nz = ncl
    return np.array([[k % nx, (k // nx) % ny, k // (nx * ny)] for k in range(nx * ny * nz)])


def cadd_csub(crd, ncl, k1, k2, k3):
    """Cell index of k1 - k2 + k3."""
    c = (crd[k1] - crd[k2] + crd[k3]) % np.array(ncl)
    return int(c[0] + ncl[0] * (c[1] + ncl[1] * c[2]))


def ovov(L, ncl):
    """ERI_out(p, q, r, s, k1, k2, k3) from L(p, q, Q, k1, k2)."""
    no, nv, nau, N, _ = L.shape
    crd = coords(ncl)
    G = np.zeros((no, nv, no, nv, N, N, N), dtype=np.complex128)
    for k1 in range(N):
        for k2 in range(N):
            A = L[:, :, :, k1, k2].reshape(no * nv, nau, order="F")
            for k3 in range(N):
                k4 = cadd_csub(crd, ncl, k1, k2, k3)
                B = L[:, :, :, k3, k4].reshape(no * nv, nau, order="F")
                G[:, :, :, :, k1, k2, k3] = ((A @ B.T) / N).reshape(no, nv, no, nv, order="F")
    return G


def kmp2(G, ncl, eps_o, occ_o, eps_v, occ_v):
    no, nv, _, _, N, _, _ = G.shape
    crd = coords(ncl)
    e2d = e2x = 0.0
    nzero, gzero = 0, 0.0
    for ki in range(N):
        for kj in range(N):
            for ka in range(N):
                kb = cadd_csub(crd, ncl, ki, ka, kj)
                for i in range(no):
                    if occ_o[ki, i] != 2:
                        continue
                    for j in range(no):
                        if occ_o[kj, j] != 2:
                            continue
                        for a in range(nv):
                            if occ_v[ka, a] != 0:
                                continue
                            for b in range(nv):
                                if occ_v[kb, b] != 0:
                                    continue
                                D = eps_v[ka, a] + eps_v[kb, b] - eps_o[ki, i] - eps_o[kj, j]
                                gd = G[i, a, j, b, ki, ka, kj]
                                if abs(D) < 1e-8:
                                    nzero += 1
                                    gzero = max(gzero, abs(gd))
                                    continue
                                gx = G[i, b, j, a, ki, kb, kj]
                                e2d -= (gd * np.conj(gd)).real / D
                                e2x -= (gd * np.conj(gx)).real / D
    return {"e2d": e2d, "e2x": e2x, "emp2": 2 * e2d - e2x, "nzero": nzero, "gzero": gzero}
