"""CPU restatement of density fitting for k-MP2 (df_init, df_L_kap, df_kMO).

TEST INFRASTRUCTURE ONLY: the checker of william_ci_b200/df.py (device
integrals + host linear algebra).  The product never imports it.  The loops
follow the reference's, with the integrals from the C oracle (shell_block,
the restated quartet kernel) on the same orbital + auxiliary + dummy system:

* metric Vm(P0, Q R) = (P0 1|Q R 1) (df_toroidal.f90:546-565);
* per k: V(k) = sum_R Vm(:, R) phase(k, R), hermitised, chol_f (pivoted
  Cholesky zpstrf to tol, ztrtri, f(piv(i), j) = conj(L^-1(j, i))), with
  f(-k) = conj f(k) (:575-594, 1174-1216);
* T3(mu0, nu, P) = (mu0 nu|P 1) (:597-626);
* df_B = T3 f in k-space, back to real space (:628-687);
* L(p, q, Q, k1, k2) per momentum transfer (df_L_kap :1053-1104).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg.lapack as lapack


def coords(ncl):
    nx, ny, nz = ncl
    return [(k % nx, (k // nx) % ny, k // (nx * ny)) for k in range(nx * ny * nz)]


def phase(ncl):
    c = coords(ncl)
    N = len(c)
    ph = np.zeros((N, N), dtype=np.complex128)
    for k in range(N):
        for r in range(N):
            th = 2 * np.pi * sum(c[k][d] * c[r][d] / max(ncl[d], 1) for d in range(3))
            ph[k, r] = np.exp(1j * th)
    return ph


def csub(ncl, r1, r2):
    c = coords(ncl)
    d = [(c[r1][x] - c[r2][x]) % ncl[x] for x in range(3)]
    return d[0] + ncl[0] * (d[1] + ncl[1] * d[2])


def chol_f(V, tol):
    n = V.shape[0]
    c, piv, m, info = lapack.zpstrf(np.asfortranarray(V.copy()), tol=tol, lower=1)
    assert info >= 0
    L = np.zeros((m, m), dtype=np.complex128)
    for j in range(m):
        for i in range(j, m):
            L[i, j] = c[i, j]
    Li, info = lapack.ztrtri(L, lower=1)
    assert info == 0
    f = np.zeros((n, n), dtype=np.complex128)
    for j in range(m):
        for i in range(m):
            f[piv[i] - 1, j] = np.conj(Li[j, i])
    return f


def integrals(orc, dfs, shells, nshuc):
    """Vm (nau, naux) and T3 (nfuc_ao, nbas_ao, naux) from oracle shell blocks (mode 0)."""
    first = [f for f, _ in shells]
    n = [c for _, c in shells]
    kind = [int(dfs.kind[f]) for f in first]
    atom = [int(dfs.sys.atom_of[f]) for f in first]
    dshell = {}
    for s, f in enumerate(first):
        if kind[s] == 2:
            dshell[atom[s]] = s
    N = int(np.prod(dfs.sys.ncell))
    nau, nf = dfs.nau, dfs.nfuc_ao
    Vm = np.zeros((nau, nau * N))
    T3 = np.zeros((nf, nf * N, nau * N))
    aux = [s for s in range(len(shells)) if kind[s] == 1]
    ao = [s for s in range(len(shells)) if kind[s] == 0]
    for p in aux:
        if p >= nshuc:
            continue
        for q in aux:
            b = orc.shell_block(p, dshell[atom[p]], q, dshell[atom[q]], mode=0)
            for x in range(n[p]):
                for y in range(n[q]):
                    Vm[dfs.aux_index[first[p] + x], dfs.aux_index[first[q] + y]] = b[x, 0, y, 0]
    for a in ao:
        if a >= nshuc:
            continue
        for bb in ao:
            for p in aux:
                blk = orc.shell_block(a, bb, p, dshell[atom[p]], mode=0)
                for x in range(n[a]):
                    for y in range(n[bb]):
                        for z in range(n[p]):
                            T3[dfs.ao_index[first[a] + x], dfs.ao_index[first[bb] + y],
                               dfs.aux_index[first[p] + z]] = blk[x, y, z, 0]
    return Vm, T3


def fitted(Vm, T3, ncl, nau, tol=1e-10):
    N = int(np.prod(ncl))
    ph = phase(ncl)
    f = np.zeros((nau, nau, N), dtype=np.complex128)
    for k in range(N):
        Mk = np.zeros((nau, nau), dtype=np.complex128)
        for r in range(N):
            Mk += Vm[:, r * nau:(r + 1) * nau] * ph[k, r]
        Mk = 0.5 * (Mk + Mk.conj().T)
        if csub(ncl, 0, k) < k:
            f[:, :, k] = np.conj(f[:, :, csub(ncl, 0, k)])
            continue
        f[:, :, k] = chol_f(Mk, tol)
    nf, nb = T3.shape[0], T3.shape[1]
    m1 = nf * nb * nau
    T = np.zeros((m1, N))
    for r in range(N):                       # Fortran (nfuc, nBas, nau) block of cell r
        T[:, r] = T3[:, :, r * nau:(r + 1) * nau].ravel(order="F")
    Cph = ph.T.real
    Sph = ph.T.imag
    Ar = T @ Cph
    Ai = T @ Sph
    for k in range(N):
        Zk = (Ar[:, k] + 1j * Ai[:, k]).reshape(nf * nb, nau, order="F")
        Wk = Zk @ f[:, :, k]
        Ar[:, k] = Wk.real.ravel(order="F")
        Ai[:, k] = Wk.imag.ravel(order="F")
    Bf = (Ar @ Cph.T + Ai @ Sph.T) / N        # (m1, R')
    B = np.zeros((nf, nb, nau * N))
    for r in range(N):
        B[:, :, r * nau:(r + 1) * nau] = Bf[:, r].reshape(nf, nb, nau, order="F")
    return B


def L_vectors(B, C_k, ncl, nf, nau, p_lo, p_hi, q_lo, q_hi):
    """L(p, q, Q, k1, k2), 0-based half-open band ranges."""
    N = int(np.prod(ncl))
    ph = phase(ncl)
    no, nv = p_hi - p_lo, q_hi - q_lo
    L = np.zeros((no, nv, nau, N, N), dtype=np.complex128)
    nb = B.shape[1]
    for kap in range(N):
        Bk = np.zeros((nf, nb, nau), dtype=np.complex128)
        for q in range(nau):
            for rq in range(N):
                Bk[:, :, q] += B[:, :, rq * nau + q] * np.conj(ph[kap, rq])
        F = np.zeros((nf, nf, nau, N), dtype=np.complex128)
        for k in range(N):
            for q in range(nau):
                for r in range(N):
                    F[:, :, q, k] += Bk[:, r * nf:(r + 1) * nf, q] * ph[k, r]
        for k2 in range(N):
            k1 = csub(ncl, k2, kap)
            C2 = C_k[k2][:, q_lo:q_hi]
            tmp = np.zeros((nf, nv, nau), dtype=np.complex128)
            for q in range(nau):
                tmp[:, :, q] = F[:, :, q, k2] @ C2
            C1 = C_k[k1][:, p_lo:p_hi]
            L[:, :, :, k1, k2] = np.einsum("ap,avq->pvq", C1.conj(), tmp)
    return L
