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
* L(p, q, Q, k1, k2) per momentum transfer (df_L_kap :1053-1104);
* df_JK (:850-956) with the k-space Bh of :660-678.
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


def khalf(ncl):
    """df_khalf :103-114: position of k in the half set {k : -k >= k} (0-based), -1 otherwise."""
    N = int(np.prod(ncl))
    khi = -np.ones(N, dtype=np.int64)
    n = 0
    for k in range(N):
        if csub(ncl, 0, k) >= k:
            khi[k] = n
            n += 1
    return khi


def cadd(ncl, r1, r2):
    c = coords(ncl)
    d = [(c[r1][x] + c[r2][x]) % ncl[x] for x in range(3)]
    return d[0] + ncl[0] * (d[1] + ncl[1] * d[2])


def fitted(Vm, T3, ncl, nau, tol=1e-10, bh=False):
    """df_B (and with bh=True also the k-space Bh(mu, Q, nu0; k1, k) of :660-678,
    complex (nf, nau, nf, N, nkh))."""
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
    khi = khalf(ncl)
    Bh = np.zeros((nf, nau, nf, N, int((khi >= 0).sum())), dtype=np.complex128) if bh else None
    for k in range(N):
        Zk = (Ar[:, k] + 1j * Ai[:, k]).reshape(nf * nb, nau, order="F")
        Wk = Zk @ f[:, :, k]
        Ar[:, k] = Wk.real.ravel(order="F")
        Ai[:, k] = Wk.imag.ravel(order="F")
        if bh and khi[k] >= 0:
            Wt = np.zeros((nf, nau, nf, N), dtype=np.complex128)
            for r in range(N):
                for nu0 in range(nf):
                    for q in range(nau):
                        Wt[:, q, nu0, r] = Wk[r * nf * nf + nu0 * nf: r * nf * nf + (nu0 + 1) * nf, q]
            for k1 in range(N):
                Bh[:, :, :, k1, khi[k]] = np.einsum("aqbr,r->aqb", Wt, ph[k1])
    Bf = (Ar @ Cph.T + Ai @ Sph.T) / N        # (m1, R')
    B = np.zeros((nf, nb, nau * N))
    for r in range(N):
        B[:, :, r * nau:(r + 1) * nau] = Bf[:, r].reshape(nf, nb, nau, order="F")
    return (B, Bh) if bh else B


def df_jk(B, Bh, P, ncl, nf, nau):
    """df_JK :850-956: J from the real-space B (gamma over the cells), K from the
    k-space Bh and the eigenvectors of P(k) with |eigenvalue| > 1e-10.  Rows
    >= nf of J and K are zero, as the reference leaves them."""
    N = int(np.prod(ncl))
    nbas = nf * N
    naux = nau * N
    ph = phase(ncl)
    khi = khalf(ncl)
    Bm = B.reshape(nf * nbas, naux, order="F")
    Ps = np.zeros((nf * nbas, N))
    for r in range(N):
        for rs in range(N):
            c = cadd(ncl, rs, r)
            Ps[rs * nf * nf:(rs + 1) * nf * nf, r] = P[r * nf:(r + 1) * nf, c * nf:(c + 1) * nf].ravel(order="F")
    G = Bm.T @ Ps
    gam = np.zeros(naux)
    for r in range(N):
        for rq in range(N):
            c = cadd(ncl, rq, r)
            gam[c * nau:(c + 1) * nau] += G[rq * nau:(rq + 1) * nau, r]
    J = np.zeros((nbas, nbas))
    J[:nf, :] = (Bm @ gam).reshape(nf, nbas, order="F")
    ck, wk = [], []
    for ik in range(N):
        pk = sum(P[:nf, r * nf:(r + 1) * nf] * ph[ik, r] for r in range(N))
        pk = 0.5 * (pk + pk.conj().T)
        ew, ev = np.linalg.eigh(pk)
        keep = np.abs(ew) > 1e-10
        ck.append(ev[:, keep])
        wk.append(ew[keep])
    Kt = np.zeros((N, nf, nf), dtype=np.complex128)
    for kk in range(N):
        Kloc = np.zeros((nf, nf), dtype=np.complex128)
        for k1 in range(N):
            no = len(wk[k1])
            if no == 0:
                continue
            k2 = csub(ncl, kk, k1)
            if khi[k2] >= 0:
                L = Bh[:, :, :, k1, khi[k2]].reshape(nf * nau, nf, order="F") @ ck[k1]
            else:
                mk1 = csub(ncl, 0, k1)
                L = np.conj(Bh[:, :, :, mk1, khi[csub(ncl, 0, k2)]].reshape(nf * nau, nf, order="F") @ np.conj(ck[k1]))
            L = L.reshape(nf, nau * no, order="F")
            w = np.repeat(wk[k1], nau)                      # column (q, i) -> w_i
            Kloc += (L * w) @ L.conj().T
        Kt[kk] = Kloc * (-0.5 / N)
    K = np.zeros((nbas, nbas))
    for r in range(N):
        pk = sum(Kt[kk] * np.conj(ph[kk, r]) for kk in range(N))
        K[:nf, r * nf:(r + 1) * nf] = pk.real / N
    return J, K


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
