"""Density-fitted k-MP2 (DF-MP2): host mirror of df_init / df_kMO / kMP2_calc.

Reference: df_toroidal.f90:352-701 (df_init), 981-1104 (df_kMO, df_L_kap),
1174-1216 (chol_f); MP2_SAO.f90:6-151 (kMP2_calc).

* The auxiliary functions are toroidal Cartesian Gaussians normalised like
  the AOs.  The 3- and 2-index integrals are ordinary shell blocks of the
  device engine with a constant dummy (an s function of exponent 0 and
  coefficient 1 at the atom) next to every auxiliary function:
  (mu nu|P) = (mu nu|P 1), (P|Q) = (P 1|Q 1) (df_toroidal.f90:25-26, 837).
  The engine is created with tce_create_blocks (no J/K set-up).
* V(k) = sum_R (P0|Q R) e^{ikR} is factorised per k by pivoted Cholesky
  (tolerance 1e-10, as chol_f: f(k) = (L^-1)^H on the pivots); B = (mu0 nu|P) f
  is formed in k-space and brought back to real space; L^Q_pq(k1,k2) from the
  SAO orbital blocks (df_L_kap).  This linear algebra stays on the host
  (numpy / LAPACK), as the SCF's does.
* (ov|ov) = 1/N sum_Q L L and the MP2 energy run on the device
  (tce_dfmp2_energy): FP64, or split-BF16 on the tensor cores with FP32
  accumulation.

Not restated: the df_schwarz skip of (mu0 nu|P) shell triples below 1e-13
(every triple is computed), the generated even-tempered / Cholesky fitting
sets (the auxiliary basis is given), the symmetry variants.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Tuple

import numpy as np
import scipy.linalg.lapack as lapack

from .engine import Engine, TCEError, dfmp2_energy, lib, tce_system
from .system import AOSystem, Basis, BasisBlock

METRIC_TOL = 1e-10           # metric_tol_aux (df_toroidal.f90:68)


def even_tempered_aux(charges, n_s=4, n_p=2, n_d=1, start=0.1, ratio=2.5) -> Basis:
    """Uncontracted even-tempered auxiliary shells per element: exponents
    start * ratio^k, k = 0..n_l-1, for l = s, p, d."""
    out: Basis = {}
    for z in sorted(set(int(c) for c in charges)):
        blocks = []
        for l, n in ((0, n_s), (1, n_p), (2, n_d)):
            if n > 0:
                ex = start * ratio ** np.arange(n, dtype=np.float64)
                blocks.append(BasisBlock(l, ex[::-1].copy(), np.eye(n)[::-1].copy()))
        out[z] = blocks
    return out


@dataclasses.dataclass
class DFSystem:
    """The engine system of density fitting: per cell the orbital functions,
    the auxiliary functions and one constant dummy per atom."""
    sys: AOSystem
    nfuc_ao: int
    nau: int
    kind: np.ndarray          # per function: 0 orbital, 1 auxiliary, 2 dummy
    ao_index: np.ndarray      # per function: index in the orbital numbering (-1 otherwise)
    aux_index: np.ndarray     # per function: index in the auxiliary numbering (-1 otherwise)
    dummy_of_atom: np.ndarray  # per supercell atom: function index of its dummy


def df_system(ao: AOSystem, aux: AOSystem) -> DFSystem:
    """Interleave the (normalised) orbital and auxiliary systems cell by cell
    and add the dummies."""
    assert ao.ncell == aux.ncell and ao.ndp == aux.ndp
    Nc = int(np.prod(ao.ncell))
    nat_cell = len(ao.charges) // Nc
    ctr, lxyz, poff, exps, coefs, labels, atom_of = [], [], [0], [], [], [], []
    kind, aoi, auxi = [], [], []
    dum = np.zeros(len(ao.charges), dtype=np.int64)

    def add(src: AOSystem, f: int, k: int):
        ctr.append(src.ctr[f])
        lxyz.append(src.lxyz[f])
        p0, p1 = src.prim_off[f], src.prim_off[f + 1]
        exps.extend(src.exps[p0:p1].tolist())
        coefs.extend(src.coefs[p0:p1].tolist())
        poff.append(len(exps))
        labels.append(src.labels[f])
        atom_of.append(int(src.atom_of[f]))
        kind.append(k)
        aoi.append(f if k == 0 else -1)
        auxi.append(f if k == 1 else -1)

    for c in range(Nc):
        for f in range(c * ao.nfuc, (c + 1) * ao.nfuc):
            add(ao, f, 0)
        for f in range(c * aux.nfuc, (c + 1) * aux.nfuc):
            add(aux, f, 1)
        for a in range(c * nat_cell, (c + 1) * nat_cell):
            dum[a] = len(ctr)
            ctr.append(ao.geometry[a])
            lxyz.append(np.zeros(3, dtype=np.int32))
            exps.append(0.0)
            coefs.append(1.0)
            poff.append(len(exps))
            labels.append("s")
            atom_of.append(a)
            kind.append(2)
            aoi.append(-1)
            auxi.append(-1)
    nf = len(ctr) // Nc
    s = AOSystem(ndp=ao.ndp, ncell=ao.ncell, nfuc=nf, L=ao.L, ctr=np.array(ctr, dtype=np.float64),
                 lxyz=np.array(lxyz, dtype=np.int32), prim_off=np.array(poff, dtype=np.int32),
                 exps=np.array(exps, dtype=np.float64), coefs=np.array(coefs, dtype=np.float64), labels=labels,
                 atom_of=np.array(atom_of, dtype=np.int32), charges=ao.charges.copy(),
                 geometry=ao.geometry.copy())
    return DFSystem(s, ao.nfuc, aux.nfuc, np.array(kind), np.array(aoi), np.array(auxi), dum)


def _coords(ncl):
    nx, ny, nz = ncl
    return np.array([[k % nx, (k // nx) % ny, k // (nx * ny)] for k in range(nx * ny * nz)])


def _phase(ncl):
    c = _coords(ncl)
    n = np.array(ncl, dtype=np.float64)
    return np.exp(2j * np.pi * ((c[:, None, :] * c[None, :, :]) / n).sum(axis=2))   # (k, R)


def _csub(ncl, c1, c2):
    c = _coords(ncl)
    d = (c[c1] - c[c2]) % np.array(ncl)
    return int(d[0] + ncl[0] * (d[1] + ncl[1] * d[2]))


class DensityFitting:
    """Integrals and fitted vectors of one system (df_init)."""

    def __init__(self, dfs: DFSystem, **engine_kw):
        self.dfs = dfs
        self.eng = Engine(dfs.sys, blocks_only=True, **engine_kw)
        sh = self.eng.shells()
        self.sh_first = np.array([f for f, _ in sh])
        self.sh_n = np.array([n for _, n in sh])
        self.sh_kind = dfs.kind[self.sh_first]
        self.ncl = tuple(dfs.sys.ncell)
        self.N = int(np.prod(self.ncl))
        nsh = len(sh)
        self.nshuc = nsh // self.N
        # the dummy shell of each shell's atom
        f2s = np.zeros(dfs.sys.nbas, dtype=np.int64)
        for s_, (f, n) in enumerate(sh):
            f2s[f:f + n] = s_
        self.dummy_shell = f2s[dfs.dummy_of_atom[dfs.sys.atom_of[self.sh_first]]]

    def _blocks(self, items):
        K, _, offs = self.eng.rule_blocks(-1, np.array(items, dtype=np.int32), mode=0)
        return K, offs

    def metric(self) -> np.ndarray:
        """Vm(P0, Q R): (nau, naux)."""
        dfs, N = self.dfs, self.N
        aux_sh = np.nonzero(self.sh_kind == 1)[0]
        uc = [s for s in aux_sh if s < self.nshuc]
        items = [(p, self.dummy_shell[p], q, self.dummy_shell[q]) for p in uc for q in aux_sh]
        K, offs = self._blocks(items)
        Vm = np.zeros((dfs.nau, dfs.nau * N))
        for it, (p, _, q, _) in enumerate(items):
            nP, nQ = self.sh_n[p], self.sh_n[q]
            blk = K[offs[it]:offs[it + 1]].reshape(nP, nQ, order="F")
            ip = dfs.aux_index[self.sh_first[p]:self.sh_first[p] + nP]
            iq = dfs.aux_index[self.sh_first[q]:self.sh_first[q] + nQ]
            Vm[np.ix_(ip, iq)] = blk
        return Vm

    def three_index(self) -> np.ndarray:
        """T3(mu0, nu, P): (nfuc_ao, nbas_ao, naux)."""
        dfs, N = self.dfs, self.N
        ao_sh = np.nonzero(self.sh_kind == 0)[0]
        aux_sh = np.nonzero(self.sh_kind == 1)[0]
        uc = [s for s in ao_sh if s < self.nshuc]
        items = [(a, b, p, self.dummy_shell[p]) for a in uc for b in ao_sh for p in aux_sh]
        K, offs = self._blocks(items)
        T3 = np.zeros((dfs.nfuc_ao, dfs.nfuc_ao * N, dfs.nau * N))
        for it, (a, b, p, _) in enumerate(items):
            nA, nB, nP = self.sh_n[a], self.sh_n[b], self.sh_n[p]
            blk = K[offs[it]:offs[it + 1]].reshape(nA, nB, nP, order="F")
            ia = dfs.ao_index[self.sh_first[a]:self.sh_first[a] + nA]
            ib = dfs.ao_index[self.sh_first[b]:self.sh_first[b] + nB]
            ip = dfs.aux_index[self.sh_first[p]:self.sh_first[p] + nP]
            T3[np.ix_(ia, ib, ip)] = blk
        return T3

    def fitted(self, Vm=None, T3=None, mtol: float = METRIC_TOL):
        """df_B(mu0, nu, Q R) from the device integrals (fit_B)."""
        Vm = self.metric() if Vm is None else Vm
        T3 = self.three_index() if T3 is None else T3
        B, self.ndrop = fit_B(Vm, T3, self.ncl, self.dfs.nau, mtol)
        return B

    def L(self, B: np.ndarray, C_k: np.ndarray, p_rng: Tuple[int, int], q_rng: Tuple[int, int]) -> np.ndarray:
        return L_vectors(B, C_k, self.ncl, self.dfs.nfuc_ao, self.dfs.nau, p_rng, q_rng)


def khalf(ncl) -> np.ndarray:
    """df_khalf (df_toroidal.f90:103-114): position of k in the half set
    {k : -k >= k}, -1 for the others."""
    N = int(np.prod(ncl))
    khi = -np.ones(N, dtype=np.int64)
    n = 0
    for k in range(N):
        if _csub(ncl, 0, k) >= k:
            khi[k] = n
            n += 1
    return khi


def fit_B(Vm: np.ndarray, T3: np.ndarray, ncl, nau: int, mtol: float = METRIC_TOL, bh: bool = False):
    """df_B(mu0, nu, Q R) = sum (mu0 nu|P) [f](P, Q): f per k from the pivoted
    Cholesky of V(k) (chol_f, f(-k) = conj f(k)), the product in k-space,
    back to real space.  Returns (B, largest number of dropped pivots), and with
    bh=True also the k-space Bh(mu, Q, nu0; k1, kh) = sum_R1 W(k)(mu, nu0 R1, Q)
    e^{i k1 R1} of df_init (:660-678), (nf, nau, nf, N, nkh), k over the half set."""
    N = int(np.prod(ncl))
    ph = _phase(ncl)
    Vr = Vm.reshape(nau, N, nau)                               # (P, R, Q)
    f = np.zeros((N, nau, nau), dtype=np.complex128)
    ndrop = 0
    for k in range(N):
        mk = _csub(ncl, 0, k)
        if mk < k:
            f[k] = f[mk].conj()
            continue
        Mk = np.einsum("r,prq->pq", ph[k], Vr)
        Mk = 0.5 * (Mk + Mk.conj().T)
        f[k], nd = chol_factor(Mk, mtol)
        ndrop = max(ndrop, nd)
    nfu, nb = T3.shape[0], T3.shape[1]
    T = T3.reshape(nfu * nb, N, nau)                           # aux index (R, P)
    Z = np.einsum("xrp,kr->kxp", T, ph)                        # sum_R T3(R) e^{ikR}
    W = np.einsum("kxp,kpq->kxq", Z, f)
    B = np.einsum("kxq,kr->xrq", W, ph.conj()).real / N        # 1/N Re sum_k W(k) e^{-ikR}
    B = B.reshape(nfu, nb, N * nau)
    if not bh:
        return B, ndrop
    khi = khalf(ncl)
    Bh = np.zeros((nfu, nau, nfu, N, int((khi >= 0).sum())), dtype=np.complex128)
    for k in np.nonzero(khi >= 0)[0]:
        Wr = W[k].reshape(nfu, N, nfu, nau)                     # (mu, R1, nu0, Q): nu = R1 nf + nu0
        Bh[:, :, :, :, khi[k]] = np.einsum("arbq,kr->aqbk", Wr, ph)
    return B, ndrop, Bh


class DFJK:
    """Density-fitted J and K on the device (tce_dfjk: df_JK, df_toroidal.f90
    :850-956), from df_B and the k-space Bh of fit_B(..., bh=True)."""

    def __init__(self, B: np.ndarray, Bh: np.ndarray, ncl, nf: int, nau: int):
        import ctypes as C
        from .engine import TCEError, lib
        self._lib = lib()
        self.nbas = B.shape[1]
        Bf = np.asfortranarray(B, dtype=np.float64).ravel(order="F").copy()
        Bhf = np.asfortranarray(Bh, dtype=np.complex128).ravel(order="F").copy().view(np.float64)
        n3 = np.array([int(x) for x in ncl], dtype=np.int32)
        self.h = C.c_void_p()
        dp = C.POINTER(C.c_double)
        code = self._lib.tce_dfjk_create(int(nf), int(self.nbas), int(nau), n3.ctypes.data_as(C.POINTER(C.c_int32)),
                                         Bf.ctypes.data_as(dp), Bhf.ctypes.data_as(dp), C.byref(self.h))
        if code != 0:
            raise TCEError(code, self._lib.tce_dfjk_last_error(None).decode())

    def __call__(self, P: np.ndarray):
        import ctypes as C
        from .engine import TCEError
        n = self.nbas
        Pf = np.asfortranarray(P, dtype=np.float64).ravel(order="F").copy()
        J = np.zeros(n * n)
        K = np.zeros(n * n)
        dp = C.POINTER(C.c_double)
        code = self._lib.tce_dfjk(self.h, Pf.ctypes.data_as(dp), J.ctypes.data_as(dp), K.ctypes.data_as(dp))
        if code != 0:
            raise TCEError(code, self._lib.tce_dfjk_last_error(self.h).decode())
        return J.reshape(n, n, order="F"), K.reshape(n, n, order="F")

    def close(self):
        if self.h:
            self._lib.tce_dfjk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def L_vectors(B: np.ndarray, C_k: np.ndarray, ncl, nf: int, nau: int, p_rng: Tuple[int, int],
              q_rng: Tuple[int, int]) -> np.ndarray:
    """L^Q_pq(k1, k2), (no, nv, nau, N, N) (df_L_kap for every kap)."""
    N = int(np.prod(ncl))
    ph = _phase(ncl)
    p0, p1 = p_rng
    q0, q1 = q_rng
    Br = B.reshape(nf, N, nf, N, nau)                          # (a, R_b, b0, R_Q, Q)
    out = np.zeros((p1 - p0, q1 - q0, nau, N, N), dtype=np.complex128)
    for kap in range(N):
        Bk = np.einsum("aRbsq,s->aRbq", Br, ph[kap].conj())    # sum_RQ B e^{-i kap RQ}
        F = np.einsum("aRbq,kR->abqk", Bk, ph)                 # sum_R ... e^{ikR}
        for k2 in range(N):
            k1 = _csub(ncl, k2, kap)
            tmp = np.einsum("abq,bv->avq", F[:, :, :, k2], C_k[k2][:, q0:q1])
            out[:, :, :, k1, k2] = np.einsum("ap,avq->pvq", C_k[k1][:, p0:p1].conj(), tmp)
    return out


def chol_factor(V: np.ndarray, tol: float):
    """chol_f (df_toroidal.f90:1174-1216): pivoted Cholesky V = P L L^H P^T to
    rank m (LAPACK zpstrf, tolerance tol), f(piv(i), j) = conj(L^-1(j, i))."""
    n = V.shape[0]
    c, piv, m, info = lapack.zpstrf(np.asfortranarray(V), tol=tol, lower=1)
    if info < 0:
        raise RuntimeError("zpstrf failed")
    Lm = np.tril(c[:m, :m])
    Li, info = lapack.ztrtri(Lm, lower=1)
    if info != 0:
        raise RuntimeError("ztrtri failed")
    f = np.zeros((n, n), dtype=np.complex128)
    pv = np.asarray(piv) - 1
    f[pv[:m], :m] = Li[:m, :m].T.conj()
    return f, n - m


def band_ranges(occ_k: np.ndarray):
    """o_hi = max_k nOcc(k), v_lo = min_k nOcc(k) + 1 (cc_dims), 0-based ranges."""
    nocc = (occ_k == 2).sum(axis=1)
    return (0, int(nocc.max())), (int(nocc.min()), occ_k.shape[1])


def dfmp2(dfit: DensityFitting, C_k, eps_k, occ_k, mode: int = 1, B=None) -> Dict[str, float]:
    """E_MP2 = 2 E2d - E2x with the device contraction (mode 1: split-BF16)."""
    B = dfit.fitted() if B is None else B
    (p0, p1), (q0, q1) = band_ranges(occ_k)
    L = dfit.L(B, C_k, (p0, p1), (q0, q1))
    return dfmp2_energy(dfit.ncl, L, eps_k[:, p0:p1], occ_k[:, p0:p1], eps_k[:, q0:q1], occ_k[:, q0:q1],
                        mode=mode)


class DeviceDF:
    """df_init, df_L_kap and kMP2_calc behind one libtce handle (tce_df_create,
    tce_dfmp2): the fit's integrals, the per-k factorisation of the metric,
    df_B and the L vectors all on the device; a Fortran caller gets E_MP2 from
    the same two calls."""

    def __init__(self, ao: AOSystem, aux: AOSystem):
        import ctypes as C
        self.ao, self.aux = ao, aux
        s1, self._k1 = tce_system(ao)
        s2, self._k2 = tce_system(aux)
        self._geo = np.asfortranarray(ao.geometry, dtype=np.float64).ravel(order="F").copy()
        self.h = C.c_void_p()
        code = lib().tce_df_create(C.byref(s1), C.byref(s2), len(ao.charges),
                                   self._geo.ctypes.data_as(C.POINTER(C.c_double)), C.byref(self.h))
        if code:
            raise TCEError(code, lib().tce_df_last_error(None).decode())
        self.ncl = tuple(ao.ncell)
        self.N = int(np.prod(self.ncl))
        self.nf, self.nau = ao.nfuc, aux.nfuc

    def _ck(self, code):
        if code:
            raise TCEError(code, lib().tce_df_last_error(self.h).decode())

    def integrals(self):
        """Vm (nau, naux) and T3 (nfuc, nbas, naux)."""
        import ctypes as C
        naux, nb = self.nau * self.N, self.nf * self.N
        Vm = np.zeros(self.nau * naux)
        T3 = np.zeros(self.nf * nb * naux)
        dp = C.POINTER(C.c_double)
        self._ck(lib().tce_df_integrals(self.h, Vm.ctypes.data_as(dp), T3.ctypes.data_as(dp)))
        return Vm.reshape(self.nau, naux, order="F"), T3.reshape(self.nf, nb, naux, order="F")

    def fitted(self, bh: bool = False):
        """df_B (nfuc, nbas, naux), the most dropped pivots, and with bh=True the
        k-space Bh (nfuc, nau, nfuc, N, nkh) of the density-fitted J/K."""
        import ctypes as C
        naux, nb = self.nau * self.N, self.nf * self.N
        B = np.zeros(self.nf * nb * naux)
        nkh = int((khalf(self.ncl) >= 0).sum())
        Bh = np.zeros(2 * self.nf * self.nau * self.nf * self.N * nkh) if bh else None
        nd = C.c_int32()
        dp = C.POINTER(C.c_double)
        self._ck(lib().tce_df_fitted(self.h, B.ctypes.data_as(dp), Bh.ctypes.data_as(dp) if bh else None,
                                     C.byref(nd)))
        B = B.reshape(self.nf, nb, naux, order="F")
        if not bh:
            return B, nd.value
        return B, nd.value, Bh.view(np.complex128).reshape(self.nf, self.nau, self.nf, self.N, nkh, order="F")

    def dfmp2(self, C_k: np.ndarray, eps_k: np.ndarray, occ_k: np.ndarray, mode: int = 0) -> Dict[str, float]:
        """E_MP2 from the SCF's k-block orbitals (N, nf, nf), energies and occupations (N, nf)."""
        import ctypes as C
        N, nf = self.N, self.nf
        n = N * nf
        coeff = np.zeros((n, n), dtype=np.complex128)
        for k in range(N):
            coeff[k * nf:(k + 1) * nf, k * nf:(k + 1) * nf] = C_k[k]
        cf = np.asfortranarray(coeff).ravel(order="F").copy().view(np.float64)
        eps = np.ascontiguousarray(eps_k, dtype=np.float64).ravel()
        occ = np.ascontiguousarray(occ_k, dtype=np.int32).ravel()
        e, e2d, e2x = C.c_double(), C.c_double(), C.c_double()
        dp = C.POINTER(C.c_double)
        self._ck(lib().tce_dfmp2(self.h, cf.ctypes.data_as(dp), eps.ctypes.data_as(dp),
                                 occ.ctypes.data_as(C.POINTER(C.c_int32)), int(mode), C.byref(e), C.byref(e2d),
                                 C.byref(e2x)))
        return {"emp2": e.value, "e2d": e2d.value, "e2x": e2x.value}

    def close(self):
        if getattr(self, "h", None):
            lib().tce_df_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
