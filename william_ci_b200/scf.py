"""Restricted Hartree-Fock in the symmetry-adapted (k-blocked) basis: the
consumer of the J/K path.

Host-side mirror of RHF_SAO (src/Energies/SAO/RHF_SAO.f90:1-553).  The SCF
loop stays on the host (small per-k linear algebra, as in the reference);
every iteration calls a J/K provider, by default the device engine
(`Engine.direct_JK`, i.e. tce_direct_jk).  Inputs are the reference's:
S, T, V (nbas x nbas, rows of every cell filled by translation), the nuclear
repulsion energy, the number of doubly occupied orbitals, the cell grid.

Pieces restated (file:line of the reference):
  get_X_from_overlap / canonical_X_real      Energies_tools.f90:84-139, 445-469
  guess_AO_RHF_SAO                           SAO/guess_RHF_SAO.f90:1-115
  guess_occupy_cut                           SAO/guess_Huckel_SAO.f90:141-192
  transform_AO_to_SAO / transform_SAO_to_AO  Tools/SAO_Transfer.f90:1-233
  get_X_from_overlap_complex_blocks          Energies_tools.f90:328-391
  shift_dropped_real / _complex              Energies_tools.f90:499-528
  DIIS_extrapolation                         DIIS_extrapolation.f90:1-51
  energies, error X^T(FPS-SPF)X, stall rule  RHF_SAO.f90:237-336
  per-k diagonalisation, aufbau, density     RHF_SAO.f90:343-409
  maxSCF = 100, thresh = 1e-9, max_diis = 8  HF_constant.f90:2-4
"""
from __future__ import annotations

import dataclasses
import time
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

MAX_SCF = 100
THRESH = 1e-9
MAX_DIIS = 8
X_THRESH = 1e-6
LINDEP_SHIFT = 1e4


def _cell_coords(ncell):
    nx, ny, nz = ncell
    c = np.zeros((nx * ny * nz, 3), dtype=np.int64)
    idx = 0
    for iz in range(nz):
        for iy in range(ny):
            for ix in range(nx):
                c[idx] = (ix, iy, iz)
                idx += 1
    return c


def _phase(ncell):
    """phase(k, R) = exp(i 2 pi k.R / n), reduced to (-pi, pi] (SAO_Transfer.f90:34-44)."""
    c = _cell_coords(ncell)
    n = np.array(ncell, dtype=np.float64)
    theta = 2 * np.pi * ((c[:, None, :] * c[None, :, :]) / n).sum(-1)
    theta = theta - 2 * np.pi * np.rint(theta / (2 * np.pi))
    return np.exp(1j * theta)


@dataclasses.dataclass
class SAO:
    nfuc: int
    ncell: Tuple[int, int, int]

    def __post_init__(self):
        self.Nc = int(np.prod(self.ncell))
        self.ph = _phase(self.ncell)
        c = _cell_coords(self.ncell)
        n = np.array(self.ncell)
        # dR index of (R, R'): (R - R') mod n per axis, cells x fastest
        d = (c[:, None, :] - c[None, :, :]) % n
        self.dR = d[..., 0] + n[0] * (d[..., 1] + n[1] * d[..., 2])

    def to_sao(self, M: np.ndarray) -> np.ndarray:
        """transform_AO_to_SAO: k blocks B_k(a,b) = sum_R phase(k,R) M(a, b + R nfuc)."""
        nf = self.nfuc
        M0 = M[:nf, :].reshape(nf, self.Nc, nf)            # (a, R, b)
        return np.einsum("kR,aRb->kab", self.ph, M0)

    def to_ao(self, B: np.ndarray) -> np.ndarray:
        """transform_SAO_to_AO: M(mu,nu) = Re (1/Nc) sum_k phase(k, R-R') B_k(a,b)."""
        nf = self.nfuc
        Bz = np.where(np.abs(B) < 1e-15, 0.0, B)
        Tm = np.einsum("kd,kab->dab", self.ph, Bz).real / self.Nc     # (dR, a, b)
        full = Tm[self.dR]                                              # (R, R', a, b)
        return full.transpose(0, 2, 1, 3).reshape(self.Nc * nf, self.Nc * nf)


def canonical_X(U: np.ndarray, e: np.ndarray) -> Tuple[np.ndarray, int]:
    """canonical_X_real / _complex: Lowdin S^-1/2, or dropped columns below 1e-6."""
    drop = e <= X_THRESH
    if not drop.any():
        return (U * (1.0 / np.sqrt(e))) @ U.conj().T, 0
    X = U / np.sqrt(np.where(drop, 1.0, e))
    X[:, drop] = 0.0
    return X, int(drop.sum())


def shift_dropped(X: np.ndarray, Fp: np.ndarray) -> None:
    for j in range(X.shape[1]):
        if np.all(X[:, j] == 0):
            Fp[j, j] = LINDEP_SHIFT


def guess_occupy_cut(nO: int, e: np.ndarray, c: np.ndarray) -> np.ndarray:
    """Aufbau guess; a degenerate level at the cut is filled fractionally."""
    n = len(e)
    if nO <= 0:
        return np.zeros((n, n))
    tol = 1e-8 * max(1.0, abs(e[nO - 1]))
    lo = nO
    while lo > 1 and abs(e[lo - 2] - e[nO - 1]) < tol:
        lo -= 1
    hi = nO
    while hi < n and abs(e[hi] - e[nO - 1]) < tol:
        hi += 1
    if hi == nO:
        return 2.0 * c[:, :nO] @ c[:, :nO].T
    occ = 2.0 * (nO - lo + 1) / (hi - lo + 1)
    cw = np.concatenate([c[:, :lo - 1] * np.sqrt(2.0), c[:, lo - 1:hi] * np.sqrt(occ)], axis=1)
    return cw @ cw.T


def reference_sort(e: np.ndarray) -> np.ndarray:
    """The ordering RHF_SAO.f90:371-383 builds (pairwise swaps, ties keep their order)."""
    idx = list(range(len(e)))
    n = len(e)
    for mu in range(n - 1):
        for nu in range(mu + 1, n):
            if e[idx[mu]] > e[idx[nu]]:
                idx[mu], idx[nu] = idx[nu], idx[mu]
    return np.array(idx)


class DIIS:
    """DIIS_extrapolation: most recent first, bordered system, reset on rcond < 1e-14."""

    def __init__(self, size: int, n: int):
        self.err = np.zeros((size, n))
        self.vec = np.zeros((size, n))
        self.n = 0
        self.size = size

    def __call__(self, err: np.ndarray, F: np.ndarray) -> np.ndarray:
        self.n = min(self.n + 1, self.size)
        self.err[1:] = self.err[:-1].copy()
        self.vec[1:] = self.vec[:-1].copy()
        self.err[0] = err.ravel(order="F")
        self.vec[0] = F.ravel(order="F")
        m = self.n
        A = np.zeros((m + 1, m + 1))
        A[:m, :m] = self.err[:m] @ self.err[:m].T
        A[:m, m] = -1.0
        A[m, :m] = -1.0
        b = np.zeros(m + 1)
        b[m] = -1.0
        try:
            rcond = 1.0 / np.linalg.cond(A, 1)
            w = np.linalg.solve(A, b)
        except np.linalg.LinAlgError:
            rcond = 0.0
        if not np.isfinite(rcond) or rcond < 1e-14:
            self.n = 0
            self.err[:] = 0.0
            self.vec[:] = 0.0
            return F
        return (w[:m] @ self.vec[:m]).reshape(F.shape, order="F")


@dataclasses.dataclass
class RHFResult:
    energy: float               # EHF + ENuc (supercell total)
    e_electronic: float
    converged: bool
    stalled: bool
    iterations: int
    orbital_energies: np.ndarray
    history: List[Dict[str, float]]
    jk_seconds: List[float]
    iter_seconds: List[float]
    # the last diagonalisation: per k block the orbitals (SAO basis, columns by
    # ascending energy), their energies and occupations (2 or 0), as the
    # reference's blk(k) and coeff_SAO blocks
    C_k: Optional[np.ndarray] = None          # (Nc, nfuc, nfuc) complex
    eps_k: Optional[np.ndarray] = None        # (Nc, nfuc)
    occ_k: Optional[np.ndarray] = None        # (Nc, nfuc) int
    P: Optional[np.ndarray] = None            # the density of the last diagonalisation (nbas x nbas)


def core_guess_density(S: np.ndarray, T: np.ndarray, V: np.ndarray, nO: int) -> np.ndarray:
    """The starting density of rhf_sao: guess_AO_RHF_SAO (SAO/guess_RHF_SAO.f90:1-115),
    the core Hamiltonian T + V diagonalised in the canonical orthogonal basis of
    S and occupied by guess_occupy_cut."""
    e, U = np.linalg.eigh(S)
    X, _ = canonical_X(U, e)
    cp = X.T @ (T + V) @ X
    shift_dropped(X, cp)
    eg, cg = np.linalg.eigh(cp)
    return guess_occupy_cut(nO, eg, X @ cg)


def rhf_sao(S: np.ndarray, T: np.ndarray, V: np.ndarray, enuc: float, nO: int, nfuc: int, ncell,
            jk: Callable[[np.ndarray], Tuple[np.ndarray, np.ndarray]], max_scf: int = MAX_SCF,
            thresh: float = THRESH, diis: bool = True, max_diis: int = MAX_DIIS) -> RHFResult:
    """RHF_SAO (RHF_SAO.f90:1-553) with J and K from `jk(P) -> (J, K)`."""
    nbas = S.shape[0]
    sao = SAO(nfuc, tuple(int(x) for x in ncell))
    Nc = sao.Nc
    Hc = T + V
    # X from the AO overlap (main.f90:489 get_X_from_overlap)
    e, U = np.linalg.eigh(S)
    X, _ = canonical_X(U, e)
    # guess_AO_RHF_SAO
    cp = X.T @ Hc @ X
    shift_dropped(X, cp)
    eg, cg = np.linalg.eigh(cp)
    P = guess_occupy_cut(nO, eg, X @ cg)
    # SAO overlap and its per-k orthogonaliser
    S_k = sao.to_sao(S)
    X_k = np.zeros_like(S_k)
    for k in range(Nc):
        ek, Uk = np.linalg.eigh(S_k[k])
        X_k[k], _ = canonical_X(Uk, ek)

    hist: List[Dict[str, float]] = []
    jk_t: List[float] = []
    it_t: List[float] = []
    dii = DIIS(max_diis, nbas * nbas) if diis and max_diis > 1 else None
    conv, ehf, ehf_old = 1.0, 0.0, 0.0
    converged = stalled = False
    n_stable = 0
    conv_hist = np.full(5, np.inf)
    eps = np.zeros(nbas)
    C_k = occ_k = None
    nscf = 0
    while nscf < max_scf:
        t_it = time.perf_counter()
        nscf += 1
        t0 = time.perf_counter()
        J, K = jk(P)
        jk_t.append(time.perf_counter() - t0)
        F = Hc + J + K
        F = sao.to_ao(sao.to_sao(F))
        ET = float(np.sum(P * T.T))
        EV = float(np.sum(P * V.T))
        EJ = 0.5 * float(np.sum(P * J.T)) * Nc
        EK = 0.5 * float(np.sum(P * K.T)) * Nc
        ehf = ET + EV + EJ + EK
        err = F @ P @ S - S @ P @ F
        err_o = X.T @ err @ X
        if nscf > 1:
            conv = float(np.max(np.abs(err_o)))
        hist.append({"iter": nscf, "E": ehf + enuc, "conv": conv, "ET": ET, "EV": EV, "EJ": EJ, "EK": EK})
        if conv < thresh:
            converged = True
            it_t.append(time.perf_counter() - t_it)
            break
        if nscf > 2 and abs(ehf - ehf_old) < max(1e-10, 2e-10 * abs(ehf)):
            n_stable += 1
        else:
            n_stable = 0
        if n_stable >= 5 and conv < 1e-6 and conv > 0.5 * conv_hist[nscf % 5]:
            converged = stalled = True
            it_t.append(time.perf_counter() - t_it)
            break
        conv_hist[nscf % 5] = conv
        ehf_old = ehf
        if dii is not None:
            F = dii(err_o, F)
        F_k = sao.to_sao(F)
        C_k = np.zeros_like(F_k)
        for k in range(Nc):
            Fp = X_k[k].conj().T @ F_k[k] @ X_k[k]
            shift_dropped(X_k[k], Fp)
            ek, Ck = np.linalg.eigh(Fp)
            eps[k * nfuc:(k + 1) * nfuc] = ek
            C_k[k] = X_k[k] @ Ck
        idx = reference_sort(eps) if nbas <= 512 else np.argsort(eps, kind="stable")
        P_k = np.zeros_like(F_k)
        occ_k = np.zeros((Nc, nfuc), dtype=np.int32)
        for i in range(nO):
            o = idx[i]
            kb, col = divmod(int(o), nfuc)
            occ_k[kb, col] = 2
            c = C_k[kb][:, col]
            P_k[kb] += 2.0 * np.outer(c, c.conj())
        P = sao.to_ao(P_k)
        it_t.append(time.perf_counter() - t_it)
    return RHFResult(energy=ehf + enuc, e_electronic=ehf, converged=converged, stalled=stalled, iterations=nscf,
                     orbital_energies=np.sort(eps), history=hist, jk_seconds=jk_t, iter_seconds=it_t,
                     C_k=C_k, eps_k=eps.reshape(Nc, nfuc).copy(), occ_k=occ_k, P=P)


def fill_with_symmetry(rows: np.ndarray, nfuc: int, ncell) -> np.ndarray:
    """Full nbas x nbas matrix from its unit-cell rows (fill_with_symmetry,
    Tools/symmetric_matrix.f90:1-52): M(a + R nfuc, j) = M(a, j shifted by -R)."""
    nx, ny, nz = ncell
    Nc = nx * ny * nz
    nbas = nfuc * Nc
    c = _cell_coords(ncell)
    n = np.array(ncell)
    M = np.zeros((nbas, nbas))
    M[:nfuc] = rows
    for R in range(1, Nc):
        src = (c - c[R]) % n
        srci = src[:, 0] + n[0] * (src[:, 1] + n[1] * src[:, 2])
        cols = (srci[:, None] * nfuc + np.arange(nfuc)[None, :]).ravel()
        M[R * nfuc:(R + 1) * nfuc] = rows[:, cols]
    return M


def n_occupied(sysm) -> int:
    """nO = n_electron / 2 (main.f90:263), neutral supercell."""
    ne = int(np.sum(sysm.charges))
    if ne % 2:
        raise ValueError("RHF needs an even number of electrons (%d)" % ne)
    return ne // 2
