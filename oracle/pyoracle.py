"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
FAST_LIB_PATH = os.path.join(HERE, "liboracle_fast.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class OrcSystem(C.Structure):
    _fields_ = [("ndp", C.c_int32), ("ncell", C.c_int32 * 3), ("nfuc", C.c_int32), ("nbas", C.c_int32),
                ("nquad", C.c_int32), ("L", C.c_double * 3), ("ctr", _dp), ("lxyz", _ip),
                ("prim_off", _ip), ("exps", _dp), ("coefs", _dp), ("t_nodes", _dp), ("t_weights", _dp),
                ("physicist", C.c_int32), ("sao", C.c_int32), ("prim_screen", C.c_int32),
                ("schwarz_thr", C.c_double), ("prim_thr", C.c_double)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def build_fast(force=True):
    """The timing build (reference compiler flags, -march=native, pair-vector
    memo) for this host; rebuilt by default since -march=native ties it to the
    machine that compiles it."""
    subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if force else []) + ["fast"], check=True)


_lib = None
_lib_fast = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = _bind(C.CDLL(LIB_PATH))
    return _lib


def lib_fast():
    """liboracle_fast.so (built for this host by build_fast first if absent)."""
    global _lib_fast
    if _lib_fast is None:
        if not os.path.exists(FAST_LIB_PATH):
            build_fast()
        _lib_fast = _bind(C.CDLL(FAST_LIB_PATH))
    return _lib_fast


def _bind(L):
    if True:
        L.orc_iv_log.restype = C.c_double
        L.orc_iv_log.argtypes = [C.c_double, C.c_double]
        L.orc_iv_scaled.restype = C.c_double
        L.orc_iv_scaled.argtypes = [C.c_int, C.c_double]
        L.orc_bessel_scaled_vector.argtypes = [C.c_int, C.c_double, _dp]
        L.orc_bessel_scaled_vector_fast.argtypes = [C.c_int, C.c_double, _dp]
        L.orc_bessel_nmax_estimate.restype = C.c_int
        L.orc_bessel_nmax_estimate.argtypes = [C.c_double]
        L.orc_fourier_sin_product.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _dp, _dp]
        L.orc_pair_vector.argtypes = [C.c_int, C.c_double, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, _dp, _dp]
        L.orc_fast_quad_points.argtypes = [C.c_int, _dp, _dp]
        L.orc_bary.argtypes = [C.c_double] * 6 + [_dp, _dp]
        L.orc_hermite_E_1D.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _dp]
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcSystem)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_nshells.restype = C.c_int
        L.orc_nshells.argtypes = [C.c_void_p, _ip, _ip]
        L.orc_shell_info.argtypes = [C.c_void_p, C.c_int, _ip, _ip]
        L.orc_schwarz.restype = _dp
        L.orc_schwarz.argtypes = [C.c_void_p]
        L.orc_schwarz_shell.restype = _dp
        L.orc_schwarz_shell.argtypes = [C.c_void_p]
        L.orc_prim_table.restype = _dp
        L.orc_prim_table.argtypes = [C.c_void_p, _ip]
        L.orc_t_tables.argtypes = [C.c_void_p, C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_ip)]
        L.orc_shell_block.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp]
        L.orc_eri_stored.restype = C.c_int64
        L.orc_eri_stored.argtypes = [C.c_void_p, _dp]
        L.orc_direct_jk.restype = C.c_int64
        L.orc_direct_jk.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_hartree_exchange.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp]
        L.orc_sym_fill_eri.argtypes = [C.c_int, C.c_int, _ip, _dp]
        L.orc_count.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_items.restype = C.c_int64
        L.orc_items.argtypes = [C.c_void_p, _ip, C.c_int64]
        L.orc_direct_jk_items.restype = C.c_int64
        L.orc_direct_jk_items.argtypes = [C.c_void_p, _ip, C.c_int64, _dp, _dp, _dp]
        L.orc_one_electron.argtypes = [C.c_void_p, C.c_int, _dp, _ip, _dp, _dp, _dp]
        L.orc_nuclear_repulsion.restype = C.c_double
        L.orc_nuclear_repulsion.argtypes = [C.c_int, _dp, C.c_int, _dp, _ip]
        L.orc_overlap_pair.restype = C.c_double
        L.orc_overlap_pair.argtypes = [C.c_int, _dp, _ip, _ip, _dp, _dp, C.c_int, _dp, _dp, C.c_int, _dp, _dp]
        L.orc_normalize.restype = C.c_double
        L.orc_normalize.argtypes = [C.c_int, _dp, C.c_int, _dp, _ip, _ip, _dp, _dp]
        L.orc_pair_cache_free.argtypes = []
        L.orc_shell_blocks.restype = C.c_int64
        L.orc_shell_blocks.argtypes = [C.c_void_p, C.c_int64, _ip, C.c_int, _dp]
    return L


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_ip)


# ---------------------------------------------------------------------------
def iv_log(v, x):
    return lib().orc_iv_log(float(v), float(x))


def iv_scaled(n, x):
    return lib().orc_iv_scaled(int(n), float(x))


def bessel_vector(N, A, fast=False):
    out = np.zeros(N + 1)
    (lib().orc_bessel_scaled_vector_fast if fast else lib().orc_bessel_scaled_vector)(int(N), float(A), dptr(out))
    return out


def nmax_estimate(A):
    return lib().orc_bessel_nmax_estimate(float(A))


def pair_vector(N, A, i, l, phA, phB, sgn):
    re = np.zeros(N + 1)
    im = np.zeros(N + 1)
    lib().orc_pair_vector(N, A, i, l, phA, phB, sgn, dptr(re), dptr(im))
    return re + 1j * im


def fast_quad(n):
    t = np.zeros(n)
    w = np.zeros(n)
    lib().orc_fast_quad_points(n, dptr(t), dptr(w))
    return t, w


def normalize(sys) -> float:
    """normalize_AO_toroidal_{1,2,3}D in place on sys.coefs; returns max |<phi|phi>-1|."""
    L = np.ascontiguousarray(sys.L, dtype=np.float64)
    ctr = np.ascontiguousarray(sys.ctr, dtype=np.float64)
    lxyz = np.ascontiguousarray(sys.lxyz, dtype=np.int32)
    poff = np.ascontiguousarray(sys.prim_off, dtype=np.int32)
    exps = np.ascontiguousarray(sys.exps, dtype=np.float64)
    coefs = np.ascontiguousarray(sys.coefs, dtype=np.float64)
    dev = lib().orc_normalize(sys.ndp, dptr(L), sys.nbas, dptr(ctr), iptr(lxyz), iptr(poff), dptr(exps), dptr(coefs))
    sys.coefs = coefs
    return dev


class Oracle:
    """The oracle engine for one supercell basis (direct_init + drivers)."""

    def __init__(self, sys, nquad=32, t_nodes=None, t_weights=None, physicist=False, sao=True,
                 prim_screen=True, schwarz_thr=1e-13, prim_thr=1e-14, fast=False):
        """fast=True: the timing build (liboracle_fast.so, reference compiler
        flags and pair-vector memo) instead of the parity build."""
        self.L = lib_fast() if fast else lib()
        self.sys = sys
        self._keep = [np.ascontiguousarray(sys.ctr, dtype=np.float64).ravel(),
                      np.ascontiguousarray(sys.lxyz, dtype=np.int32).ravel(),
                      np.ascontiguousarray(sys.prim_off, dtype=np.int32),
                      np.ascontiguousarray(sys.exps, dtype=np.float64),
                      np.ascontiguousarray(sys.coefs, dtype=np.float64)]
        s = OrcSystem()
        s.ndp = sys.ndp
        for d in range(3):
            s.ncell[d] = sys.ncell[d]
            s.L[d] = sys.L[d]
        s.nfuc = sys.nfuc
        s.nbas = sys.nbas
        s.nquad = nquad
        s.ctr = dptr(self._keep[0])
        s.lxyz = iptr(self._keep[1])
        s.prim_off = iptr(self._keep[2])
        s.exps = dptr(self._keep[3])
        s.coefs = dptr(self._keep[4])
        if t_nodes is not None:
            tn = np.ascontiguousarray(t_nodes, dtype=np.float64)
            tw = np.ascontiguousarray(t_weights, dtype=np.float64)
            self._keep += [tn, tw]
            s.nquad = len(tn)
            s.t_nodes = dptr(tn)
            s.t_weights = dptr(tw)
        s.physicist = int(physicist)
        s.sao = int(sao)
        s.prim_screen = int(prim_screen)
        s.schwarz_thr = schwarz_thr
        s.prim_thr = prim_thr
        self.nquad = s.nquad
        self.sao = sao
        self.physicist = physicist
        self._s = s
        self.h = self.L.orc_create(C.byref(s))

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- introspection
    def shells(self):
        nshuc = C.c_int32()
        ncap = C.c_int32()
        nsh = self.L.orc_nshells(self.h, C.byref(nshuc), C.byref(ncap))
        out = []
        for s in range(nsh):
            f = C.c_int32()
            n = C.c_int32()
            self.L.orc_shell_info(self.h, s, C.byref(f), C.byref(n))
            out.append((f.value, n.value))
        return out, nshuc.value, ncap.value

    def schwarz(self):
        n = self.sys.nbas
        p = self.L.orc_schwarz(self.h)
        return np.ctypeslib.as_array(p, shape=(n * n,)).reshape(n, n, order="F").copy()

    def prim_table(self):
        mp = C.c_int32()
        p = self.L.orc_prim_table(self.h, C.byref(mp))
        if not p:
            return None
        sh, nshuc, _ = self.shells()
        tot = mp.value * mp.value * nshuc * len(sh)
        return np.ctypeslib.as_array(p, shape=(tot,)).reshape(mp.value, mp.value, nshuc, len(sh), order="F").copy()

    def t_tables(self):
        node = _dp()
        w = _dp()
        tb = _dp()
        tn = _ip()
        self.L.orc_t_tables(self.h, C.byref(node), C.byref(w), C.byref(tb), C.byref(tn))
        _, _, ncap = self.shells()
        nq, ndp = self.nquad, self.sys.ndp
        return (np.ctypeslib.as_array(node, shape=(nq,)).copy(), np.ctypeslib.as_array(w, shape=(nq,)).copy(),
                np.ctypeslib.as_array(tb, shape=((ncap + 1) * nq * ndp,)).reshape(ncap + 1, nq, ndp, order="F").copy(),
                np.ctypeslib.as_array(tn, shape=(nq * ndp,)).reshape(nq, ndp, order="F").copy())

    def shell_block(self, S1, S2, S3, S4, mode=1):
        sh, _, _ = self.shells()
        n = [sh[S][1] for S in (S1, S2, S3, S4)]
        blk = np.zeros(n[0] * n[1] * n[2] * n[3])
        self.L.orc_shell_block(self.h, S1, S2, S3, S4, mode, dptr(blk))
        return blk.reshape(n, order="F")

    def shell_blocks(self, items, mode=1):
        """Blocks of the given shell quartets (rows of 4), concatenated in item
        order (each column-major), and their offsets; OpenMP over the quartets."""
        it = np.ascontiguousarray(items, dtype=np.int32).reshape(-1, 4)
        sh, _, _ = self.shells()
        n = np.array([x[1] for x in sh], dtype=np.int64)
        sizes = np.prod(n[it], axis=1) if len(it) else np.zeros(0, dtype=np.int64)
        offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        out = np.zeros(max(int(offs[-1]), 1))
        if len(it):
            self.L.orc_shell_blocks(self.h, len(it), iptr(it), int(mode), dptr(out))
        return out[:offs[-1]], offs

    def eri_stored(self):
        n = self.sys.nbas
        esz = self.sys.nfuc if self.sao else n
        eri = np.zeros(esz * n * n * n)
        nq = self.L.orc_eri_stored(self.h, dptr(eri))
        return eri.reshape((esz, n, n, n), order="F"), nq

    def direct_jk(self, P):
        n = self.sys.nbas
        Pf = np.asfortranarray(P, dtype=np.float64).ravel(order="F").copy()
        J = np.zeros(n * n)
        K = np.zeros(n * n)
        nq = self.L.orc_direct_jk(self.h, dptr(Pf), dptr(J), dptr(K))
        return J.reshape(n, n, order="F"), K.reshape(n, n, order="F"), nq

    def items(self) -> np.ndarray:
        n = self.L.orc_items(self.h, None, 0)
        out = np.zeros((max(n, 1), 4), dtype=np.int32)
        self.L.orc_items(self.h, iptr(out), n)
        return out[:n]

    def direct_jk_items(self, items, P, J=None, K=None):
        """Accumulate the J/K contributions of the given quartets; returns (J, K, nfunc)."""
        n = self.sys.nbas
        it = np.ascontiguousarray(items, dtype=np.int32)
        Pf = np.asfortranarray(P, dtype=np.float64).ravel(order="F").copy()
        Jf = np.zeros(n * n) if J is None else np.asfortranarray(J).ravel(order="F").copy()
        Kf = np.zeros(n * n) if K is None else np.asfortranarray(K).ravel(order="F").copy()
        nf = self.L.orc_direct_jk_items(self.h, iptr(it), len(it), dptr(Pf), dptr(Jf), dptr(Kf))
        return Jf.reshape(n, n, order="F"), Kf.reshape(n, n, order="F"), nf

    def one_electron(self):
        """S, T, V of the supercell (rows of the unit cell computed, the rest by translation)."""
        n = self.sys.nbas
        geo = np.ascontiguousarray(self.sys.geometry, dtype=np.float64).ravel()
        Z = np.ascontiguousarray(self.sys.charges, dtype=np.int32)
        S, T, V = (np.zeros(n * n) for _ in range(3))
        self.L.orc_one_electron(self.h, len(Z), dptr(geo), iptr(Z), dptr(S), dptr(T), dptr(V))
        return tuple(M.reshape(n, n, order="F") for M in (S, T, V))

    def count(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        self.L.orc_count(self.h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value


def hartree_exchange(n1, P, eri, physicist=False):
    n = P.shape[0]
    Pf = np.asfortranarray(P, dtype=np.float64).ravel(order="F").copy()
    E = np.asfortranarray(eri, dtype=np.float64).ravel(order="F").copy()
    J = np.zeros(n * n)
    K = np.zeros(n * n)
    lib().orc_hartree_exchange(n1, n, int(physicist), dptr(Pf), dptr(E), dptr(J), dptr(K))
    return J.reshape(n, n, order="F"), K.reshape(n, n, order="F")


def nuclear_repulsion(sys) -> float:
    L = np.ascontiguousarray(sys.L, dtype=np.float64)
    geo = np.ascontiguousarray(sys.geometry, dtype=np.float64).ravel()
    Z = np.ascontiguousarray(sys.charges, dtype=np.int32)
    return lib().orc_nuclear_repulsion(sys.ndp, dptr(L), len(Z), dptr(geo), iptr(Z))
