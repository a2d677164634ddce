"""Python host mirror of the reference's integral/SCF-path interface, over the
C ABI of libtce.so (include/tce.h).

Names follow the Fortran routines they replace:

    Engine(system)                  direct_init (eri_direct.f90:76) + ERI driver preamble
    Engine.ERI_shell_block(...)     ERI_shell_block_toroidal (ERI_shell_block_toroidal.f90:28)
    Engine.ERI_integral_toroidal()  ERI_integral_toroidal (ERI_toroidal.f90:36)
    Engine.direct_JK(P)             direct_JK (eri_direct.f90:262)
    Engine.stored_JK(P)             hartree_exchange_potential on the device-resident ERIs
    hartree_exchange_potential(...) hartree_exchange_potential (hartree_exchange_potential.f90:30)

Errors: the reference stops (`error stop`); here a nonzero status raises
TCEError with the library's message.  There is no CPU fallback: without the
library or a usable GPU every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple

import numpy as np

from .system import AOSystem

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtce.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)

TCE_OK, TCE_ERR_ARG, TCE_ERR_UNSUPPORTED, TCE_ERR_CUDA, TCE_ERR_STATE, TCE_ERR_NOMEM = range(6)

# every symbol include/tce.h declares
EXPORTS = ["tce_create", "tce_destroy", "tce_last_error", "tce_get_info", "tce_shell_block", "tce_shells",
           "tce_schwarz", "tce_eri_stored", "tce_stored_jk", "tce_hartree_exchange", "tce_direct_jk",
           "tce_direct_jk_device", "tce_last_kernel_ms", "tce_set_shard", "tce_shard_plan", "tce_fp64_peak",
           "tce_shell_block_noalloc", "tce_version",
           "tce_items", "tce_item_features", "tce_lg_set_rules", "tce_lg_rule_gmax", "tce_set_plain_rule",
           "tce_lg_set_item_rules", "tce_lg_item_rules", "tce_set_method", "tce_set_tolerances", "tce_lg_stats",
           "tce_rule_blocks", "tce_mlp_create", "tce_mlp_destroy", "tce_mlp_last_error", "tce_mlp_nparams",
           "tce_mlp_get_params", "tce_mlp_set_params", "tce_mlp_loss_grad", "tce_mlp_train", "tce_mlp_predict",
           "tce_lg_predict_rules", "tce_lg_work", "tce_quad_self_check", "tce_set_graph",
           "tce_set_fp32_threshold", "tce_dfmp2_energy", "tce_mp2_last_error", "tce_create_blocks",
           "tce_pass_kernels", "tce_set_tensor_cores", "tce_set_list_streams", "tce_nuclear_attraction", "tce_quad_self_check_nuc",
           "tce_lg_autotune", "tce_lg_lists", "tce_dfjk_create", "tce_dfjk", "tce_dfjk_destroy",
           "tce_dfjk_last_error", "tce_ao_to_kmo", "tce_shard_items", "tce_lg_list_profile",
           "tce_df_create", "tce_df_destroy", "tce_df_last_error", "tce_df_integrals", "tce_df_fitted", "tce_dfmp2",
           "tce_gk_rule", "tce_lg_dictionary", "tce_lg_setup", "tce_lg_set_list_form",
           "tce_trexio_eri"]

TCE_METHOD_FIXED, TCE_METHOD_LEARNED, TCE_METHOD_PLAIN = 0, 1, 2
TCE_NFEAT = 12
_fp = C.POINTER(C.c_float)
_lp = C.POINTER(C.c_int64)


class TCEError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("libtce error %d: %s" % (code, msg))
        self.code = code


class TceSystem(C.Structure):
    _fields_ = [("ndp", C.c_int32), ("ncell", C.c_int32 * 3), ("nfuc", C.c_int32), ("nbas", C.c_int32),
                ("nquad", C.c_int32), ("L", C.c_double * 3), ("ctr", _dp), ("lxyz", _ip),
                ("prim_off", _ip), ("exps", _dp), ("coefs", _dp), ("t_nodes", _dp), ("t_weights", _dp),
                ("physicist", C.c_int32), ("sao", C.c_int32), ("prim_screen", C.c_int32),
                ("schwarz_thr", C.c_double), ("prim_thr", C.c_double)]


class TceInfo(C.Structure):
    _fields_ = [("nsh", C.c_int32), ("nshuc", C.c_int32), ("ncap", C.c_int32), ("nquad", C.c_int32),
                ("n_shell_quartets", C.c_int64), ("n_func_quartets", C.c_int64),
                ("n_unit_pairs", C.c_int64), ("device_bytes", C.c_int64), ("n_prim_quartets", C.c_int64),
                ("jk_flops", C.c_double), ("shard_rank", C.c_int32), ("shard_nranks", C.c_int32),
                ("shard_shell_quartets", C.c_int64)]


_lib = None


def lib():
    """Load libtce.so (built in-tree).  Raises if it is missing: no fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise TCEError(TCE_ERR_CUDA, "libtce.so is not built (run william_ci_b200.build.build())")
        L = C.CDLL(LIB_PATH)
        L.tce_create.argtypes = [C.POINTER(TceSystem), C.POINTER(C.c_void_p)]
        L.tce_create_blocks.argtypes = [C.POINTER(TceSystem), C.POINTER(C.c_void_p)]
        L.tce_destroy.argtypes = [C.c_void_p]
        L.tce_last_error.restype = C.c_char_p
        L.tce_last_error.argtypes = [C.c_void_p]
        L.tce_get_info.argtypes = [C.c_void_p, C.POINTER(TceInfo)]
        L.tce_shell_block.argtypes = [C.c_void_p, _ip, C.c_int32, _dp]
        L.tce_shell_block_noalloc.argtypes = [C.c_void_p, _ip, C.c_int32, _dp]
        L.tce_shells.argtypes = [C.c_void_p, _ip, _ip]
        L.tce_schwarz.argtypes = [C.c_void_p, _dp]
        L.tce_eri_stored.argtypes = [C.c_void_p, C.c_int64, _dp]
        L.tce_stored_jk.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.tce_hartree_exchange.argtypes = [C.c_int32, C.c_int32, C.c_int32, _dp, _dp, _dp, _dp]
        L.tce_direct_jk.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.tce_direct_jk_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.tce_last_kernel_ms.argtypes = [C.c_void_p, _dp]
        L.tce_set_shard.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
        L.tce_shard_plan.argtypes = [_dp, C.c_int64, C.c_int32, _ip]
        L.tce_shard_items.argtypes = [C.c_void_p, _lp, _ip]
        L.tce_fp64_peak.argtypes = [_dp]
        L.tce_version.restype = C.c_char_p
        L.tce_items.argtypes = [C.c_void_p, _ip]
        L.tce_item_features.argtypes = [C.c_void_p, C.c_int64, _ip, _fp]
        L.tce_lg_set_rules.argtypes = [C.c_void_p, C.c_int32, _ip, _dp, _dp, _dp]
        L.tce_lg_rule_gmax.argtypes = [C.c_void_p, _ip]
        L.tce_set_plain_rule.argtypes = [C.c_void_p, C.c_int32, _dp, _dp, _dp, C.c_double]
        L.tce_lg_set_item_rules.argtypes = [C.c_void_p, _ip]
        L.tce_lg_item_rules.argtypes = [C.c_void_p, _ip]
        L.tce_set_method.argtypes = [C.c_void_p, C.c_int32]
        L.tce_set_tolerances.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int32]
        L.tce_lg_stats.argtypes = [C.c_void_p, _lp]
        L.tce_rule_blocks.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int64, _ip, _dp, _dp]
        L.tce_mlp_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(C.c_void_p)]
        L.tce_mlp_destroy.argtypes = [C.c_void_p]
        L.tce_mlp_last_error.restype = C.c_char_p
        L.tce_mlp_last_error.argtypes = [C.c_void_p]
        L.tce_mlp_nparams.argtypes = [C.c_void_p, _lp]
        L.tce_mlp_get_params.argtypes = [C.c_void_p, _fp, _fp, _fp]
        L.tce_mlp_set_params.argtypes = [C.c_void_p, _fp, _fp, _fp]
        L.tce_mlp_loss_grad.argtypes = [C.c_void_p, C.c_int64, _fp, _fp, _fp, _fp]
        L.tce_mlp_train.argtypes = [C.c_void_p, C.c_int64, _fp, _fp, C.c_int32, C.c_int32, C.c_float, C.c_uint64,
                                    _fp]
        L.tce_mlp_predict.argtypes = [C.c_void_p, C.c_int64, _fp, _fp]
        L.tce_lg_predict_rules.argtypes = [C.c_void_p, C.c_void_p, C.c_double]
        L.tce_lg_work.argtypes = [C.c_void_p, _dp, _lp]
        L.tce_quad_self_check.argtypes = [C.c_void_p, C.c_void_p, _dp, _ip]
        L.tce_set_graph.argtypes = [C.c_void_p, C.c_int32]
        L.tce_pass_kernels.argtypes = [C.c_void_p, _ip]
        L.tce_set_tensor_cores.argtypes = [C.c_void_p, C.c_int32]
        L.tce_set_list_streams.argtypes = [C.c_void_p, C.c_int32]
        L.tce_nuclear_attraction.argtypes = [C.c_void_p, C.c_int32, _dp, _ip, _dp]
        L.tce_lg_autotune.argtypes = [C.c_void_p, C.c_int32, _ip, _ip, _dp]
        L.tce_lg_lists.argtypes = [C.c_void_p, _ip, _ip]
        L.tce_lg_list_profile.argtypes = [C.c_void_p, C.c_int32, _ip, _dp, _dp]
        L.tce_lg_set_list_form.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
        L.tce_trexio_eri.argtypes = [C.c_void_p, C.c_int64, _ip, _dp, _lp]
        L.tce_ao_to_kmo.argtypes = [C.c_void_p, _dp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _dp]
        L.tce_dfjk_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, _ip, _dp, _dp, C.POINTER(C.c_void_p)]
        L.tce_dfjk.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.tce_dfjk_destroy.argtypes = [C.c_void_p]
        L.tce_dfjk_last_error.restype = C.c_char_p
        L.tce_dfjk_last_error.argtypes = [C.c_void_p]
        L.tce_quad_self_check_nuc.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, _dp, _ip, _dp, _dp, _ip, _ip]
        L.tce_set_fp32_threshold.argtypes = [C.c_void_p, C.c_double]
        L.tce_dfmp2_energy.argtypes = [C.c_int32, _ip, _ip, C.c_int32, C.c_int32, C.c_int32, _dp, _dp, _ip, _dp,
                                       _ip, C.c_int32, _dp, _dp, _lp, _dp, _dp]
        L.tce_mp2_last_error.restype = C.c_char_p
        L.tce_df_create.argtypes = [C.POINTER(TceSystem), C.POINTER(TceSystem), C.c_int32, _dp, C.POINTER(C.c_void_p)]
        L.tce_df_destroy.argtypes = [C.c_void_p]
        L.tce_df_last_error.restype = C.c_char_p
        L.tce_df_last_error.argtypes = [C.c_void_p]
        L.tce_df_integrals.argtypes = [C.c_void_p, _dp, _dp]
        L.tce_df_fitted.argtypes = [C.c_void_p, _dp, _dp, _ip]
        L.tce_dfmp2.argtypes = [C.c_void_p, _dp, _dp, _ip, C.c_int32, _dp, _dp, _dp]
        L.tce_gk_rule.argtypes = [C.c_int32, _dp, _dp, _dp]
        L.tce_lg_dictionary.argtypes = [_ip, _ip, _dp, _dp, _dp]
        L.tce_lg_setup.argtypes = [C.c_void_p, C.c_int64, C.c_uint64, C.c_int32, C.c_double, C.POINTER(C.c_void_p)]
        _lib = L
    return _lib


def _check(code: int, h=None):
    if code != TCE_OK:
        msg = lib().tce_last_error(h)
        raise TCEError(code, msg.decode() if msg else "")


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def tce_system(system: AOSystem, nquad: int = 32, t_nodes=None, t_weights=None, physicist=False, sao=True,
               prim_screen=True, schwarz_thr=1e-13, prim_thr=1e-14):
    """The flat tce_system of a supercell basis, and the arrays it points into
    (keep them alive as long as the struct is used)."""
    keep = [np.ascontiguousarray(system.ctr, dtype=np.float64).ravel(),
            np.ascontiguousarray(system.lxyz, dtype=np.int32).ravel(),
            np.ascontiguousarray(system.prim_off, dtype=np.int32),
            np.ascontiguousarray(system.exps, dtype=np.float64),
            np.ascontiguousarray(system.coefs, dtype=np.float64)]
    s = TceSystem()
    s.ndp = system.ndp
    for d in range(3):
        s.ncell[d] = system.ncell[d]
        s.L[d] = system.L[d]
    s.nfuc = system.nfuc
    s.nbas = system.nbas
    s.nquad = nquad
    s.ctr, s.lxyz, s.prim_off, s.exps, s.coefs = (_d(keep[0]), _i(keep[1]), _i(keep[2]), _d(keep[3]), _d(keep[4]))
    if t_nodes is not None:
        tn = np.ascontiguousarray(t_nodes, dtype=np.float64)
        tw = np.ascontiguousarray(t_weights, dtype=np.float64)
        keep += [tn, tw]
        s.nquad = len(tn)
        s.t_nodes, s.t_weights = _d(tn), _d(tw)
    s.physicist, s.sao, s.prim_screen = int(physicist), int(sao), int(prim_screen)
    s.schwarz_thr, s.prim_thr = schwarz_thr, prim_thr
    return s, keep


class Engine:
    """Device engine for one supercell basis (normalised coefficients)."""

    def __init__(self, system: AOSystem, nquad: int = 32, t_nodes=None, t_weights=None, physicist=False,
                 sao=True, prim_screen=True, schwarz_thr=1e-13, prim_thr=1e-14, blocks_only=False):
        self.sys = system
        self.physicist = bool(physicist)
        self.sao = bool(sao)
        s, self._keep = tce_system(system, nquad, t_nodes, t_weights, physicist, sao, prim_screen, schwarz_thr,
                                   prim_thr)
        self._s = s
        h = C.c_void_p()
        create = lib().tce_create_blocks if blocks_only else lib().tce_create
        code = create(C.byref(s), C.byref(h))
        if code != TCE_OK:
            msg = lib().tce_last_error(None)
            raise TCEError(code, msg.decode() if msg else "")
        self.h = h
        self.nbas = system.nbas
        self.nfuc = system.nfuc

    def close(self):
        if getattr(self, "h", None):
            lib().tce_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---------------- introspection ----------------
    def info(self) -> dict:
        inf = TceInfo()
        _check(lib().tce_get_info(self.h, C.byref(inf)), self.h)
        return {f: getattr(inf, f) for f, _ in TceInfo._fields_}

    def shells(self):
        n = self.info()["nsh"]
        first = np.zeros(n, dtype=np.int32)
        cnt = np.zeros(n, dtype=np.int32)
        _check(lib().tce_shells(self.h, _i(first), _i(cnt)), self.h)
        return list(zip(first.tolist(), cnt.tolist()))

    def schwarz(self) -> np.ndarray:
        Q = np.zeros(self.nbas * self.nbas)
        _check(lib().tce_schwarz(self.h, _d(Q)), self.h)
        return Q.reshape(self.nbas, self.nbas, order="F")

    # ---------------- the path ----------------
    def ERI_shell_block(self, S1, S2, S3, S4, mode=1) -> np.ndarray:
        sh = self.shells()
        n = [sh[S][1] for S in (S1, S2, S3, S4)]
        blk = np.zeros(int(np.prod(n)))
        q = np.array([S1, S2, S3, S4], dtype=np.int32)
        _check(lib().tce_shell_block(self.h, _i(q), int(mode), _d(blk)), self.h)
        return blk.reshape(n, order="F")

    def ERI_shell_block_noalloc(self, S1, S2, S3, S4, mode=1) -> np.ndarray:
        """tce_shell_block_noalloc: the same block, scratch in the library's static device array."""
        sh = self.shells()
        n = [sh[S][1] for S in (S1, S2, S3, S4)]
        blk = np.zeros(int(np.prod(n)))
        q = np.array([S1, S2, S3, S4], dtype=np.int32)
        _check(lib().tce_shell_block_noalloc(self.h, _i(q), int(mode), _d(blk)), self.h)
        return blk.reshape(n, order="F")

    def trexio_eri(self):
        """The integral stream of the TREXIO export (tce_trexio_eri) from the full
        stored integrals (run ERI_integral_toroidal with sao=False first):
        indices (count, 4) 1-based (i, j, k, l) and values ERI(i, k, j, l)."""
        n = C.c_int64()
        _check(lib().tce_trexio_eri(self.h, 0, None, None, C.byref(n)), self.h)
        idx = np.zeros(4 * max(n.value, 1), dtype=np.int32)
        val = np.zeros(max(n.value, 1))
        _check(lib().tce_trexio_eri(self.h, n.value, _i(idx), _d(val), C.byref(n)), self.h)
        return idx[:4 * n.value].reshape(n.value, 4), val[:n.value]

    def ERI_integral_toroidal(self) -> np.ndarray:
        n = self.nbas
        esz = self.nfuc if self.sao else n
        eri = np.zeros(esz * n * n * n)
        _check(lib().tce_eri_stored(self.h, esz, _d(eri)), self.h)
        return eri.reshape((esz, n, n, n), order="F")

    def ao_to_kmo(self, C_k: np.ndarray, p_rng, q_rng) -> np.ndarray:
        """(p k1, q k2 | r k3, s k4) from the stored SAO integrals (tce_ao_to_kmo);
        C_k (cells, nfuc, nfuc) the k-block orbitals, p_rng / q_rng 0-based
        half-open band ranges.  Run ERI_integral_toroidal first (SAO, chemist)."""
        N, nf = C_k.shape[0], C_k.shape[1]
        n = self.nbas
        coeff = np.zeros((n, n), dtype=np.complex128)
        for k in range(N):
            coeff[k * nf:(k + 1) * nf, k * nf:(k + 1) * nf] = C_k[k]
        cf = np.asfortranarray(coeff).ravel(order="F").copy().view(np.float64)
        (p0, p1), (q0, q1) = p_rng, q_rng
        no, nv = p1 - p0, q1 - q0
        out = np.zeros(2 * no * nv * no * nv * N ** 3)
        _check(lib().tce_ao_to_kmo(self.h, _d(cf), p0 + 1, p1, q0 + 1, q1, _d(out)), self.h)
        return out.view(np.complex128).reshape((no, nv, no, nv, N, N, N), order="F")

    def direct_JK(self, P: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        n = self.nbas
        Pf = np.asfortranarray(P, dtype=np.float64).ravel(order="F").copy()
        J = np.zeros(n * n)
        K = np.zeros(n * n)
        _check(lib().tce_direct_jk(self.h, _d(Pf), _d(J), _d(K)), self.h)
        return J.reshape(n, n, order="F"), K.reshape(n, n, order="F")

    def direct_JK_ptrs(self, P_ptr: int, J_ptr: int, K_ptr: int):
        """tce_direct_jk on caller-owned host buffers (e.g. pinned), nbas x nbas column-major."""
        _check(lib().tce_direct_jk(self.h, C.cast(P_ptr, _dp), C.cast(J_ptr, _dp), C.cast(K_ptr, _dp)), self.h)

    def direct_JK_device(self, dP_ptr: int, dJ_ptr: int, dK_ptr: int, stream_ptr: int = 0):
        _check(lib().tce_direct_jk_device(self.h, C.c_void_p(dP_ptr), C.c_void_p(dJ_ptr), C.c_void_p(dK_ptr),
                                          C.c_void_p(stream_ptr)), self.h)

    def last_kernel_ms(self) -> float:
        v = C.c_double()
        _check(lib().tce_last_kernel_ms(self.h, C.byref(v)), self.h)
        return v.value

    def set_shard(self, rank: int, nranks: int):
        _check(lib().tce_set_shard(self.h, int(rank), int(nranks)), self.h)

    def shard_items(self) -> np.ndarray:
        """The shell quartets of the current shard (tce_shard_items), shape (n, 4)."""
        n = C.c_int64()
        _check(lib().tce_shard_items(self.h, C.byref(n), None), self.h)
        it = np.zeros(4 * max(n.value, 1), dtype=np.int32)
        _check(lib().tce_shard_items(self.h, C.byref(n), _i(it)), self.h)
        return it[:4 * n.value].reshape(n.value, 4)

    def stored_JK(self, P: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        n = self.nbas
        Pf = np.asfortranarray(P, dtype=np.float64).ravel(order="F").copy()
        J = np.zeros(n * n)
        K = np.zeros(n * n)
        _check(lib().tce_stored_jk(self.h, _d(Pf), _d(J), _d(K)), self.h)
        return J.reshape(n, n, order="F"), K.reshape(n, n, order="F")


    # ---------------- learned grid / plain method ----------------
    def items(self) -> np.ndarray:
        """The engine's unique shell quartets (most expensive first), shape (n, 4)."""
        n = self.info()["n_shell_quartets"]
        it = np.zeros(4 * n, dtype=np.int32)
        if n:
            _check(lib().tce_items(self.h, _i(it)), self.h)
        return it.reshape(n, 4)

    def item_features(self, items: Optional[np.ndarray] = None) -> np.ndarray:
        if items is None:
            n = self.info()["n_shell_quartets"]
            ptr = None
        else:
            items = np.ascontiguousarray(items, dtype=np.int32).reshape(-1, 4)
            n = len(items)
            ptr = _i(items)
        F = np.zeros(n * TCE_NFEAT, dtype=np.float32)
        if n:
            _check(lib().tce_item_features(self.h, n, ptr, F.ctypes.data_as(_fp)), self.h)
        return F.reshape(n, TCE_NFEAT)

    def lg_set_rules(self, rules):
        """rules: list of (t, wk, wg) arrays of at most 64 nodes each."""
        R = len(rules)
        nn = np.array([len(r[0]) for r in rules], dtype=np.int32)
        t = np.zeros((R, 64))
        wk = np.zeros((R, 64))
        wg = np.zeros((R, 64))
        for r, (tt, kk, gg) in enumerate(rules):
            t[r, :len(tt)], wk[r, :len(tt)], wg[r, :len(tt)] = tt, kk, gg
        _check(lib().tce_lg_set_rules(self.h, R, _i(nn), _d(t), _d(wk), _d(wg)), self.h)
        self.nrules = R

    def lg_rule_gmax(self) -> np.ndarray:
        g = np.zeros(self.nrules * 48, dtype=np.int32)
        _check(lib().tce_lg_rule_gmax(self.h, _i(g)), self.h)
        return g.reshape(self.nrules, 3, 16)

    def set_plain_rule(self, u, wk, wg, scale=0.6):
        u, wk, wg = (np.ascontiguousarray(x, dtype=np.float64) for x in (u, wk, wg))
        _check(lib().tce_set_plain_rule(self.h, len(u), _d(u), _d(wk), _d(wg), float(scale)), self.h)

    def lg_set_item_rules(self, rule: np.ndarray):
        r = np.ascontiguousarray(rule, dtype=np.int32)
        _check(lib().tce_lg_set_item_rules(self.h, _i(r)), self.h)

    def lg_item_rules(self) -> np.ndarray:
        r = np.zeros(self.info()["n_shell_quartets"], dtype=np.int32)
        _check(lib().tce_lg_item_rules(self.h, _i(r)), self.h)
        return r

    def lg_setup(self, n_train: int = 16000, seed: int = 2026, epochs: int = 80, label_tol: float = 3e-14):
        """The learned grid's whole set-up inside libtce (tce_lg_setup): dictionary,
        labels, training on the GPU, per-quartet rules."""
        _check(lib().tce_lg_setup(self.h, int(n_train), int(seed), int(epochs), float(label_tol), None), self.h)
        n = C.c_int32()
        _check(lib().tce_lg_dictionary(C.byref(n), None, None, None, None))
        self.nrules = n.value

    def lg_predict_rules(self, net, plain_factor: float = 10.0):
        _check(lib().tce_lg_predict_rules(self.h, net.h, float(plain_factor)), self.h)

    def lg_work(self):
        """(FP64 operations, primitive quartets) of the learned-grid pass."""
        f = C.c_double()
        n = C.c_int64()
        _check(lib().tce_lg_work(self.h, C.byref(f), C.byref(n)), self.h)
        return f.value, n.value

    def pass_kernels(self) -> int:
        """Kernels one J/K pass launches with the current method and work lists."""
        n = C.c_int32()
        _check(lib().tce_pass_kernels(self.h, C.byref(n)), self.h)
        return n.value

    def nuclear_attraction(self, geometry=None, charges=None) -> np.ndarray:
        """Nuclear attraction matrix (nbas x nbas) on the device (tce_nuclear_attraction);
        the system's own atoms by default."""
        geo = np.asfortranarray(self.sys.geometry if geometry is None else geometry, dtype=np.float64)
        Z = np.ascontiguousarray(self.sys.charges if charges is None else charges, dtype=np.int32)
        V = np.zeros(self.nbas * self.nbas)
        g = geo.ravel(order="F").copy()
        _check(lib().tce_nuclear_attraction(self.h, int(len(Z)), _d(g), _i(Z), _d(V)), self.h)
        return V.reshape(self.nbas, self.nbas, order="F")

    def lg_autotune(self, reps: int = 2) -> dict:
        """Time each learned-grid list with its CUDA-core and tensor-core kernels
        and keep the faster (tce_lg_autotune)."""
        nt, ns = C.c_int32(), C.c_int32()
        saved = C.c_double()
        _check(lib().tce_lg_autotune(self.h, int(reps), C.byref(nt), C.byref(ns), C.byref(saved)), self.h)
        return {"lists_tuned": nt.value, "lists_switched": ns.value, "ms_saved_per_pass": saved.value}

    def lg_lists(self) -> list:
        """The learned-grid work lists: dicts of kind, cls, nq, fp32, tc (kernel form in use), n."""
        n = C.c_int32(0)
        _check(lib().tce_lg_lists(self.h, C.byref(n), None), self.h)
        info = np.zeros(6 * max(n.value, 1), dtype=np.int32)
        _check(lib().tce_lg_lists(self.h, C.byref(n), _i(info)), self.h)
        keys = ("kind", "cls", "nq", "fp32", "tc", "n")
        return [dict(zip(keys, (int(x) for x in info[6 * i:6 * i + 6]))) for i in range(n.value)]

    def lg_list_profile(self, reps: int = 3) -> list:
        """Each learned-grid list launched alone (tce_lg_list_profile): the lists
        of lg_lists() with their fastest time (ms) and algorithmic FP64 operations."""
        n = C.c_int32(0)
        _check(lib().tce_lg_list_profile(self.h, int(reps), C.byref(n), None, None), self.h)
        ms = np.zeros(max(n.value, 1))
        fl = np.zeros(max(n.value, 1))
        _check(lib().tce_lg_list_profile(self.h, int(reps), C.byref(n), _d(ms), _d(fl)), self.h)
        out = self.lg_lists()
        for i, w in enumerate(out[:n.value]):
            w["ms"], w["flops"] = float(ms[i]), float(fl[i])
        return out[:n.value]

    def lg_set_list_form(self, i: int, form: int):
        """Kernel form of learned-grid list i by hand (tce_lg_set_list_form)."""
        _check(lib().tce_lg_set_list_form(self.h, int(i), int(form)), self.h)

    def set_tensor_cores(self, on: bool = True):
        """FP64 tensor-core node sums where a kernel has them (tce_set_tensor_cores)."""
        _check(lib().tce_set_tensor_cores(self.h, int(bool(on))), self.h)

    def set_list_streams(self, n: int = 2):
        """The learned-grid lists of a pass as n chains on their own streams (tce_set_list_streams)."""
        _check(lib().tce_set_list_streams(self.h, int(n)), self.h)

    def set_graph(self, on: bool = True):
        """Capture each J/K pass into a CUDA graph and replay it (tce_set_graph)."""
        _check(lib().tce_set_graph(self.h, int(bool(on))), self.h)

    def set_method(self, method: int):
        _check(lib().tce_set_method(self.h, int(method)), self.h)

    def set_tolerances(self, judge_tol=1e-10, plain_tol=1e-11, plain_max_panels=24):
        _check(lib().tce_set_tolerances(self.h, float(judge_tol), float(plain_tol), int(plain_max_panels)), self.h)

    def lg_stats(self) -> dict:
        st = np.zeros(5, dtype=np.int64)
        _check(lib().tce_lg_stats(self.h, st.ctypes.data_as(_lp)), self.h)
        return {"learned": int(st[0]), "rejected": int(st[1]), "plain_direct": int(st[2]),
                "plain_node_evals": int(st[3]), "fp32": int(st[4])}

    def set_fp32_threshold(self, thr: float = 1e-6):
        """FP32 node sums for learned-grid quartets with Schwarz product below thr (0: off)."""
        _check(lib().tce_set_fp32_threshold(self.h, float(thr)), self.h)

    def rule_blocks(self, rule: int, items: np.ndarray, mode: int = 1, judge: bool = False):
        """Blocks of the given shell quartets with one quadrature (rule >= 0 dictionary,
        -1 the system's rule, -2 the plain method); list of arrays (and Gauss estimates)."""
        items = np.ascontiguousarray(items, dtype=np.int32).reshape(-1, 4)
        sh = self.shells()
        sizes = [int(np.prod([sh[S][1] for S in q])) for q in items]
        tot = int(sum(sizes))
        K = np.zeros(max(tot, 1))
        G = np.zeros(max(tot, 1)) if (judge and rule >= 0) else None
        _check(lib().tce_rule_blocks(self.h, int(rule), int(mode), len(items), _i(items), _d(K),
                                     _d(G) if G is not None else None), self.h)
        offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        return K[:tot], (G[:tot] if G is not None else None), offs


def fast_quad_self_check(fast: Engine, full: Engine, tol: float = 1e-10):
    """fast_quad_self_check (fast_quad_self_check.f90:30-233), ERI part: the
    largest block difference between the fast-rule and full-table engines on the
    reference's sample, and whether the fast rule is kept (dmax <= tol)."""
    d = C.c_double()
    n = C.c_int32()
    _check(lib().tce_quad_self_check(fast.h, full.h, C.byref(d), C.byref(n)), fast.h)
    return d.value, n.value, d.value <= tol


def fast_quad_self_check_nuc(fast: Engine, full: Engine, tol: float = 1e-10):
    """The whole fast_quad_self_check (fast_quad_self_check.f90:30-233): ERI and
    nuclear-attraction samples on the fast-rule and full-table engines; returns
    (dmax, dV, n_eri, n_v, keep) with keep = dmax <= tol and dV <= tol."""
    geo = np.asfortranarray(fast.sys.geometry, dtype=np.float64).ravel(order="F").copy()
    Z = np.ascontiguousarray(fast.sys.charges, dtype=np.int32)
    d, dv = C.c_double(), C.c_double()
    nq, nv = C.c_int32(), C.c_int32()
    _check(lib().tce_quad_self_check_nuc(fast.h, full.h, int(len(Z)), _d(geo), _i(Z), C.byref(d), C.byref(dv),
                                         C.byref(nq), C.byref(nv)), fast.h)
    return d.value, dv.value, nq.value, nv.value, (d.value <= tol and dv.value <= tol)


def dfmp2_energy(ncl, L, eps_o, occ_o, eps_v, occ_v, mode: int = 1):
    """DF-MP2 contraction and energy on the device (tce_dfmp2_energy).

    L: complex array (no, nv, nau, N, N) = L(p, q, Q, k1, k2); eps_*/occ_*: (N, no) and (N, nv).
    Returns dict(e2d, e2x, emp2 = 2 e2d - e2x, nzero, gzero, ms)."""
    ncl = np.array([int(x) for x in ncl], dtype=np.int32)
    N = int(np.prod(ncl))
    no, nv, nau = L.shape[0], L.shape[1], L.shape[2]
    assert L.shape == (no, nv, nau, N, N)
    Lf = np.ascontiguousarray(np.asfortranarray(L, dtype=np.complex128).ravel(order="F")).view(np.float64).copy()
    crd = np.array([[k % ncl[0], (k // ncl[0]) % ncl[1], k // (ncl[0] * ncl[1])] for k in range(N)],
                   dtype=np.int32).ravel()
    eo = np.ascontiguousarray(eps_o, dtype=np.float64).ravel()
    ev = np.ascontiguousarray(eps_v, dtype=np.float64).ravel()
    oo = np.ascontiguousarray(occ_o, dtype=np.int32).ravel()
    ovv = np.ascontiguousarray(occ_v, dtype=np.int32).ravel()
    e2d, e2x, gz, ms = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    nz = C.c_int64()
    code = lib().tce_dfmp2_energy(N, _i(ncl), _i(crd), no, nv, nau, _d(Lf), _d(eo), _i(oo), _d(ev), _i(ovv),
                                  int(mode), C.byref(e2d), C.byref(e2x), C.byref(nz), C.byref(gz), C.byref(ms))
    if code != TCE_OK:
        raise TCEError(code, lib().tce_mp2_last_error().decode())
    return {"e2d": e2d.value, "e2x": e2x.value, "emp2": 2 * e2d.value - e2x.value, "nzero": nz.value,
            "gzero": gz.value, "ms": ms.value}


def hartree_exchange_potential(n1: int, P: np.ndarray, ERI: np.ndarray, physicist: bool = False):
    n = P.shape[0]
    Pf = np.asfortranarray(P, dtype=np.float64).ravel(order="F").copy()
    E = np.asfortranarray(ERI, dtype=np.float64).ravel(order="F").copy()
    J = np.zeros(n * n)
    K = np.zeros(n * n)
    _check(lib().tce_hartree_exchange(int(n1), int(n), int(physicist), _d(Pf), _d(E), _d(J), _d(K)))
    return J.reshape(n, n, order="F"), K.reshape(n, n, order="F")


def shard_plan(cost: np.ndarray, nranks: int) -> np.ndarray:
    """Cost-balanced owner of each work item (host-only, no GPU needed)."""
    c = np.ascontiguousarray(cost, dtype=np.float64)
    owner = np.zeros(len(c), dtype=np.int32)
    _check(lib().tce_shard_plan(_d(c), len(c), int(nranks), _i(owner)))
    return owner


def fp64_peak_tflops() -> float:
    """Measured FP64 FMA throughput of the current device (probe kernel)."""
    v = C.c_double()
    _check(lib().tce_fp64_peak(C.byref(v)))
    return v.value


def gk_rule(n: int):
    """(2n+1)-point Gauss-Kronrod rule on [0,1] built by libtce (host-only, no GPU
    needed): nodes, Kronrod weights, embedded Gauss weights."""
    u, wk, wg = (np.zeros(2 * n + 1) for _ in range(3))
    _check(lib().tce_gk_rule(int(n), _d(u), _d(wk), _d(wg)))
    return u, wk, wg


def lg_dictionary():
    """The rule dictionary libtce builds (tce_lg_dictionary): list of (t, wk, wg)."""
    n = C.c_int32()
    _check(lib().tce_lg_dictionary(C.byref(n), None, None, None, None))
    R = n.value
    nn = np.zeros(R, dtype=np.int32)
    t, wk, wg = (np.zeros(64 * R) for _ in range(3))
    _check(lib().tce_lg_dictionary(C.byref(n), _i(nn), _d(t), _d(wk), _d(wg)))
    return [(t[64 * r:64 * r + nn[r]], wk[64 * r:64 * r + nn[r]], wg[64 * r:64 * r + nn[r]]) for r in range(R)]
