"""Learned-grid t-quadrature: host side of the rule dictionary, the
rule-picking network and its training labels.

The t-integral of a shell quartet, (2/sqrt(pi)) int_0^inf f(t) dt, is
evaluated in the reference with one fixed rule per run (fast_quad or the
64/128-point tables, precompute_t.f90:5-14, 906-942).  Here each quartet gets
its own rule from a dictionary of mapped Gauss-Kronrod rules
(quadrature.rule_dictionary: orders K15/K21/K31 x scales 0.6 * 2^(j/2)):

* labels: for a sample of quartets, every dictionary rule's block is compared
  with a 128-node reference block; the label is the cheapest rule whose block
  is within LABEL_TOL of it, or PLAIN (= number of rules) when none is;
* the network (TCE_NFEAT -> 64 -> 64 -> rules, FP32) predicts for every rule
  the probability that the judge accepts it and its block is correct; it is
  trained on the GPU by libtce's own forward / backward / Adam kernels
  (RuleNet.train) against the per-rule targets of the labels;
* at set-up the engine computes every quartet's features, runs the network
  and picks the rule of least expected cost on the device
  (tce_lg_predict_rules); in the J/K pass the embedded Gauss estimate judges
  each block and rejects go to the plain adaptive method.

Nothing here evaluates integrals on the CPU: blocks, features, training and
prediction all run in libtce.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Tuple

import numpy as np

from . import quadrature as Q
from .engine import TCE_NFEAT, Engine, TCEError, _fp, _i, lib

# a rule is correct for a quartet when its block is within this of the reference
# block.  Measured on the 64-cell chain: 1e-11 -> 1e-12 -> 1e-13 -> 3e-14 gave
# held-out errors 2.6e-12 / 2.0e-13 / 3.1e-14 / 1.4e-14 at the same pass time
# (87.8-89.1 ms), so the tight bound costs nothing
LABEL_TOL = 3e-14
JUDGE_TOL = 1e-10      # the judge accepts a block whose error estimate (judge_estimate) is at most this
MARGIN = 2             # scales below a label that must be correct too
HIDDEN = 64


def dictionary():
    """The rule dictionary as (t, wk, wg) triples, with (scale, order) metadata."""
    rules, meta = [], []
    for s, n, t, wk, wg in Q.rule_dictionary():
        rules.append((t, wk, wg))
        meta.append((s, n))
    return rules, meta


def plain_rule() -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """15-point Kronrod rule on u in [0,1] with the embedded 7-point Gauss weights."""
    return Q.gauss_kronrod(7)


def reference_rule(n: int = 128, scale: float = 1.0):
    """Mapped Gauss-Legendre rule used for the label reference blocks."""
    return Q.mapped_gauss_legendre(n, scale)


class ReferenceBlocks:
    """Label reference: blocks with the 128-node mapped Gauss-Legendre rule,
    evaluated as the sum of two 64-node engines (a rule is a sum over its
    nodes), so that every angular-momentum class fits the 64-node kernel."""

    def __init__(self, system, **kw):
        t, w = reference_rule()
        self.engines = [Engine(system, t_nodes=t[i:i + 64], t_weights=w[i:i + 64], **kw) for i in (0, 64)]

    def rule_blocks(self, rule, items, mode=1, judge=False):
        assert rule == -1
        parts = [e.rule_blocks(-1, items, mode=mode) for e in self.engines]
        return parts[0][0] + parts[1][0], None, parts[0][2]

    def close(self):
        for e in self.engines:
            e.close()


class DictionaryReference:
    """The same label reference on the engine itself: the 128-node rule is
    loaded as a two-rule dictionary (its two halves of 64 nodes), both halves'
    blocks are summed, and the rule dictionary is loaded back.  No second
    handle is built, which matters for large systems (the 8x8 sheet's handle
    takes tens of seconds and gigabytes to build).  Per-item rules keep their
    indices: the dictionary put back is the same."""

    def __init__(self, engine: Engine):
        self.eng = engine

    def rule_blocks(self, rule, items, mode=1, judge=False):
        assert rule == -1
        t, w = reference_rule()
        z = np.zeros(64)
        self.eng.lg_set_rules([(t[:64], w[:64], z), (t[64:], w[64:], z)])
        try:
            K0, _, offs = self.eng.rule_blocks(0, items, mode=mode)
            K1, _, _ = self.eng.rule_blocks(1, items, mode=mode)
        finally:
            rules, _ = dictionary()
            self.eng.lg_set_rules(rules)
        return K0 + K1, None, offs

    def close(self):
        pass


def setup(engine: Engine, net: Optional["RuleNet"] = None):
    """Load the dictionary and the plain rule into an engine; predict rules with `net`."""
    rules, _ = dictionary()
    engine.lg_set_rules(rules)
    u, wk, wg = plain_rule()
    engine.set_plain_rule(u, wk, wg, 0.6)
    if net is not None:
        engine.lg_predict_rules(net)


def rule_costs(engine: Engine, nmax: np.ndarray) -> np.ndarray:
    """Work of each rule per quartet: sum over node groups of 8 nodes x (orders used),
    the orders capped by the quartet's truncation order nmax (items x rules)."""
    g = engine.lg_rule_gmax()[:, :engine.sys.ndp, :8]          # rules x ndp x 8 node groups
    n = np.asarray(nmax, dtype=np.int64)[:, None, None, None]
    used = np.where(g[None] >= 0, np.minimum(g[None], n) + 1, 0)
    return 8.0 * used.sum(axis=(2, 3))


def judge_estimate(K: np.ndarray, G: np.ndarray, offs: np.ndarray) -> np.ndarray:
    """Per-block error estimate of the device judge (block_judge): with
    e = max|K - G| and M = max|K| over the block, M min(1, (200 e / M)^1.5)."""
    seg = np.repeat(np.arange(len(offs) - 1), np.diff(offs))
    e = np.zeros(len(offs) - 1)
    M = np.zeros(len(offs) - 1)
    np.maximum.at(e, seg, np.abs(K - G))
    np.maximum.at(M, seg, np.abs(K))
    r = np.where(M > 0, 200.0 * e / np.where(M > 0, M, 1.0), 0.0)
    est = np.where(r >= 1.0, M, M * r * np.sqrt(r))
    return np.where((M > 0) & (e > 0), est, e)


def make_labels(engine: Engine, truth, items: np.ndarray, tol: float = LABEL_TOL,
                judge_tol: float = JUDGE_TOL, mode: int = 1, margin: int = MARGIN) -> Dict[str, np.ndarray]:
    """Features, per-rule errors / judge estimates and labels for the given
    quartets.  The label is the cheapest rule that the judge accepts, whose
    block is within `tol` of the reference block, and whose `margin` next
    smaller scales of the same order are within `tol` too (so that a
    prediction one or two scales too small still holds); PLAIN (= number of
    rules) if no rule is."""
    items = np.ascontiguousarray(items, dtype=np.int32).reshape(-1, 4)
    T, _, offs = truth.rule_blocks(-1, items, mode=mode)
    R = engine.nrules
    err = np.zeros((len(items), R))
    judge = np.zeros((len(items), R))
    kg = np.zeros((len(items), R))
    seg = np.repeat(np.arange(len(items)), np.diff(offs))
    for r in range(R):
        K, G, _ = engine.rule_blocks(r, items, mode=mode, judge=True)
        e = np.zeros(len(items))
        np.maximum.at(e, seg, np.abs(K - T))
        err[:, r] = e
        judge[:, r] = judge_estimate(K, G, offs)
        e = np.zeros(len(items))
        np.maximum.at(e, seg, np.abs(K - G))
        kg[:, r] = e
    M = np.zeros(len(items))
    np.maximum.at(M, seg, np.abs(T))
    X = engine.item_features(items)
    nmax = np.rint(np.expm1(X[:, 11].astype(np.float64))).astype(np.int64)
    cost = rule_costs(engine, nmax)
    good = err <= tol
    ok = good & (judge <= judge_tol)
    nS = len(Q.RULE_SCALES)
    if R == nS * len(Q.RULE_ORDERS):
        g3 = good.reshape(len(items), -1, nS)
        ok3 = ok.reshape(len(items), -1, nS).copy()
        for k in range(1, margin + 1):
            sh = np.zeros_like(g3)
            sh[:, :, k:] = g3[:, :, :-k]
            ok3 &= sh
        ok = ok3.reshape(len(items), R)
    masked = np.where(ok, cost, np.inf)
    y = np.where(ok.any(axis=1), masked.argmin(axis=1), R).astype(np.int32)
    return {"X": X, "y": y, "ok": ok.astype(np.float32), "err": err, "judge": judge, "kg": kg, "scale": M,
            "cost": cost, "items": items}


class RuleNet:
    """The rule-picking network, held on the device by libtce (tce_mlp_*)."""

    def __init__(self, nclass: int, nfeat: int = TCE_NFEAT, hidden: int = HIDDEN, seed: int = 0):
        h = C.c_void_p()
        code = lib().tce_mlp_create(int(nfeat), int(hidden), int(nclass), int(seed), C.byref(h))
        if code:
            raise TCEError(code, lib().tce_mlp_last_error(None).decode())
        self.h = h
        self.nf, self.nh, self.nc = nfeat, hidden, nclass
        n = C.c_int64()
        self._ck(lib().tce_mlp_nparams(self.h, C.byref(n)))
        self.nparams = n.value

    def _ck(self, code):
        if code:
            raise TCEError(code, lib().tce_mlp_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().tce_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        mu = np.zeros(self.nf, dtype=np.float32)
        sig = np.zeros(self.nf, dtype=np.float32)
        self._ck(lib().tce_mlp_get_params(self.h, p.ctypes.data_as(_fp), mu.ctypes.data_as(_fp),
                                          sig.ctypes.data_as(_fp)))
        return p, mu, sig

    def set_params(self, p=None, mu=None, sig=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float32) for a in (p, mu, sig)]
        ptrs = [None if a is None else a.ctypes.data_as(_fp) for a in arrs]
        self._ck(lib().tce_mlp_set_params(self.h, *ptrs))

    def loss_grad(self, X, Y):
        """Summed sigmoid cross-entropy (mean over rows) against targets Y and its gradient."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        loss = C.c_float()
        g = np.zeros(self.nparams, dtype=np.float32)
        self._ck(lib().tce_mlp_loss_grad(self.h, len(Y), X.ctypes.data_as(_fp), Y.ctypes.data_as(_fp),
                                         C.byref(loss), g.ctypes.data_as(_fp)))
        return loss.value, g

    def train(self, X, Y, epochs=40, batch=256, lr=3e-3, seed=0) -> float:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        loss = C.c_float()
        self._ck(lib().tce_mlp_train(self.h, len(Y), X.ctypes.data_as(_fp), Y.ctypes.data_as(_fp), int(epochs),
                                     int(batch), float(lr), int(seed), C.byref(loss)))
        return loss.value

    def predict(self, X) -> np.ndarray:
        """Probabilities (rows x outputs)."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros((len(X), self.nc), dtype=np.float32)
        self._ck(lib().tce_mlp_predict(self.h, len(X), X.ctypes.data_as(_fp), out.ctypes.data_as(_fp)))
        return out

    def save(self, path: str):
        p, mu, sig = self.params()
        np.savez(path, p=p, mu=mu, sig=sig, shape=np.array([self.nf, self.nh, self.nc]))

    @classmethod
    def load(cls, path: str) -> "RuleNet":
        z = np.load(path)
        nf, nh, nc = (int(x) for x in z["shape"])
        net = cls(nc, nf, nh)
        net.set_params(z["p"], z["mu"], z["sig"])
        return net


def train_rule_net(engine: Engine, truth: Engine, items: np.ndarray, epochs=60, batch=256, lr=3e-3,
                   seed=0) -> Tuple[RuleNet, Dict[str, np.ndarray], float]:
    """Labels for `items`, then a network trained on them on the GPU."""
    data = make_labels(engine, truth, items)
    net = RuleNet(engine.nrules, seed=seed)
    loss = net.train(data["X"], data["ok"], epochs=epochs, batch=batch, lr=lr, seed=seed)
    return net, data, loss

