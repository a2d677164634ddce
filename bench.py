#!/usr/bin/env python
"""Benchmark: toroidal ERI quartets/s of one integral-direct J/K build,
learned grid vs the plain adaptive method.

Workload (the Tori1D RHF H chain the metric is quoted on): 64 cells,
spacing 1.8 bohr, torus length 115.2 bohr, per H 3 contracted s (4 primitives,
exponents log-uniform in [0.1,20], seeded) + 1 p (0.727); 384 functions;
synthetic inputs (seeded), normalised as the Fortran caller would.

A step is one direct_JK pass (eri_direct.f90:262): every symmetry-unique shell
quartet evaluated and contracted with the density into J and K.  Unit of the
metric: function quartets (ij|kl) of the translation- and 8-fold-unique set
after the Schwarz screen, counted the same way for the CPU baseline.

The headline pass uses the learned grid: before timing, labels for a sample
of quartets are made against a 128-node reference rule and the rule-picking
network is trained on the GPU (reported as set-up time, not timed); each
quartet then gets one Gauss-Kronrod rule, the judge re-routes the quartets it
rejects to the plain method inside the same pass.  The plain adaptive method
and the reference's fixed 32-node rule are timed on the same device for
comparison, and the held-out error of each against the reference is reported.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N > 1) each rank evaluates a cost-balanced shard of the
quartets and the partial J/K are summed with one NCCL all-reduce per step.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "toroidal ERI quartets/s at ≤1e-10 err, learned-grid vs plain; RHF SCF iter time"
WORKLOAD = "h_chain64"
SYSTEM_FIXTURE = os.path.join(ROOT, "tests", "golden", "systems", WORKLOAD + ".npz")
ONEE_FIXTURE = os.path.join(ROOT, "tests", "golden", "systems", WORKLOAD + "_onee.npz")
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "jk_pass_learned_grid_h_chain64_traffic.json")
GOLD = os.path.join(ROOT, "tests", "golden")
# the 2D and 3D workloads at their named shapes: each timed on one cost-balanced
# shard of its quartet list (a full pass of the sheet takes over a minute)
NAMED = {"li_cube": {"shard": 256, "train": 6000,
                     "workload": "Tori3D Li cube, 4x4x4 cells, d=2.5, L=10 bohr, 3s+2p per Li, nbas=576"},
         "h2_sheet": {"shard": 1024, "train": 3000,
                      "workload": "Tori2D H2 sheet, 8x8 cells, d=2.0, L=16x16 bohr, 2s+1p+1d per H, nbas=1408"}}
L2_FLUSH_BYTES = 512 << 20
FP32_THRESHOLD = 1e-6        # Schwarz product below which the node sums run in FP32


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-pass", action="store_true",
                    help="for ncu --profile-from-start off: set the learned grid up (tce_lg_setup), run two warm "
                         "passes, then one pass between cudaProfilerStart and cudaProfilerStop, and exit")
    return ap.parse_args()


def density(n, seed=2026):
    rng = np.random.default_rng(seed)
    P = rng.standard_normal((n, n)) * 0.1
    return np.asfortranarray(P + P.T)


def config(sysm, extra=None):
    c = {"workload": "Tori1D H chain, 64 cells, d=1.8, L=115.2 bohr, 3s(4 prim)+1p per H, nbas=%d, one direct J/K pass"
                     % sysm.nbas,
         "nbas": sysm.nbas, "nfuc": sysm.nfuc, "quadrature": "32-node mapped Gauss-Legendre (fast_quad)",
         "l2": "flushed between timed steps (512 MiB write)"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# CPU baseline: the oracle port (C restatement of the reference, OpenMP)
# ---------------------------------------------------------------------------
def cpu_baseline(sysm, stride):
    """The oracle port on all host cores, two builds: the parity build (-O2,
    no fast-math, pair vectors recomputed) and the timing build with the
    reference's own compiler flags (-O3 -ffast-math -funroll-loops
    -march=native, built here for this host) and its pair-vector memo.  `value`
    is the faster one (the strongest CPU path available); each build's best of
    two passes over the sample (the second pass reads the memo)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    pyoracle.build_fast(force=True)
    P = density(sysm.nbas)
    res, items, nf = {}, None, 0
    for kind, fast, reps in (("parity_build", False, 1), ("timing_build", True, 2)):
        o = pyoracle.Oracle(sysm, fast=fast)
        if items is None:
            items = o.items()
        sample = items[::stride]
        best = None
        for _ in range(reps):
            t0 = time.perf_counter()
            _, _, nf = o.direct_jk_items(sample, P)
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        res[kind] = {"value": nf / best, "seconds": best}
        o.close()
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": res["timing_build"]["value"], "unit": "quartets/s", "cores": cores, "kind": "port",
            "sample": "direct_JK over every %d-th of the %d unique shell quartets (%d function quartets); C "
                      "restatement of the reference (no Fortran compiler here or on the GPU box), timing build: the "
                      "reference's flags -O3 -ffast-math -funroll-loops -march=native and its pair-vector memo"
                      % (stride, len(items), nf),
            "timing_build": res["timing_build"], "parity_build": res["parity_build"]}


def nuclear_attraction_stage(eng, sysm):
    """Nuclear attraction matrix on the device (tce_nuclear_attraction, every atom
    of the 64-cell chain): wall time of the call (host output), and its unit-cell
    rows against the oracle's committed rows."""
    z = np.load(ONEE_FIXTURE)
    eng.nuclear_attraction()
    t0 = time.perf_counter()
    V = eng.nuclear_attraction()
    t = time.perf_counter() - t0
    d = float(np.abs(V[:sysm.nfuc] - z["V"]).max())
    return V, {"ms": 1e3 * t, "elements": int(sysm.nfuc * sysm.nbas), "atoms": int(len(sysm.charges)),
               "max_abs_diff_vs_oracle_rows": d,
               "api": "tce_nuclear_attraction (rows of the unit cell on the device, the rest by translation, "
                      "host output)"}


def converged_scf(eng, sysm, V=None):
    """RHF to convergence (RHF_SAO mirror, thresh 1e-9: host linear algebra +
    device direct J/K through tce_direct_jk, one CUDA graph per pass) with the
    learned grid and with the fixed 32-node rule, each energy against the
    oracle's converged energy with the same quadrature (tests/golden/
    scf_h_chain64.json: the reference's 128-point table, and its 32-node rule);
    V of the 32-node rule from the device when given, V of the learned-grid
    SCF from a 128-node handle."""
    from william_ci_b200 import scf
    from william_ci_b200.engine import TCE_METHOD_FIXED, TCE_METHOD_LEARNED
    z = np.load(ONEE_FIXTURE)
    ref = json.load(open(os.path.join(GOLD, "scf_h_chain64.json")))
    S_, T_, V_ = (scf.fill_with_symmetry(z[k], sysm.nfuc, sysm.ncell) for k in ("S", "T", "V"))
    if V is not None:
        V_ = V
    # the nuclear attraction integrals use the t-quadrature too: the learned-grid
    # SCF takes V from a handle with the 128-node reference rule, as the oracle's
    # 128-table SCF takes it from that table
    from william_ci_b200 import learned_grid as LG
    from william_ci_b200.engine import Engine
    t128, w128 = LG.reference_rule()
    with Engine(sysm, t_nodes=t128, t_weights=w128) as e128:
        V128 = e128.nuclear_attraction()
    out, res = {}, None
    for key, method, truth, Vm in (("learned_grid", TCE_METHOD_LEARNED, "table_128", V128),
                                   ("fixed_32_node_rule", TCE_METHOD_FIXED, "fast_quad_32", V_)):
        args = (S_, T_, Vm, float(z["enuc"]), scf.n_occupied(sysm), sysm.nfuc, sysm.ncell)
        eng.set_method(method)
        r = scf.rhf_sao(*args, eng.direct_JK)
        it = r.iter_seconds[1:] if len(r.iter_seconds) > 1 else r.iter_seconds
        jk = r.jk_seconds[1:] if len(r.jk_seconds) > 1 else r.jk_seconds
        out[key] = {"energy": r.energy, "converged": bool(r.converged), "iterations": r.iterations,
                    "iter_ms": 1e3 * float(np.mean(it)), "jk_ms": 1e3 * float(np.mean(jk)),
                    "oracle_energy": ref[truth]["energy"], "abs_diff_vs_oracle": abs(r.energy - ref[truth]["energy"]),
                    "oracle_quadrature": truth}
        if method == TCE_METHOD_LEARNED:
            res = r
    eng.set_method(TCE_METHOD_LEARNED)
    out["oracle_32_vs_128_energy_diff"] = abs(ref["fast_quad_32"]["energy"] - ref["table_128"]["energy"])
    out["host"] = "numpy (SAO transforms, per-k eigh, DIIS)"
    return out, res


def ao_to_kmo_stage(eng, r):
    """(ov|ov) k-space MO integrals of the 64-cell chain (tce_ao_to_kmo) from the
    stored SAO integrals, with the SCF stage's orbitals: wall times of both."""
    from william_ci_b200 import df
    t0 = time.perf_counter()
    eri = eng.ERI_integral_toroidal()
    te = time.perf_counter()
    gb = eri.nbytes / 1e9
    del eri                                   # the host copy; the device keeps its own
    pr, qr = df.band_ranges(r.occ_k)
    eng.ao_to_kmo(r.C_k, pr, qr)              # warm-up (module load, first allocations)
    t1 = time.perf_counter()
    out = eng.ao_to_kmo(r.C_k, pr, qr)
    t2 = time.perf_counter()
    return {"stored_eri_s": te - t0, "stored_eri_gb": gb, "ao_to_kmo_s": t2 - t1, "shape": list(out.shape),
            "api": "tce_eri_stored then tce_ao_to_kmo (integrals resident on the device, host output)"}


def dfmp2_timing(n_scf=8):
    """DF-MP2 on the 128-cell chain (the DF-MP2 configuration: the 64-cell chain's
    cell and basis on 128 cells, even-tempered auxiliary 4s/2p/1d per H, ratio
    2.5 from 0.1): orbitals from n_scf RHF iterations (timing, not converged),
    then the C-ABI route a Fortran caller takes: tce_df_create (device
    integrals, per-k metric factorisation, df_B) and tce_dfmp2 (L vectors,
    (ov|ov) contraction and energy) in FP64 and in split-BF16 on the tensor
    cores; the density-fitted J/K of the SCF (tce_dfjk) from the handle's df_B
    and Bh."""
    from william_ci_b200 import df, scf
    from william_ci_b200.engine import Engine
    from william_ci_b200.system import AOSystem
    base = os.path.join(ROOT, "tests", "golden", "systems")
    ao = AOSystem.load(os.path.join(base, "h_chain128.npz"))
    aux = AOSystem.load(os.path.join(base, "h_chain128_aux.npz"))
    z = np.load(os.path.join(base, "h_chain128_onee.npz"))
    S_, T_, V_ = (scf.fill_with_symmetry(z[k], ao.nfuc, ao.ncell) for k in ("S", "T", "V"))
    t0 = time.perf_counter()
    with Engine(ao) as eng:
        r = scf.rhf_sao(S_, T_, V_, float(z["enuc"]), scf.n_occupied(ao), ao.nfuc, ao.ncell, eng.direct_JK,
                        max_scf=n_scf)
    t1 = time.perf_counter()
    dev = df.DeviceDF(ao, aux)
    t2 = time.perf_counter()
    e64 = dev.dfmp2(r.C_k, r.eps_k, r.occ_k, mode=0)           # first call: module load, allocations
    t3 = time.perf_counter()
    e64 = dev.dfmp2(r.C_k, r.eps_k, r.occ_k, mode=0)
    t4 = time.perf_counter()
    e16 = dev.dfmp2(r.C_k, r.eps_k, r.occ_k, mode=1)
    t5 = time.perf_counter()
    B, ndrop, Bh = dev.fitted(bh=True)
    dev.close()
    (p0, p1), (q0, q1) = df.band_ranges(r.occ_k)
    N, nau = int(np.prod(ao.ncell)), aux.nfuc
    # density-fitted J/K of the SCF (df_JK) on the device, with the last RHF density
    jk = df.DFJK(B, Bh, ao.ncell, ao.nfuc, nau)
    jk(r.P)
    tj = []
    for _ in range(5):
        t = time.perf_counter()
        jk(r.P)
        tj.append(time.perf_counter() - t)
    jk.close()
    return {"workload": "Tori1D H chain, 128 cells, L=230.4, nbas=768, aux 4s/2p/1d per H (naux %d), no=%d nv=%d"
                        % (N * nau, p1 - p0, q1 - q0),
            "rhf_iterations": r.iterations, "rhf_s": t1 - t0,
            "df_create_s": t2 - t1, "dfmp2_fp64_s": t4 - t3, "dfmp2_split_bf16_s": t5 - t4,
            "stage_s_excluding_rhf": (t2 - t1) + (t4 - t3),
            "metric_pivots_dropped": int(ndrop),
            "emp2_split_bf16": e16["emp2"], "emp2_fp64": e64["emp2"],
            "split_bf16_rel_err_vs_fp64": abs(e16["emp2"] - e64["emp2"]) / max(abs(e64["emp2"]), 1e-300),
            "df_jk_ms": 1e3 * float(np.median(tj)),
            "api": "tce_df_create (integrals, fitting, df_B on the device) + tce_dfmp2 (L vectors, contraction, "
                   "energy); tce_dfjk with the handle's df_B and Bh",
            "note": "orbitals of %d RHF iterations of a half-filled band (zero-gap terms left out as kMP2_calc does); "
                    "times the DF-MP2 stage, not a converged MP2 energy" % n_scf}


def reference_arm(args, sysm):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    pyoracle.build_fast(force=True)          # -march=native: compiled for this host
    o = pyoracle.Oracle(sysm, fast=True)
    items = o.items()
    stride = 8
    sample = items[::stride]
    P = density(sysm.nbas)
    for w in range(args.warmup):             # the first warm-up pass fills the pair-vector memo
        o.direct_jk_items(sample if w == 0 else sample[:max(1, len(sample) // 8)], P)
    tot, nf_tot = 0.0, 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, _, nf = o.direct_jk_items(sample, P)
        tot += time.perf_counter() - t0
        nf_tot += nf
    v = nf_tot / tot
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {"metric": METRIC, "value": v, "unit": "quartets/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "impl": "reference",
            "config": config(sysm, {"sample": "every %d-th unique shell quartet per step" % stride}),
            "cpu_baseline": {"value": v, "unit": "quartets/s", "cores": cores, "kind": "port",
                             "sample": "direct_JK over every %d-th of %d unique shell quartets per step; C restatement "
                                       "of the reference's OpenMP path (the Fortran reference cannot be compiled: no "
                                       "Fortran compiler), built with the reference's flags (-O3 -ffast-math "
                                       "-funroll-loops -march=native) and its pair-vector memo" % (stride, len(items))},
            "e2e": {"value": v, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# learned-grid set-up (untimed): labels on a sample, network trained on the GPU
# ---------------------------------------------------------------------------
def heldout(name):
    """Held-out quartets of a workload and the oracle's blocks of them with the
    reference's 128-point table (tests/golden/heldout_<name>.npz)."""
    z = np.load(os.path.join(GOLD, "heldout_%s.npz" % name))
    return z["items"], z["blocks"], z["offsets"]


def item_lookup(items, queries):
    """Positions of the query quartets in the engine's item list."""
    key = lambda a: ((a[:, 0].astype(np.int64) * 4096 + a[:, 1]) * 4096 + a[:, 2]) * 4096 + a[:, 3]
    ki = key(items)
    order = np.argsort(ki)
    pos = order[np.searchsorted(ki[order], key(queries))]
    assert np.array_equal(items[pos], queries)
    return pos


def training_sample(items, held, n, seed=2026):
    """n quartets drawn from the engine's list, none of them held out."""
    rng = np.random.default_rng(seed)
    cand = rng.choice(len(items), min(len(items), n + len(held) + 100), replace=False)
    hs = {tuple(q) for q in held}
    keep = [i for i in cand if tuple(items[i]) not in hs][:n]
    return items[np.array(keep)]


def pass_error(eng, items, rules, T, offs):
    """Largest difference from the truth blocks T of what a learned-grid pass
    computes for the given quartets: the rule's block where the judge accepts
    it, the plain method's block where the rule is plain or rejected."""
    from william_ci_b200 import learned_grid as LG
    worst, n_rej = 0.0, 0
    plain_idx = []
    for r in np.unique(rules):
        m = np.nonzero(rules == r)[0]
        if r >= eng.nrules:
            plain_idx.extend(m.tolist())
            continue
        K, G, o2 = eng.rule_blocks(int(r), items[m], judge=True)
        keep = LG.judge_estimate(K, G, o2) <= LG.JUDGE_TOL
        plain_idx.extend(m[~keep].tolist())
        n_rej += int((~keep).sum())
        for j in np.nonzero(keep)[0]:
            i = m[j]
            worst = max(worst, float(np.abs(K[o2[j]:o2[j + 1]] - T[offs[i]:offs[i + 1]]).max(initial=0.0)))
    if plain_idx:
        m = np.array(sorted(plain_idx))
        K, _, o2 = eng.rule_blocks(-2, items[m])
        for j, i in enumerate(m):
            worst = max(worst, float(np.abs(K[o2[j]:o2[j + 1]] - T[offs[i]:offs[i + 1]]).max(initial=0.0)))
    return worst, n_rej


def learned_grid_setup(eng, sysm, name, n_train=16000, seed=2026):
    """Labels for a training sample (against the 128-node reference rule on the
    engine itself), the network trained on the GPU, rules predicted for every
    quartet.  The held-out quartets (committed, every angular class) are not
    trained on; the blocks the pass computes for them are compared with the
    oracle's blocks under the reference's own 128-point table."""
    from william_ci_b200 import learned_grid as LG
    t0 = time.perf_counter()
    LG.setup(eng)
    items = eng.items()
    ho, T, offs = heldout(name)
    tr = training_sample(items, ho, n_train, seed)
    t1 = time.perf_counter()
    data = LG.make_labels(eng, LG.DictionaryReference(eng), tr)
    t2 = time.perf_counter()
    net = LG.RuleNet(eng.nrules, seed=0)
    loss = net.train(data["X"], data["ok"], epochs=80, batch=256, lr=2e-3, seed=0)
    t3 = time.perf_counter()
    eng.lg_predict_rules(net, 10.0)
    rules = eng.lg_item_rules()
    t4 = time.perf_counter()
    hr = rules[item_lookup(items, ho)]
    worst_lg, n_rej = pass_error(eng, ho, hr, T, offs)
    Pl, _, _ = eng.rule_blocks(-2, ho)
    Fx, _, _ = eng.rule_blocks(-1, ho)
    R = eng.nrules
    # the method without the network: the one dictionary rule that the most
    # training quartets accept (cheaper rule on ties), judged, rejects to plain
    okfrac = data["ok"].mean(axis=0)
    single = int(np.argmax(okfrac - 1e-9 * data["cost"].mean(axis=0)))
    return net, {"labels_s": t2 - t1, "train_s": t3 - t2, "predict_s": t4 - t3, "setup_total_s": t4 - t0,
                 "train_quartets": int(len(tr)), "rules": R, "train_loss": float(loss),
                 "on_learned_grid": int(np.sum(rules < R)), "plain_direct": int(np.sum(rules >= R)),
                 "heldout_judge_rejects": n_rej,
                 "max_err_vs_oracle_table128": {
                     "learned_grid": worst_lg, "plain": float(np.abs(Pl - T).max()),
                     "fixed_32_node_rule": float(np.abs(Fx - T).max()),
                     "sample": "%d held-out shell quartets (every angular class), oracle blocks with the reference's "
                               "128-point table (tests/golden/heldout_%s.npz)" % (len(ho), name)}}, \
        {"single_rule": single, "single_rule_ok_fraction": float(okfrac[single]), "rules": rules}


def function_quartets(Q, first, nsh, items, thr=1e-13):
    """Function quartets of the given shell quartets that pass the Schwarz
    screen Q(ij) Q(kl) >= thr (the unit of the metric), counted on the host."""
    tot = 0
    sizes = nsh[items]
    key = ((sizes[:, 0] * 7 + sizes[:, 1]) * 7 + sizes[:, 2]) * 7 + sizes[:, 3]
    for k in np.unique(key):
        grp = items[key == k]
        n = nsh[grp[0]]
        a = np.arange(n[0]); b = np.arange(n[1]); c = np.arange(n[2]); d = np.arange(n[3])
        for lo in range(0, len(grp), 20000):
            g = grp[lo:lo + 20000]
            fA, fB, fC, fD = (first[g[:, i]] for i in range(4))
            qb = Q[fA[:, None, None] + a[None, :, None], fB[:, None, None] + b[None, None, :]]
            qk = Q[fC[:, None, None] + c[None, :, None], fD[:, None, None] + d[None, None, :]]
            tot += int(np.count_nonzero(qb.reshape(len(g), -1, 1) * qk.reshape(len(g), 1, -1) >= thr))
    return tot


def named_shape_stage(name, flush, steps=5):
    """One of the 2D / 3D workloads at its named shape (the whole supercell in
    the handle): set-up, the learned grid trained on it, the held-out errors
    against the 128-table oracle, and the J/K pass timed on one cost-balanced
    shard of its quartet list with the learned grid, the fixed 32-node rule
    and the plain method (CUDA events on the handle's stream, L2 flushed
    between timed passes, one CUDA graph per pass)."""
    import torch
    from william_ci_b200.engine import TCE_METHOD_FIXED, TCE_METHOD_LEARNED, TCE_METHOD_PLAIN, Engine
    from william_ci_b200.system import AOSystem
    cfg = NAMED[name]
    sysm = AOSystem.load(os.path.join(GOLD, "systems", name + ".npz"))
    t0 = time.perf_counter()
    eng = Engine(sysm)
    create_s = time.perf_counter() - t0
    info = eng.info()
    _, lg, _ = learned_grid_setup(eng, sysm, name, n_train=cfg["train"])
    eng.set_shard(0, cfg["shard"])
    lg["autotune"] = eng.lg_autotune(2)           # CUDA-core or tensor-core rows per generic list
    sh = eng.shard_items()
    Q = eng.schwarz()
    first = np.array([f for f, _ in eng.shells()])
    nsh = np.array([n for _, n in eng.shells()])
    nfq = function_quartets(Q, first, nsh, sh)
    dev = torch.device("cuda", torch.cuda.current_device())
    n, nf = sysm.nbas, sysm.nfuc
    P = density(n)
    dP = torch.from_numpy(P.ravel(order="F").copy()).to(dev)
    dJ = torch.zeros(nf * n, dtype=torch.float64, device=dev)
    dK = torch.zeros(nf * n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    eng.set_graph(True)

    def timed(method, nsteps, warm):
        eng.set_method(method)
        for _ in range(warm):
            eng.direct_JK_device(dP.data_ptr(), dJ.data_ptr(), dK.data_ptr(), stream.cuda_stream)
            torch.cuda.synchronize()
        tot = 0.0
        for i in range(nsteps):
            flush.fill_(float(i))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.direct_JK_device(dP.data_ptr(), dJ.data_ptr(), dK.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / nsteps

    lg_ms = timed(TCE_METHOD_LEARNED, steps, 2)
    flops, nprim = eng.lg_work()
    fixed_ms = timed(TCE_METHOD_FIXED, steps, 1)
    plain_ms = timed(TCE_METHOD_PLAIN, 1, 1)
    eng.close()
    peak = _fp64_peak()
    return {"workload": cfg["workload"], "nbas": sysm.nbas, "create_s": create_s,
            "shell_quartets": info["n_shell_quartets"], "function_quartets": info["n_func_quartets"],
            "device_bytes": info["device_bytes"],
            "timed_shard": {"of": cfg["shard"], "shell_quartets": int(len(sh)), "function_quartets": nfq,
                            "plan": "cost-balanced shard 0 of %d (tce_set_shard)" % cfg["shard"]},
            "learned_grid": {"value": nfq / (lg_ms * 1e-3), "unit": "quartets/s", "ms_per_pass": lg_ms},
            "fixed_rule": {"value": nfq / (fixed_ms * 1e-3), "ms_per_pass": fixed_ms},
            "plain": {"value": nfq / (plain_ms * 1e-3), "ms_per_pass": plain_ms},
            "lg_over_plain": plain_ms / lg_ms,
            "roofline": {"bound": "fp64", "achieved": flops / (lg_ms * 1e-3) / 1e12, "peak": peak,
                         "unit": "TFLOP/s", "frac": flops / (lg_ms * 1e-3) / 1e12 / peak,
                         "algorithmic_flops_per_pass": flops, "primitive_quartets": nprim},
            "setup": lg}


_PEAK = []


def _fp64_peak():
    from william_ci_b200.engine import fp64_peak_tflops
    if not _PEAK:
        _PEAK.append(fp64_peak_tflops())
    return _PEAK[0]


def timed_passes(eng, step, steps, flush, stream, world, dist):
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    kern = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    for i in range(steps):
        flush.fill_(float(i))                     # evict L2 between timed steps (not timed)
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
        torch.cuda.synchronize()
        kern.append(eng.last_kernel_ms())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    return sum(a.elapsed_time(b) for a, b in ev), float(np.mean(kern))


def profile_pass(sysm):
    """One learned-grid pass of the workload inside cudaProfilerStart/Stop (the
    kernels of the pass as separate launches, no graph), after the set-up
    through the C ABI (tce_lg_setup), the kernel-form tuning and two warm
    passes (the judge's rejects moved to the plain list)."""
    import torch
    from william_ci_b200.engine import TCE_METHOD_LEARNED, Engine
    eng = Engine(sysm)
    eng.lg_setup(n_train=16000, seed=2026, epochs=80)
    eng.set_method(TCE_METHOD_LEARNED)
    eng.set_fp32_threshold(FP32_THRESHOLD)
    eng.lg_autotune(3)
    P = density(sysm.nbas)
    for _ in range(2):
        eng.direct_JK(P)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    eng.direct_JK(P)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profiled": "one learned-grid J/K pass", "kernels": eng.pass_kernels(),
                      "kernel_ms": eng.last_kernel_ms(), "stats": eng.lg_stats()}))
    eng.close()


def main():
    args = parse()
    from william_ci_b200.system import AOSystem
    sysm = AOSystem.load(SYSTEM_FIXTURE)
    if args.impl == "reference":
        reference_arm(args, sysm)
        return

    import torch
    import torch.distributed as dist
    from william_ci_b200.engine import TCE_METHOD_FIXED, TCE_METHOD_LEARNED, TCE_METHOD_PLAIN, Engine
    if args.profile_pass:
        profile_pass(sysm)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    eng = Engine(sysm)
    net, lg_info, lg_extra = learned_grid_setup(eng, sysm, WORKLOAD)
    if world > 1:
        eng.set_shard(rank, world)
    info = eng.info()
    n, nf = sysm.nbas, sysm.nfuc
    Ph = density(n)
    dP = torch.from_numpy(Ph.ravel(order="F").copy()).to(dev)
    dJ = torch.zeros(nf * n, dtype=torch.float64, device=dev)
    dK = torch.zeros(nf * n, dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step_on(e):
        def step():
            e.direct_JK_device(dP.data_ptr(), dJ.data_ptr(), dK.data_ptr(), stream.cuda_stream)
            if world > 1:
                dist.all_reduce(dJ)
                dist.all_reduce(dK)
        return step

    step = step_on(eng)

    def run(method, steps, warmup, e=None):
        e = eng if e is None else e
        st_ = step_on(e)
        e.set_method(method)
        for _ in range(warmup):      # synchronised: one-time list changes (rejects moved) finish here
            st_()
            torch.cuda.synchronize()
        tot, kern = timed_passes(e, st_, steps, flush, stream, world, dist)
        t = torch.tensor([tot, kern], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t[0]) / steps, float(t[1])

    nq_total = info["n_func_quartets"]
    # FP32 panels (Schwarz product < 1e-6): their J/K error against the all-FP64 pass
    eng.set_method(TCE_METHOD_LEARNED)
    J64, K64 = eng.direct_JK(Ph)
    eng.set_fp32_threshold(FP32_THRESHOLD)
    J32, K32 = eng.direct_JK(Ph)
    fp32 = {"threshold": FP32_THRESHOLD, "quartets": eng.lg_stats()["fp32"],
            "max_abs_jk_diff_vs_fp64": float(max(np.abs(J32 - J64).max(), np.abs(K32 - K64).max())),
            "density_abs_sum": float(np.abs(Ph).sum())}
    # kernel form (CUDA cores or FP64 tensor cores) per work list, chosen by timing both
    tune = eng.lg_autotune(3) if world == 1 else None
    if tune is not None:
        names = {0: "generic", 1: "all-s", 2: "one-p"}
        shapes = {1: {1: "16x32", 2: "32x16", 3: "16x16", 4: "8x64", 5: "8x32"}, 2: {1: "8x32", 2: "16x32", 3: "8x64"}}

        def form(w):
            if not w["tc"]:
                return "CUDA cores"
            return "tensor cores" + (" %s tiles per pass" % shapes[w["kind"]][w["tc"]] if w["kind"] in shapes else "")
        tune["lists"] = ["%s cls%d nq%d%s: %s, %d quartets" % (names[w["kind"]], w["cls"], w["nq"],
                                                                " fp32" if w["fp32"] else "", form(w), w["n"])
                         for w in eng.lg_lists()]
    # every pass is one CUDA-graph launch from here on
    eng.set_graph(True)
    # the headline: learned-grid J/K passes, clocks sampled during them
    clocks = ClockSampler(local)
    eng.set_method(TCE_METHOD_LEARNED)
    for _ in range(args.warmup):     # synchronised: one-time list changes (rejects moved) finish here
        step()
        torch.cuda.synchronize()
    clocks.start()
    tot_ms, lg_kern = timed_passes(eng, step, args.steps, flush, stream, world, dist)
    clk = clocks.stop()
    t = torch.tensor([tot_ms, lg_kern], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step, lg_kern = float(t[0]) / args.steps, float(t[1])
    value = nq_total / (ms_step * 1e-3)
    st = eng.lg_stats()
    # kernels of one learned-grid pass: one per work list (kernel class, rule size,
    # FP32 panels), the plain list on the side stream, the judge's fallback launch
    launches_per_step = eng.pass_kernels()
    # the lists as one chain on one stream against the default two chains (tce_set_list_streams):
    # what the overlap of one list's tail with the next list's start buys
    eng.set_list_streams(1)
    one_chain_ms, _ = run(TCE_METHOD_LEARNED, args.steps, args.warmup)
    eng.set_list_streams(2)
    # each work list's kernel alone: time and algorithmic work, for per-kernel fractions
    per_list = eng.lg_list_profile(3) if world == 1 else None
    # comparison arms on the same device: the plain adaptive method and the system's 32-node rule
    plain_steps = max(2, min(args.steps, 3))
    plain_ms, _ = run(TCE_METHOD_PLAIN, plain_steps, 1)
    fixed_ms, fixed_kern = run(TCE_METHOD_FIXED, args.steps, args.warmup)
    eng.set_fp32_threshold(0.0)
    lg64_ms, _ = run(TCE_METHOD_LEARNED, args.steps, args.warmup)
    eng.set_fp32_threshold(FP32_THRESHOLD)
    # the reference's own higher-accuracy setting (nquad_128: the 40-node mapped rule)
    ho, T_ho, offs_ho = heldout(WORKLOAD)
    eng40 = Engine(sysm, nquad=40)
    if world > 1:
        eng40.set_shard(rank, world)
    eng40.set_graph(True)
    r40_ms, _ = run(TCE_METHOD_FIXED, args.steps, args.warmup, e=eng40)
    B40, _, _ = eng40.rule_blocks(-1, ho)
    err40 = float(np.abs(B40 - T_ho).max())
    eng40.close()
    # the method without the network: one dictionary rule for every quartet, judged
    net_rules = eng.lg_item_rules()
    single = lg_extra["single_rule"]
    eng.lg_set_item_rules(np.full(len(net_rules), single, dtype=np.int32))
    single_ms, _ = run(TCE_METHOD_LEARNED, args.steps, args.warmup)
    single_err, single_rej = pass_error(eng, ho, np.full(len(ho), single), T_ho, offs_ho)
    single_plain = eng.lg_stats()["plain_direct"]
    eng.lg_set_item_rules(net_rules)
    # the reference's own rules on the learned grid's kernels (tensor cores, FP32 panels,
    # autotuned forms; the 40-node rule padded to 64 nodes): a one-rule dictionary whose Gauss
    # weights are its own weights, so that the judge accepts every block; the blocks are those
    # of the fixed_rule and rule_40_node arms
    from william_ci_b200 import learned_grid as LGm
    from william_ci_b200 import quadrature as Qm

    def reference_rule_on_tc(nodes):
        e = Engine(sysm)
        if world > 1:
            e.set_shard(rank, world)
        tr, wr = Qm.mapped_gauss_legendre(nodes)
        e.lg_set_rules([(tr, wr, wr)])
        e.set_plain_rule(*LGm.plain_rule(), 0.6)
        e.lg_set_item_rules(np.zeros(len(e.items()), dtype=np.int32))
        e.set_fp32_threshold(FP32_THRESHOLD)
        e.set_method(TCE_METHOD_LEARNED)
        if world == 1:
            e.lg_autotune(3)
        e.set_graph(True)
        ms, _ = run(TCE_METHOD_LEARNED, args.steps, args.warmup, e=e)
        B, _, _ = e.rule_blocks(0, ho)
        err = float(np.abs(B - T_ho).max())
        e.close()
        return ms, err

    r32tc_ms, err32tc = reference_rule_on_tc(32)
    r40tc_ms, err40tc = reference_rule_on_tc(40)
    eng.set_method(TCE_METHOD_LEARNED)
    for _ in range(2):               # back to the network's rules (their rejects already routed)
        step()
        torch.cuda.synchronize()

    # ---- end to end through the public API: pinned host P in, J/K out, every step;
    # L2 flushed before each step (outside the timed call), as for the device timing
    Pp = torch.from_numpy(Ph.ravel(order="F").copy()).pin_memory()
    Jp = torch.zeros(n * n, dtype=torch.float64).pin_memory()
    Kp = torch.zeros(n * n, dtype=torch.float64).pin_memory()
    e2e_steps = max(3, args.steps // 2)
    e2e_s = 0.0
    if world == 1:
        eng.direct_JK_ptrs(Pp.data_ptr(), Jp.data_ptr(), Kp.data_ptr())     # warm
        for i in range(e2e_steps):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.direct_JK_ptrs(Pp.data_ptr(), Jp.data_ptr(), Kp.data_ptr())
            e2e_s += time.perf_counter() - t0
        e2e_s /= e2e_steps
    else:
        for i in range(e2e_steps):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            dist.barrier()
            t0 = time.perf_counter()
            dP.copy_(Pp, non_blocking=True)
            step()
            Jp[: nf * n].copy_(dJ, non_blocking=True)
            Kp[: nf * n].copy_(dK, non_blocking=True)
            torch.cuda.synchronize()
            e2e_s += time.perf_counter() - t0
        e2e_s /= e2e_steps
        te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
        e2e_s = float(te[0])
    e2e = {"value": nq_total / e2e_s, "unit": "quartets/s", "h2d_bytes_per_step": 8 * n * n,
           "d2h_bytes_per_step": 2 * 8 * nf * n, "ms_per_step": 1e3 * e2e_s, "l2": "flushed before each step",
           "api": "tce_direct_jk, learned grid (host buffers, pinned)" if world == 1 else
                  "tce_direct_jk_device + NCCL all-reduce + pinned copies"}

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    peak = _fp64_peak()
    lg_flops, lg_nprim = eng.lg_work() if world == 1 else (None, None)
    achieved = lg_flops / (lg_kern * 1e-3) / 1e12 if world == 1 else None
    traffic = None
    if os.path.exists(PROFILE_TRAFFIC):
        try:
            traffic = json.load(open(PROFILE_TRAFFIC)).get("dram_bytes_per_pass")
        except Exception:
            traffic = None
    kernels = None
    if per_list:
        kernels = []
        for w in per_list:
            # kind 1 all-s, 2 one or two p shells (their CUDA-core forms: k_quartets_r1 for one
            # p shell, the generic kernel for two), 0 generic
            if w["kind"] == 0 or (w["kind"] == 2 and not w["tc"] and bin(w["cls"]).count("1") >= 2):
                nm = "k_quartets<%d>" % w["nq"]
            elif w["kind"] == 1:
                nm = "k_quartets_s%s<%d>" % ("_tc" if w["tc"] else "", w["nq"])
            else:
                nm = ("k_quartets_sp_tc<%d>" if w["tc"] else "k_quartets_r1<%d>") % w["nq"]
            if w["kind"] in (1, 2) and w["tc"]:
                nm += " tile shape %d" % w["tc"]
            kernels.append({"kernel": nm + (" fp32" if w["fp32"] else ""), "cls": w["cls"], "quartets": w["n"],
                            "ms": w["ms"], "flops": w["flops"],
                            "tflops": w["flops"] / (w["ms"] * 1e-3) / 1e12 if w["ms"] > 0 else None,
                            "frac": w["flops"] / (w["ms"] * 1e-3) / 1e12 / peak if w["ms"] > 0 else None})
    roofline = {"bound": "fp64", "kernel": "the learned-grid J/K pass, one CUDA graph: k_quartets<32|64>, "
                                           "k_quartets_s[_tc], k_quartets_sp_tc, k_quartets_r1 (per-quartet rule, judge, fused "
                                           "J/K scatter) and the plain launches",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if (achieved and peak) else None, "traffic": traffic,
                "peak_source": "measured FP64 FMA throughput of this GPU (tce_fp64_peak probe); MEASURED_PEAKS.json "
                               "holds no FP64 figure",
                "algorithmic_flops_per_launch": lg_flops, "primitive_quartets": lg_nprim, "pass_ms": lg_kern,
                "per_list": kernels}
    lg_err = lg_info["max_err_vs_oracle_table128"]
    line = {"metric": METRIC, "value": value, "unit": "quartets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded exponents/coefficients)",
            "config": config(sysm, {"parallelism": "quartet shards x%d + NCCL all-reduce of J/K" % world
                                    if world > 1 else "single GPU",
                                    "quadrature": "learned grid: per-quartet Gauss-Kronrod rule (K15..K61, 21 map "
                                                  "scales) picked by the network, judge <= 1e-10, plain fallback; "
                                                  "FP32 node sums below Schwarz 1e-6",
                                    "shell_quartets": info["n_shell_quartets"],
                                    "function_quartets": nq_total}),
            "plain": {"value": nq_total / (plain_ms * 1e-3), "ms_per_step": plain_ms, "steps": plain_steps,
                      "method": "device adaptive Gauss-Kronrod bisection (15/7 panels, Bessel columns per panel)"},
            "fixed_rule": {"value": nq_total / (fixed_ms * 1e-3), "ms_per_step": fixed_ms,
                           "max_err_vs_oracle_table128": lg_err["fixed_32_node_rule"],
                           "method": "the reference's default 32-node mapped Gauss-Legendre rule on the same engine"},
            "rule_40_node": {"value": nq_total / (r40_ms * 1e-3), "ms_per_step": r40_ms,
                             "max_err_vs_oracle_table128": err40,
                             "method": "the reference's nquad_128 setting: 40-node mapped Gauss-Legendre rule, same "
                                       "engine"},
            "single_rule_judged": {"value": nq_total / (single_ms * 1e-3), "ms_per_step": single_ms,
                                   "max_err_vs_oracle_table128": single_err, "rule": single,
                                   "train_accept_fraction": lg_extra["single_rule_ok_fraction"],
                                   "plain_list": single_plain, "heldout_judge_rejects": single_rej,
                                   "method": "the method without the network: the one dictionary rule most training "
                                             "quartets accept, for every quartet, judge and plain fallback"},
            "fixed_rule_tensor_cores": {"value": nq_total / (r32tc_ms * 1e-3), "ms_per_step": r32tc_ms,
                                        "max_err_vs_oracle_table128": err32tc,
                                        "method": "the reference's default 32-node rule on the learned grid's "
                                                  "kernels (FP64 tensor cores, FP32 panels, autotuned forms)"},
            "list_chains": {"two_chains_ms_per_step": ms_step, "one_chain_ms_per_step": one_chain_ms,
                            "note": "the learned-grid lists split into two cost-balanced chains on two streams "
                                    "(the default, the headline) or run one after another on one stream"},
            "rule_40_node_tensor_cores": {"value": nq_total / (r40tc_ms * 1e-3), "ms_per_step": r40tc_ms,
                                          "max_err_vs_oracle_table128": err40tc,
                                          "method": "the reference's nquad_128 setting (40-node rule, padded to 64 "
                                                    "nodes) on the learned grid's kernels"},
            "learned_grid_fp64_only": {"value": nq_total / (lg64_ms * 1e-3), "ms_per_step": lg64_ms},
            "fp32_panels": fp32,
            "cuda_graph": "each J/K pass replayed as one CUDA graph (tce_set_graph)",
            "autotune": tune,
            "learned_grid": dict(lg_info, judge_rejected_last_pass=st["rejected"],
                                 plain_list_last_pass=st["plain_direct"]),
            "e2e": e2e, "roofline": roofline, "clocks": clk, "gpu_launches": args.steps * launches_per_step}
    if world == 1:
        Vdev, line["nuclear_attraction"] = nuclear_attraction_stage(eng, sysm)
        line["rhf_scf"], r_scf = converged_scf(eng, sysm, V=Vdev)
        line["ao_to_kmo"] = ao_to_kmo_stage(eng, r_scf)
        eng.close()
        line["dfmp2"] = dfmp2_timing()
        line["named_shapes"] = {nm: named_shape_stage(nm, flush) for nm in NAMED}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sysm, stride=1)
    # the headline figures last (speed-ups, held-out errors, pass times, energies), so that a
    # reader of the end of the line has them
    summary = {"lg_over_plain": plain_ms / ms_step,
               "lg_over_rule_40_node": r40_ms / ms_step, "lg_over_single_rule_judged": single_ms / ms_step,
               "lg_over_fixed_rule_tensor_cores": r32tc_ms / ms_step,
               "lg_over_rule_40_node_tensor_cores": r40tc_ms / ms_step,
               "max_err_vs_oracle_table128": {"learned_grid": lg_err["learned_grid"], "rule_40_node": err40,
                                              "single_rule_judged": single_err,
                                              "fixed_32_node_rule": lg_err["fixed_32_node_rule"],
                                              "fixed_32_node_rule_tensor_cores": err32tc,
                                              "rule_40_node_tensor_cores": err40tc,
                                              "plain": lg_err["plain"]},
               "pass_ms": {"learned_grid": ms_step, "rule_40_node": r40_ms, "single_rule_judged": single_ms,
                           "learned_grid_one_chain": one_chain_ms,
                           "fixed_32_node_rule": fixed_ms, "fixed_32_node_rule_tensor_cores": r32tc_ms,
                           "rule_40_node_tensor_cores": r40tc_ms,
                           "plain": plain_ms}}
    if "rhf_scf" in line:
        summary["rhf_energy_abs_diff_vs_oracle"] = {k: line["rhf_scf"][k]["abs_diff_vs_oracle"]
                                                    for k in ("learned_grid", "fixed_32_node_rule")}
    if "named_shapes" in line:
        summary["named_shapes"] = {k: {"lg_quartets_per_s": v["learned_grid"]["value"],
                                       "lg_over_plain": v["lg_over_plain"],
                                       "lg_max_err_vs_oracle_table128":
                                           v["setup"]["max_err_vs_oracle_table128"]["learned_grid"],
                                       "roofline_frac": v["roofline"]["frac"]}
                                   for k, v in line["named_shapes"].items()}
    if "cpu_baseline" in line:
        summary["cpu_baseline_timing_build"] = line["cpu_baseline"]["value"]
    line["summary"] = summary
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
