"""Converged RHF energies of the 64-cell H chain with the oracle's J/K.

Writes tests/golden/scf_h_chain64.json: the RHF_SAO mirror
(william_ci_b200.scf.rhf_sao, RHF_SAO.f90:237-336, thresh 1e-9) run with the
CPU oracle's direct J/K (oracle/tce_oracle.c, direct_JK of
eri_direct.f90:262-374) under two t-rules:

* "fast_quad_32": the reference's default 32-node mapped Gauss-Legendre rule
  (precompute_t.f90:906-942), the rule of the device's fixed method;
* "table_128": the reference's own 128-point table (gauss_legendre_points,
  precompute_t.f90:484-895, from tests/golden/quad_tables.json), the
  converged quadrature the learned grid is held to.

The oracle takes minutes per SCF on a few cores, too slow for the GPU test
run, so the energies are committed.  Run from the repository root:

    python tests/golden/make_scf_fixtures.py [fast_quad_32|table_128 ...]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

OUT = os.path.join(HERE, "scf_h_chain64.json")


def run(rule):
    import pyoracle as po
    from conftest import make_system
    from william_ci_b200 import scf
    sysm = make_system("h_chain64")
    kw = {}
    if rule == "table_128":
        tab = json.load(open(os.path.join(HERE, "quad_tables.json")))["128"]
        kw = {"t_nodes": tab["t_val"], "t_weights": tab["w_val"]}
    o = po.Oracle(sysm, **kw)
    S, T, V = o.one_electron()
    en = po.nuclear_repulsion(sysm)
    t0 = time.time()
    r = scf.rhf_sao(S, T, V, en, scf.n_occupied(sysm), sysm.nfuc, sysm.ncell, lambda P: o.direct_jk(P)[:2])
    return {"energy": r.energy, "converged": bool(r.converged), "stalled": bool(r.stalled),
            "iterations": int(r.iterations), "seconds": time.time() - t0,
            "history": [{"iter": h["iter"], "E": h["E"], "conv": h["conv"]} for h in r.history]}


def main(rules):
    out = json.load(open(OUT)) if os.path.exists(OUT) else {}
    out["system"] = "tests/golden/systems/h_chain64.npz geometry and basis (workload h_chain64, seed 2026)"
    for rule in rules:
        out[rule] = run(rule)
        with open(OUT, "w") as f:
            json.dump(out, f, indent=1)
        print(rule, out[rule]["energy"], out[rule]["iterations"], flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["fast_quad_32", "table_128"])
