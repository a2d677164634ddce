"""J and K of the full 64-cell H chain from the oracle with the reference's
128-point t-table, the converged quadrature the learned grid is held to.

Writes tests/golden/jk_h_chain64_table128.npz: the density P (the SCF's
starting density, scf.core_guess_density: the core Hamiltonian of the oracle's
S, T, V occupied by guess_occupy_cut), and the unit-cell rows of J and K from
the oracle's direct_JK (oracle/tce_oracle.c; eri_direct.f90:262-374) with
t_val / w_val of gauss_legendre_points (precompute_t.f90:484-895, from
tests/golden/quad_tables.json).  The 128-node oracle pass takes minutes on a
few cores, so the result is committed.  Run from the repository root:

    python tests/golden/make_jk_fixtures.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

OUT = os.path.join(HERE, "jk_h_chain64_table128.npz")


def main():
    import pyoracle as po
    from conftest import make_system
    from william_ci_b200 import scf
    sysm = make_system("h_chain64")
    tab = json.load(open(os.path.join(HERE, "quad_tables.json")))["128"]
    o32 = po.Oracle(sysm)
    S, T, V = o32.one_electron()
    P = scf.core_guess_density(S, T, V, scf.n_occupied(sysm))
    o = po.Oracle(sysm, t_nodes=tab["t_val"], t_weights=tab["w_val"])
    t0 = time.time()
    J, K, nq = o.direct_jk(P)
    nf = sysm.nfuc
    np.savez(OUT, P=P, J=J[:nf], K=K[:nf], n_func_quartets=nq)
    print("wrote", OUT, "quartets", nq, "%.0f s" % (time.time() - t0))


if __name__ == "__main__":
    main()
