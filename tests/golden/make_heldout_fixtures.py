"""Held-out shell-quartet samples of the named workloads, with the oracle's
blocks under the reference's 128-point t-table.

For each workload at its named shape (h_chain64: Tori1D 64 cells; li_cube:
Tori3D 4x4x4; h2_sheet: Tori2D 8x8) a seeded sample of the unique shell
quartets (the oracle's orbit-minimum enumeration, ERI_toroidal.f90:342-401),
stratified over the angular-momentum classes (lA, lB | lC, lD) so that every
class is present, (dd|dd) included, and the oracle's blocks of those quartets
(ERI_shell_block_toroidal.f90:28-366 with the primitive screen, mode 1) with
t_val / w_val of gauss_legendre_points (precompute_t.f90:484-895, from
tests/golden/quad_tables.json).  The blocks are the converged reference that
the learned grid's blocks are measured against; the quartets are held out of
its training.  Writes tests/golden/heldout_<workload>.npz (items, blocks,
offsets).  Run from the repository root:

    python tests/golden/make_heldout_fixtures.py [workload ...]
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

SAMPLES = {"h_chain64": 2000, "li_cube": 2000, "h2_sheet": 1200}
SEED = 7


def stratified(classes, n, rng):
    """About n indices, every class represented: classes share n evenly, the
    share a small class cannot use going to the others."""
    keys, counts = np.unique(classes, return_counts=True)
    quota = np.zeros(len(keys), dtype=np.int64)
    left, open_ = n, np.ones(len(keys), bool)
    while left > 0 and open_.any():
        share = max(1, left // int(open_.sum()))
        for i in np.nonzero(open_)[0]:
            take = min(share, counts[i] - quota[i], left)
            quota[i] += take
            left -= take
            if quota[i] == counts[i]:
                open_[i] = False
            if left == 0:
                break
    out = []
    for k, q in zip(keys, quota):
        idx = np.nonzero(classes == k)[0]
        out.append(rng.choice(idx, int(q), replace=False))
    return np.sort(np.concatenate(out))


def shell_l(o, sysm):
    sh, _, _ = o.shells()
    return np.array([int(sysm.lxyz[f].sum()) for f, _ in sh], dtype=np.int64)


def main(names):
    import pyoracle as po
    from conftest import make_system
    tab = json.load(open(os.path.join(HERE, "quad_tables.json")))["128"]
    for name in names:
        t0 = time.time()
        sysm = make_system(name)
        o = po.Oracle(sysm, t_nodes=tab["t_val"], t_weights=tab["w_val"])
        items = o.items()
        ls = shell_l(o, sysm)[items]
        cls = ((ls[:, 0] * 3 + ls[:, 1]) * 3 + ls[:, 2]) * 3 + ls[:, 3]
        sel = items[stratified(cls, SAMPLES[name], np.random.default_rng(SEED))]
        del items
        B, offs = o.shell_blocks(sel, mode=1)
        out = os.path.join(HERE, "heldout_%s.npz" % name)
        np.savez_compressed(out, items=sel.astype(np.int32), blocks=B, offsets=offs)
        print(name, len(sel), "quartets", len(np.unique(cls)), "classes", B.size, "doubles", "%.0f s" % (time.time() - t0),
              flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or list(SAMPLES))
