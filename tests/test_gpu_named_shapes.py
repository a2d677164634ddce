"""The 2D and 3D workloads at their named shapes, against the oracle.

* h2_sheet: Tori2D, 8 x 8 cells, spacing 2.0, torus 16 x 16 bohr, two H per
  cell, 2 s + 1 p + 1 d shell per atom: 1408 functions, every class from
  (ss|ss) to (dd|dd) (src/calculation_type/Tori2D.f90; the two-periodic-
  direction branch of ERI_shell_block_toroidal.f90:268-296);
* li_cube: Tori3D, 4 x 4 x 4 cells, spacing 2.5, torus 10 bohr per axis, one
  Z = 3 atom per cell at a seeded offset, 3 s + 2 p shells: 576 functions
  (Tori3D.f90).

No shrunken geometry: the handles hold the whole supercell.  Checked:

* shell blocks of a seeded sample stratified over the angular classes (the
  committed held-out quartets: 2000 of the cube, 1200 of the sheet, every
  class present, (dd|dd) included) with the system's 32-node rule against the
  oracle's blocks of the same quartets, 1e-10;
* direct J/K of one cost-balanced shard of the quartet list (tce_set_shard; a
  full pass of the sheet takes over a minute on the device and hours on the
  oracle) against the oracle's direct_JK over the same quartets, 1e-9;
* the learned grid at size: a network trained on quartets outside the
  held-out sample; the blocks of the rules it picks (judged, rejects by the
  plain method) against the oracle's blocks with the reference's 128-point
  table (committed), 1e-10; and the learned-grid J/K of the shard against the
  128-table oracle's, 1e-9.
"""
import json
import os

import numpy as np
import pytest

import pyoracle as po
from conftest import ROOT, make_system, random_density

pytestmark = pytest.mark.gpu

GOLD = os.path.join(ROOT, "tests", "golden")
TOL_INT = 1e-10
SHARDS = {"li_cube": 512, "h2_sheet": 4096}
N_TRAIN = {"li_cube": 6000, "h2_sheet": 3000}


@pytest.fixture(scope="module", params=["li_cube", "h2_sheet"])
def named(request):
    from william_ci_b200.engine import Engine
    name = request.param
    sysm = make_system(name)
    eng = Engine(sysm)
    yield name, sysm, eng, np.load(os.path.join(GOLD, "heldout_%s.npz" % name))
    eng.close()


def _classes(sysm, eng, items):
    first = np.array([f for f, _ in eng.shells()])
    ls = sysm.lxyz[first].sum(axis=1)[items]
    return {tuple(int(x) for x in r) for r in ls}


def test_blocks_vs_oracle(named):
    name, sysm, eng, ho = named
    it = ho["items"]
    o = po.Oracle(sysm)
    B, offs = o.shell_blocks(it, mode=1)
    D, _, offs2 = eng.rule_blocks(-1, it, mode=1)
    assert np.array_equal(offs, offs2)
    assert np.abs(D - B).max() <= TOL_INT, np.abs(D - B).max()
    cls = _classes(sysm, eng, it)
    if name == "h2_sheet":
        assert (2, 2, 2, 2) in cls and (0, 0, 0, 0) in cls and len(cls) >= 30


def test_shard_jk_vs_oracle(named):
    from william_ci_b200.engine import TCE_METHOD_FIXED
    name, sysm, eng, ho = named
    eng.set_method(TCE_METHOD_FIXED)
    eng.set_shard(0, SHARDS[name])
    try:
        items = eng.shard_items()
        assert len(items) > 10000
        P = random_density(sysm.nbas, 5) * 0.05
        J, K = eng.direct_JK(P)
        Jo, Ko, nf = po.Oracle(sysm).direct_jk_items(items, P)
    finally:
        eng.set_shard(0, 1)
    d = max(np.abs(J - Jo).max(), np.abs(K - Ko).max())
    assert d <= 1e-9, d


def test_learned_grid_at_size_vs_oracle_table128(named):
    from william_ci_b200 import learned_grid as LG
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    name, sysm, eng, ho = named
    LG.setup(eng)
    items = eng.items()
    held = {tuple(q) for q in ho["items"]}
    rng = np.random.default_rng(2026)
    cand = items[rng.choice(len(items), N_TRAIN[name] + len(held) + 100, replace=False)]
    train = np.array([q for q in cand if tuple(q) not in held][:N_TRAIN[name]])
    net, _, _ = LG.train_rule_net(eng, LG.DictionaryReference(eng), train, epochs=60, seed=0)
    eng.lg_predict_rules(net)
    rules = eng.lg_item_rules()
    # held-out blocks of the picked rules against the 128-table oracle
    pos = {tuple(q): i for i, q in enumerate(items)} if len(items) < 3e7 else None
    it, T, offs = ho["items"], ho["blocks"], ho["offsets"]
    if pos is not None:
        hr = np.array([rules[pos[tuple(q)]] for q in it])
    else:                                   # 1e8 quartets: look the held-out ones up by sorting
        key = lambda a: ((a[:, 0].astype(np.int64) * 4096 + a[:, 1]) * 4096 + a[:, 2]) * 4096 + a[:, 3]
        ki, kh = key(items), key(it)
        order = np.argsort(ki)
        hr = rules[order[np.searchsorted(ki[order], kh)]]
    worst, n_rej = 0.0, 0
    for r in np.unique(hr):
        m = np.nonzero(hr == r)[0]
        if r == eng.nrules:
            K, _, o2 = eng.rule_blocks(-2, it[m])
            keep = np.ones(len(m), bool)
        else:
            K, G, o2 = eng.rule_blocks(int(r), it[m], judge=True)
            keep = LG.judge_estimate(K, G, o2) <= LG.JUDGE_TOL
            rej = m[~keep]
            n_rej += len(rej)
            if len(rej):
                Kp, _, op = eng.rule_blocks(-2, it[rej])
                for j, i in enumerate(rej):
                    worst = max(worst, float(np.abs(Kp[op[j]:op[j + 1]] - T[offs[i]:offs[i + 1]]).max()))
        for j in np.nonzero(keep)[0]:
            i = m[j]
            worst = max(worst, float(np.abs(K[o2[j]:o2[j + 1]] - T[offs[i]:offs[i + 1]]).max(initial=0.0)))
    assert worst <= TOL_INT, worst
    assert n_rej <= 0.02 * len(it), n_rej
    # learned-grid J/K of a shard against the 128-table oracle over the same quartets
    tab = json.load(open(os.path.join(GOLD, "quad_tables.json")))["128"]
    eng.set_method(TCE_METHOD_LEARNED)
    eng.set_shard(0, SHARDS[name])
    try:
        sh = eng.shard_items()
        P = random_density(sysm.nbas, 6) * 0.05
        for _ in range(2):                   # the second pass with the judge's rejects routed
            J, K = eng.direct_JK(P)
        o = po.Oracle(sysm, t_nodes=tab["t_val"], t_weights=tab["w_val"])
        Jo, Ko, _ = o.direct_jk_items(sh, P)
    finally:
        eng.set_shard(0, 1)
    d = max(np.abs(J - Jo).max(), np.abs(K - Ko).max())
    assert d <= 1e-9, d
