"""The engine's multi-GPU shard path, on one GPU.

tce_set_shard(rank, nranks) keeps a cost-balanced share of the unique shell
quartets (tce_shard_plan over the engine's own cost array); the ranks' partial
J/K sum to the full J/K, which the caller all-reduces (one NCCL all-reduce of
2 nfuc nbas doubles per SCF iteration).  Here both shards run as two handles
on the same device, one after the other (no peer memory, no kernel waits on
another), with the learned grid, graphs and the judge's reject routing on:

* two passes each, so that the judge's rejects move to the plain list between
  them (the lists are rebuilt per shard, from the shard's own items);
* J0 + J1 and K0 + K1 equal the unsharded pass to 1e-12 of the density scale;
* the shards' quartets (tce_shard_items) partition the engine's list.
"""
import numpy as np
import pytest

from conftest import random_density

pytestmark = pytest.mark.gpu


def _sample(items, n, seed=0):
    rng = np.random.default_rng(seed)
    return items[rng.choice(len(items), min(n, len(items)), replace=False)]


def test_shards_sum_to_unsharded_pass(systems):
    from william_ci_b200 import learned_grid as LG
    from william_ci_b200.engine import TCE_METHOD_LEARNED, Engine
    sysm = systems("h_chain64", (16, 1, 1))
    P = random_density(sysm.nbas, seed=4)
    scale = np.abs(P).sum()
    full = Engine(sysm)
    LG.setup(full)
    ref = LG.ReferenceBlocks(sysm)
    net, _, _ = LG.train_rule_net(full, ref, _sample(full.items(), 4000), epochs=40, seed=0)
    full.lg_predict_rules(net)
    rules = full.lg_item_rules()
    items = full.items()
    full.set_method(TCE_METHOD_LEARNED)
    full.set_graph(True)
    for _ in range(2):
        J, K = full.direct_JK(P)
    parts, shard_items = [], []
    for rank in range(2):
        eng = Engine(sysm)
        LG.setup(eng)
        assert np.array_equal(eng.items(), items)        # same list, same order on every rank
        eng.lg_set_item_rules(rules)
        eng.set_shard(rank, 2)
        eng.set_method(TCE_METHOD_LEARNED)
        eng.set_graph(True)
        for _ in range(2):
            Jr, Kr = eng.direct_JK(P)
        parts.append((Jr, Kr))
        shard_items.append(eng.shard_items())
        info = eng.info()
        assert info["shard_rank"] == rank and info["shard_nranks"] == 2
        assert info["shard_shell_quartets"] == len(shard_items[-1])
        eng.close()
    Js = parts[0][0] + parts[1][0]
    Ks = parts[0][1] + parts[1][1]
    assert np.abs(Js - J).max() <= 1e-12 * scale
    assert np.abs(Ks - K).max() <= 1e-12 * scale
    # the shards partition the list
    both = np.concatenate(shard_items)
    assert len(both) == len(items)
    key = lambda a: np.sort(a.view([("", a.dtype)] * 4).ravel())
    assert np.array_equal(key(np.ascontiguousarray(both)), key(np.ascontiguousarray(items)))
    full.close()
    ref.close()
