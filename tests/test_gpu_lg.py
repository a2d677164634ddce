"""Learned-grid and plain-method quadrature on the device (through the C ABI).

* plain adaptive method vs the 128-node reference rule (blocks), 1e-11;
* the network's forward/backward kernels vs the numpy restatement
  (oracle/mlp_ref.py), FP32 tolerance;
* learned-grid J/K: rules picked by a network trained on the GPU; the blocks
  of the picked rules are within 1e-10 of the reference, J/K agree with the
  plain method's, the judge rejects few quartets, and the trained network
  beats the method without it (one fixed dictionary rule + judge);
* RHF energy with learned-grid J/K vs the oracle's, 1e-8 Eh.
"""
import numpy as np
import pytest

import mlp_ref
from conftest import make_system, random_density

pytestmark = pytest.mark.gpu

TOL_INT = 1e-10

CASES = [
    ("h_chain64", (8, 1, 1)),
    ("h2_sheet", (2, 2, 1)),
    ("li_cube", (2, 2, 2)),
]


def _lg_engine(sysm):
    from william_ci_b200 import learned_grid as LG
    from william_ci_b200.engine import Engine
    eng = Engine(sysm)
    LG.setup(eng)
    return eng


def _sample(items, n, seed=0):
    rng = np.random.default_rng(seed)
    return items[rng.choice(len(items), min(n, len(items)), replace=False)]


@pytest.mark.parametrize("name,ncell", CASES)
def test_plain_blocks_vs_reference(systems, name, ncell):
    from william_ci_b200 import learned_grid as LG
    sysm = systems(name, ncell)
    eng = _lg_engine(sysm)
    ref = LG.ReferenceBlocks(sysm)
    it = _sample(eng.items(), 400)
    P, _, offs = eng.rule_blocks(-2, it, mode=1)
    T, _, _ = ref.rule_blocks(-1, it, mode=1)
    assert np.abs(P - T).max() < 1e-11


def test_reference_blocks_split_equals_single_engine(systems):
    """The 128-node reference evaluated as two 64-node halves equals one 128-node engine."""
    from william_ci_b200 import learned_grid as LG
    from william_ci_b200.engine import Engine
    sysm = systems("h_chain64", (8, 1, 1))
    t, w = LG.reference_rule()
    one = Engine(sysm, t_nodes=t, t_weights=w)
    ref = LG.ReferenceBlocks(sysm)
    it = _sample(one.items(), 300)
    A, _, _ = one.rule_blocks(-1, it)
    B, _, _ = ref.rule_blocks(-1, it)
    assert np.abs(A - B).max() < 1e-13


def test_mlp_loss_grad_vs_oracle():
    from william_ci_b200 import learned_grid as LG
    rng = np.random.default_rng(3)
    nc = 9
    net = LG.RuleNet(nc, seed=5)
    p, _, _ = net.params()
    X = rng.standard_normal((257, 12)).astype(np.float32) * 3 + 1
    Y = (rng.random((257, nc)) < 0.4).astype(np.float32)
    mu = X.mean(0).astype(np.float32)
    sig = X.std(0).astype(np.float32)
    net.set_params(None, mu, sig)
    L, g = net.loss_grad(X, Y)
    Lr, gr = mlp_ref.loss_grad(p, mu, sig, X, Y, 12, 64, nc)
    assert abs(L - Lr) <= 1e-5 * abs(Lr)
    assert np.abs(g - gr).max() <= 1e-4 * np.abs(gr).max()
    pr = net.predict(X)
    np.testing.assert_allclose(pr, mlp_ref.predict(p, mu, sig, X, 12, 64, nc), atol=1e-5)


def test_mlp_training_fits_separable_targets():
    from william_ci_b200 import learned_grid as LG
    rng = np.random.default_rng(4)
    X = rng.standard_normal((4096, 12)).astype(np.float32)
    W = rng.standard_normal((12, 5))
    Y = (X @ W > 0).astype(np.float32)
    net = LG.RuleNet(5, seed=1)
    p0, _, _ = net.params()
    L0, _ = net.loss_grad(X, Y)
    L1 = net.train(X, Y, epochs=30, batch=128, lr=3e-3, seed=2)
    assert L1 < 0.2 * L0
    acc = ((net.predict(X) > 0.5) == (Y > 0.5)).mean()
    assert acc > 0.97


def _trained(eng, sysm, n_train=6000, seed=0):
    from william_ci_b200 import learned_grid as LG
    ref = LG.ReferenceBlocks(sysm)
    items = eng.items()
    tr = _sample(items, n_train, seed)
    net, data, _ = LG.train_rule_net(eng, ref, tr, epochs=60, seed=seed)
    return net, data, ref


@pytest.mark.parametrize("name,ncell", [("h_chain64", (16, 1, 1)), ("li_cube", (2, 2, 2))])
def test_learned_grid_jk(systems, name, ncell):
    from william_ci_b200 import learned_grid as LG
    from william_ci_b200.engine import TCE_METHOD_LEARNED, TCE_METHOD_PLAIN
    sysm = systems(name, ncell)
    eng = _lg_engine(sysm)
    net, data, ref = _trained(eng, sysm)
    eng.lg_predict_rules(net)
    rules = eng.lg_item_rules()
    items = eng.items()
    # blocks of the chosen rules on a held-out sample: within 1e-10 of the reference
    rng = np.random.default_rng(11)
    sel = rng.choice(len(items), min(1500, len(items)), replace=False)
    T, _, offs = ref.rule_blocks(-1, items[sel])
    worst = 0.0
    for r in np.unique(rules[sel]):
        m = np.nonzero(rules[sel] == r)[0]
        if r == eng.nrules:
            K, _, o2 = eng.rule_blocks(-2, items[sel][m])
        else:
            K, G, o2 = eng.rule_blocks(int(r), items[sel][m], judge=True)
            est = LG.judge_estimate(K, G, o2)
            m, K, o2 = _accepted(m, K, o2, est)
        for j, i in enumerate(m):
            worst = max(worst, np.abs(K[o2[j]:o2[j + 1]] - T[offs[i]:offs[i + 1]]).max(initial=0.0))
    assert worst <= TOL_INT
    # J/K: learned grid vs the plain method
    P = random_density(sysm.nbas, 1) * 0.05
    eng.set_method(TCE_METHOD_PLAIN)
    Jp, Kp = eng.direct_JK(P)
    eng.set_method(TCE_METHOD_LEARNED)
    Jl, Kl = eng.direct_JK(P)
    st = eng.lg_stats()
    assert st["learned"] + st["plain_direct"] == eng.info()["n_shell_quartets"]
    assert st["rejected"] <= 0.01 * max(st["learned"], 1)
    scale = np.abs(P).sum()
    assert np.abs(Jl - Jp).max() <= 1e-10 * scale
    assert np.abs(Kl - Kp).max() <= 1e-10 * scale


def _accepted(m, K, offs, est):
    """Keep the blocks the judge accepts (the others are re-evaluated by the plain method)."""
    keep = np.nonzero(est <= 1e-10)[0]
    Kk = np.concatenate([K[offs[j]:offs[j + 1]] for j in keep]) if len(keep) else np.zeros(0)
    o = np.concatenate([[0], np.cumsum(np.diff(offs)[keep])]).astype(np.int64)
    return m[keep], Kk, o


def test_network_gain_over_single_rule(systems):
    """What the trained network buys: the rules it picks cost less than the one
    dictionary rule that is acceptable for the most quartets (the method
    without the network), with few judge rejections."""
    from william_ci_b200 import learned_grid as LG
    sysm = systems("h_chain64", (16, 1, 1))
    eng = _lg_engine(sysm)
    net, data, ref = _trained(eng, sysm)
    items = eng.items()
    test = _sample(items, 3000, seed=9)
    d = LG.make_labels(eng, ref, test)
    eng.lg_predict_rules(net)
    rule_of = {tuple(q): r for q, r in zip(items, eng.lg_item_rules())}
    pr = np.array([rule_of[tuple(q)] for q in test])
    R = eng.nrules
    plain_cost = 10.0 * d["cost"].max(axis=1)
    lg = np.where(pr < R, d["cost"][np.arange(len(pr)), np.minimum(pr, R - 1)], plain_cost)
    rejected = (pr < R) & (d["judge"][np.arange(len(pr)), np.minimum(pr, R - 1)] > 1e-10)
    lg_total = (lg + rejected * plain_cost).sum()
    okfrac = data["ok"].mean(axis=0)
    best = int(np.argmax(okfrac - 1e-9 * data["cost"].mean(axis=0)))
    single = d["cost"][:, best] + (d["judge"][:, best] > 1e-10) * plain_cost
    assert rejected.mean() < 0.01
    assert lg_total < 0.9 * single.sum(), (lg_total, single.sum())


@pytest.mark.parametrize("which", ["dimer_chain", "h2_sheet_2x2"])
def test_rhf_energy_learned_grid_vs_oracle(which):
    import pyoracle as po  # noqa: F401
    from test_scf import dimer_chain, rhf_inputs
    from william_ci_b200 import scf
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    sysm = dimer_chain(8) if which == "dimer_chain" else make_system("h2_sheet", (2, 2, 1))
    o, St, Tt, Vt, en, nO = rhf_inputs(sysm)
    ref = scf.rhf_sao(St, Tt, Vt, en, nO, sysm.nfuc, sysm.ncell, lambda P: o.direct_jk(P)[:2])
    eng = _lg_engine(sysm)
    net, _, _ = _trained(eng, sysm, n_train=4000)
    eng.lg_predict_rules(net)
    eng.set_method(TCE_METHOD_LEARNED)
    dev = scf.rhf_sao(St, Tt, Vt, en, nO, sysm.nfuc, sysm.ncell, eng.direct_JK)
    assert ref.converged and dev.converged
    assert abs(dev.energy - ref.energy) < 1e-8, (dev.energy, ref.energy)


@pytest.fixture(scope="module")
def chain16_lg(systems):
    sysm = systems("h_chain64", (16, 1, 1))
    eng = _lg_engine(sysm)
    net, _, _ = _trained(eng, sysm)
    eng.lg_predict_rules(net)
    return sysm, eng, net


def test_graph_replay_matches_direct_launches(chain16_lg):
    from william_ci_b200.engine import TCE_METHOD_FIXED, TCE_METHOD_LEARNED
    sysm, eng, net = chain16_lg
    P = random_density(sysm.nbas, 3) * 0.05
    scale = np.abs(P).sum()
    for method in (TCE_METHOD_LEARNED, TCE_METHOD_FIXED):
        eng.set_graph(False)
        eng.set_method(method)
        J0, K0 = eng.direct_JK(P)
        eng.set_graph(True)
        J1, K1 = eng.direct_JK(P)          # captured
        J2, K2 = eng.direct_JK(0.5 * P)    # replayed with new data in the same buffers
        assert np.abs(J1 - J0).max() <= 1e-13 * scale and np.abs(K1 - K0).max() <= 1e-13 * scale
        assert np.abs(J2 - 0.5 * J0).max() <= 1e-13 * scale and np.abs(K2 - 0.5 * K0).max() <= 1e-13 * scale
    eng.set_graph(False)


def test_one_and_two_list_chains_give_the_same_jk(chain16_lg):
    """The learned-grid lists as one chain or as two chains on two streams
    (tce_set_list_streams), with and without the CUDA graph: J/K equal to
    1e-13 of the density scale (only the order of the atomic sums differs),
    and the judge rejects nothing more."""
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    sysm, eng, net = chain16_lg
    P = random_density(sysm.nbas, 7) * 0.05
    scale = np.abs(P).sum()
    eng.set_method(TCE_METHOD_LEARNED)
    eng.lg_predict_rules(net)
    eng.direct_JK(P)                     # the judge's rejects move to the plain list
    assert len(eng.lg_lists()) > 2
    eng.set_graph(False)
    eng.set_list_streams(1)
    J0, K0 = eng.direct_JK(P)
    for graph in (False, True):
        eng.set_graph(graph)
        eng.set_list_streams(2)
        for _ in range(2):               # captured, then replayed
            J, K = eng.direct_JK(P)
            assert eng.lg_stats()["rejected"] == 0
            assert np.abs(J - J0).max() <= 1e-13 * scale and np.abs(K - K0).max() <= 1e-13 * scale, graph
    eng.set_graph(False)
    from william_ci_b200.engine import TCEError
    with pytest.raises(TCEError):
        eng.set_list_streams(3)
    eng.set_list_streams(2)


def test_fp32_panels_error_vs_fp64(chain16_lg):
    """FP32 node sums for quartets with Schwarz product below 1e-6: the J/K
    difference from the all-FP64 pass stays below 1e-10 per unit density."""
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    sysm, eng, net = chain16_lg
    P = random_density(sysm.nbas, 4) * 0.05
    scale = np.abs(P).sum()
    eng.set_method(TCE_METHOD_LEARNED)
    eng.set_fp32_threshold(0.0)
    J0, K0 = eng.direct_JK(P)
    eng.set_fp32_threshold(1e-6)
    J1, K1 = eng.direct_JK(P)
    st = eng.lg_stats()
    eng.set_fp32_threshold(0.0)
    assert st["fp32"] > 0.2 * st["learned"]
    err = max(np.abs(J1 - J0).max(), np.abs(K1 - K0).max())
    assert err <= 1e-10 * scale, err


def test_graph_on_the_legacy_stream(chain16_lg):
    """tce_direct_jk_device on the legacy default stream with graphs on: the pass
    runs on the handle's stream, ordered with the caller's stream by events."""
    import torch
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    sysm, eng, net = chain16_lg
    n, nf = sysm.nbas, sysm.nfuc
    P = random_density(n, 5) * 0.05
    eng.set_method(TCE_METHOD_LEARNED)
    eng.set_graph(False)
    J0, K0 = eng.direct_JK(P)
    dP = torch.from_numpy(np.asfortranarray(P).ravel(order="F").copy()).cuda()
    dJ = torch.zeros(nf * n, dtype=torch.float64, device="cuda")
    dK = torch.zeros(nf * n, dtype=torch.float64, device="cuda")
    eng.set_graph(True)
    for _ in range(2):
        eng.direct_JK_device(dP.data_ptr(), dJ.data_ptr(), dK.data_ptr(), 0)
        J1 = dJ.view(n, nf).T.cpu().numpy()       # device J is nfuc x nbas, column-major
        K1 = dK.view(n, nf).T.cpu().numpy()
        scale = np.abs(P).sum()
        assert np.abs(J1 - J0[:nf]).max() <= 1e-13 * scale
        assert np.abs(K1 - K0[:nf]).max() <= 1e-13 * scale
    eng.set_graph(False)


def test_rejects_move_to_the_plain_list(chain16_lg):
    """The judge's rejects of one pass go to the plain list (side stream) from
    the next pass on: the judge then rejects nothing, the plain list grows by
    the reject count, the item rules report them as plain, and J/K stay the
    same (the same plain method evaluates those quartets in both passes)."""
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    sysm, eng, net = chain16_lg
    P = random_density(sysm.nbas, 6) * 0.05
    scale = np.abs(P).sum()
    eng.set_method(TCE_METHOD_LEARNED)
    eng.set_graph(False)
    eng.lg_predict_rules(net)                 # the network's rules again (earlier passes moved rejects)
    try:
        J1, K1 = eng.direct_JK(P)
        s1 = eng.lg_stats()
        plain1 = int(np.sum(eng.lg_item_rules() == eng.nrules))
        assert 0 < s1["rejected"] <= 4096, s1
        for graph in (False, True):
            eng.set_graph(graph)
            J2, K2 = eng.direct_JK(P)
            s2 = eng.lg_stats()
            assert s2["rejected"] == 0, s2
            assert s2["plain_direct"] == s1["plain_direct"] + s1["rejected"], (s1, s2)
            assert s2["learned"] == s1["learned"] - s1["rejected"]
            assert int(np.sum(eng.lg_item_rules() == eng.nrules)) == plain1 + s1["rejected"]
            assert np.abs(J2 - J1).max() <= 1e-13 * scale and np.abs(K2 - K1).max() <= 1e-13 * scale
            assert eng.pass_kernels() >= 2      # at least the plain list and the judge's fallback
    finally:
        eng.set_graph(False)


def test_tensor_core_node_sums_match_cuda_cores(chain16_lg):
    """All-s learned-grid quartets with the node sums on the FP64 tensor cores
    (mma.sync m8n8k4) against the FP64 CUDA-core kernel: same J/K up to the
    summation order."""
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    sysm, eng, net = chain16_lg
    P = random_density(sysm.nbas, 7) * 0.05
    scale = np.abs(P).sum()
    eng.set_method(TCE_METHOD_LEARNED)
    eng.set_fp32_threshold(0.0)
    eng.set_graph(False)
    try:
        out = {}
        for tc in (False, True):
            eng.set_tensor_cores(tc)
            for _ in range(2):                 # the second pass: the judge's rejects routed
                J, K = eng.direct_JK(P)
            out[tc] = (J, K, eng.lg_stats())
        assert out[False][2]["rejected"] == 0 and out[True][2]["rejected"] == 0
        for a, b in zip(out[False][:2], out[True][:2]):
            assert np.abs(a - b).max() <= 1e-12 * scale, np.abs(a - b).max() / scale
    finally:
        eng.set_tensor_cores(True)


def test_autotune_keeps_the_results(chain16_lg):
    """tce_lg_autotune times the CUDA-core and tensor-core form of every list
    that has both and keeps the faster: J/K unchanged up to the summation order,
    and the choice survives the rebuild that moves the judge's rejects."""
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    sysm, eng, net = chain16_lg
    P = random_density(sysm.nbas, 8) * 0.05
    scale = np.abs(P).sum()
    eng.set_method(TCE_METHOD_LEARNED)
    eng.set_fp32_threshold(0.0)
    eng.set_graph(False)
    eng.lg_predict_rules(net)
    J0, K0 = eng.direct_JK(P)
    info = eng.lg_autotune(reps=1)
    assert info["lists_tuned"] >= 1
    for graph in (False, True):          # the second call also rebuilds the lists (rejects moved)
        eng.set_graph(graph)
        J1, K1 = eng.direct_JK(P)
        assert np.abs(J1 - J0).max() <= 1e-12 * scale and np.abs(K1 - K0).max() <= 1e-12 * scale
    eng.set_graph(False)


def test_learned_grid_setup_from_the_c_abi(systems):
    """tce_lg_setup: the dictionary, labels, training and prediction inside
    libtce (the route of a Fortran caller): held-out blocks of the rules it sets
    within 1e-10 of the 128-node reference, J/K equal to the plain method's."""
    from william_ci_b200 import learned_grid as LG
    from william_ci_b200.engine import TCE_METHOD_LEARNED, TCE_METHOD_PLAIN, Engine
    sysm = systems("h_chain64", (16, 1, 1))
    eng = Engine(sysm)
    eng.lg_setup(n_train=4000, seed=7, epochs=60)
    rules = eng.lg_item_rules()
    items = eng.items()
    ref = LG.ReferenceBlocks(sysm)
    sel = np.random.default_rng(12).choice(len(items), 1500, replace=False)
    T, _, offs = ref.rule_blocks(-1, items[sel])
    worst = 0.0
    for r in np.unique(rules[sel]):
        m = np.nonzero(rules[sel] == r)[0]
        if r == eng.nrules:
            K, _, o2 = eng.rule_blocks(-2, items[sel][m])
        else:
            K, G, o2 = eng.rule_blocks(int(r), items[sel][m], judge=True)
            m, K, o2 = _accepted(m, K, o2, LG.judge_estimate(K, G, o2))
        for j, i in enumerate(m):
            worst = max(worst, np.abs(K[o2[j]:o2[j + 1]] - T[offs[i]:offs[i + 1]]).max(initial=0.0))
    assert worst <= TOL_INT
    P = random_density(sysm.nbas, 2) * 0.05
    eng.set_method(TCE_METHOD_PLAIN)
    Jp, Kp = eng.direct_JK(P)
    eng.set_method(TCE_METHOD_LEARNED)
    Jl, Kl = eng.direct_JK(P)
    scale = np.abs(P).sum()
    assert np.abs(Jl - Jp).max() <= 1e-10 * scale and np.abs(Kl - Kp).max() <= 1e-10 * scale
    ref.close()
    eng.close()


def test_every_all_s_tile_shape_gives_the_same_jk(chain16_lg):
    """The all-s tensor-core kernel in each tile shape the autotuner can pick
    (16 x 32, 32 x 16, 16 x 16, 8 x 64, 8 x 32 primitive quartets x nodes per
    pass),
    set by hand on every all-s list: J/K equal the CUDA-core kernel's to 1e-12
    of the density scale."""
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    sysm, eng, net = chain16_lg
    P = random_density(sysm.nbas, 9) * 0.05
    scale = np.abs(P).sum()
    eng.set_method(TCE_METHOD_LEARNED)
    eng.set_fp32_threshold(0.0)
    eng.set_graph(False)
    eng.lg_predict_rules(net)
    eng.direct_JK(P)                     # the judge's rejects move to the plain list
    lists = eng.lg_lists()
    alls = [i for i, w in enumerate(lists) if w["kind"] == 1]
    assert alls
    for i in alls:
        eng.lg_set_list_form(i, 0)
    J0, K0 = eng.direct_JK(P)
    for shape in (1, 2, 3, 4, 5):
        for i in alls:
            eng.lg_set_list_form(i, shape)
        J, K = eng.direct_JK(P)
        assert np.abs(J - J0).max() <= 1e-12 * scale and np.abs(K - K0).max() <= 1e-12 * scale, shape
    for i in alls:
        eng.lg_set_list_form(i, 1)


def test_every_one_p_tile_shape_gives_the_same_jk(chain16_lg):
    """The one-p tensor-core kernel (both power combinations per step loop,
    the real directions by moments) in each tile shape the autotuner can pick
    (8 x 32, 16 x 32 and, for 64-node rules, 8 x 64 primitive quartets x nodes
    per pass), set by hand on every one-p list: J/K equal the CUDA-core
    kernel's to 1e-12 of the density scale, with no more judge rejects."""
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    sysm, eng, net = chain16_lg
    P = random_density(sysm.nbas, 11) * 0.05
    scale = np.abs(P).sum()
    eng.set_method(TCE_METHOD_LEARNED)
    eng.set_fp32_threshold(0.0)
    eng.set_graph(False)
    eng.lg_predict_rules(net)
    eng.direct_JK(P)                     # the judge's rejects move to the plain list
    lists = eng.lg_lists()
    onep = [(i, w["nq"]) for i, w in enumerate(lists) if w["kind"] == 2]
    assert onep and {nq for _, nq in onep} == {32, 64}
    for i, _ in onep:
        eng.lg_set_list_form(i, 0)
    J0, K0 = eng.direct_JK(P)
    for shape in (1, 2, 3):
        for i, nq in onep:
            eng.lg_set_list_form(i, shape if shape <= (3 if nq == 64 else 2) else 1)
        J, K = eng.direct_JK(P)
        assert eng.lg_stats()["rejected"] == 0
        assert np.abs(J - J0).max() <= 1e-12 * scale and np.abs(K - K0).max() <= 1e-12 * scale, shape
    for i, _ in onep:
        eng.lg_set_list_form(i, 1)


@pytest.mark.parametrize("name,ncell", [("h2_sheet", (2, 2, 1)), ("li_cube", (2, 2, 2))])
def test_tensor_core_rows_in_2d_and_3d(systems, name, ncell):
    """The generic kernel's rows on the FP64 tensor cores for two and three
    periodic directions (one tile pass per direction), set by hand on every
    generic learned-grid list: J/K equal the CUDA-core rows' to 1e-12 of the
    density scale."""
    from william_ci_b200.engine import TCE_METHOD_LEARNED
    sysm = systems(name, ncell)
    eng = _lg_engine(sysm)
    net, _, _ = _trained(eng, sysm, n_train=3000)
    eng.lg_predict_rules(net)
    eng.set_method(TCE_METHOD_LEARNED)
    P = random_density(sysm.nbas, 10) * 0.05
    scale = np.abs(P).sum()
    eng.direct_JK(P)                     # the judge's rejects move to the plain list
    gen = [i for i, w in enumerate(eng.lg_lists()) if w["kind"] == 0]
    assert gen
    out = {}
    for form in (0, 1):
        for i in gen:
            eng.lg_set_list_form(i, form)
        out[form] = eng.direct_JK(P)
    for a, b in zip(out[0], out[1]):
        assert np.abs(a - b).max() <= 1e-12 * scale
    eng.close()
