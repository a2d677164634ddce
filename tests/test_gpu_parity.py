"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Tolerances: 1e-10 absolute per integral (shell blocks, stored ERIs, Schwarz
bounds); J and K, which are sums of ~1e5-1e6 integral x density products,
within 1e-9 absolute.
"""
import numpy as np
import pytest

from conftest import random_density

pytestmark = pytest.mark.gpu

TOL_INT = 1e-10
TOL_JK = 1e-9

CASES = [
    ("h2_ring", None),
    ("h_chain64", (8, 1, 1)),
    ("h2_sheet", (2, 2, 1)),
    ("li_cube", (2, 2, 2)),
]


def _engines(systems, name, ncell, **kw):
    import pyoracle
    from william_ci_b200.engine import Engine
    sysm = systems(name, ncell)
    return sysm, Engine(sysm, **kw), pyoracle.Oracle(sysm, **kw)


@pytest.mark.parametrize("name,ncell", CASES)
def test_schwarz_and_shells(systems, name, ncell):
    sysm, eng, orc = _engines(systems, name, ncell)
    sh_o, nshuc, ncap = orc.shells()
    assert eng.shells() == sh_o
    inf = eng.info()
    assert inf["nshuc"] == nshuc and inf["ncap"] == ncap
    np.testing.assert_allclose(eng.schwarz(), orc.schwarz(), rtol=0, atol=TOL_INT)
    ns, nf, npq = orc.count()
    assert inf["n_shell_quartets"] == ns
    assert inf["n_func_quartets"] == nf


@pytest.mark.parametrize("name,ncell", CASES)
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_shell_blocks(systems, name, ncell, mode):
    sysm, eng, orc = _engines(systems, name, ncell)
    sh, nshuc, _ = orc.shells()
    nsh = len(sh)
    rng = np.random.default_rng(7 + mode)
    quartets = [(0, 0, 0, 0), (0, min(1, nsh - 1), 0, min(1, nsh - 1))]
    for _ in range(12):
        q = [int(rng.integers(0, nshuc))] + [int(x) for x in rng.integers(0, nsh, 3)]
        quartets.append(tuple(q))
    for q in quartets:
        b_gpu = eng.ERI_shell_block(*q, mode=mode)
        b_orc = orc.shell_block(*q, mode=mode)
        assert b_gpu.shape == b_orc.shape
        np.testing.assert_allclose(b_gpu, b_orc, rtol=0, atol=TOL_INT, err_msg=str(q))


@pytest.mark.parametrize("name,ncell", CASES)
def test_direct_jk(systems, name, ncell):
    sysm, eng, orc = _engines(systems, name, ncell)
    P = random_density(sysm.nbas, seed=3)
    J, K = eng.direct_JK(P)
    Jo, Ko, _ = orc.direct_jk(P)
    np.testing.assert_allclose(J, Jo, rtol=0, atol=TOL_JK)
    np.testing.assert_allclose(K, Ko, rtol=0, atol=TOL_JK)
    assert np.all(J[sysm.nfuc:] == 0) and np.all(K[sysm.nfuc:] == 0)


@pytest.mark.parametrize("name,ncell", CASES[:3])
@pytest.mark.parametrize("physicist", [False, True])
def test_stored_eri_and_jk(systems, name, ncell, physicist):
    import pyoracle
    sysm, eng, orc = _engines(systems, name, ncell, physicist=physicist)
    E = eng.ERI_integral_toroidal()
    Eo, _ = orc.eri_stored()
    assert E.shape == Eo.shape
    np.testing.assert_allclose(E, Eo, rtol=0, atol=TOL_INT)
    P = random_density(sysm.nbas, seed=5)
    J, K = eng.stored_JK(P)
    Jo, Ko = pyoracle.hartree_exchange(sysm.nfuc, P, Eo, physicist=physicist)
    np.testing.assert_allclose(J, Jo, rtol=0, atol=TOL_JK)
    np.testing.assert_allclose(K, Ko, rtol=0, atol=TOL_JK)


def test_stored_nonsao_small(systems):
    sysm, eng, orc = _engines(systems, "h_chain64", (4, 1, 1), sao=False)
    E = eng.ERI_integral_toroidal()
    Eo, _ = orc.eri_stored()
    np.testing.assert_allclose(E, Eo, rtol=0, atol=TOL_INT)


def test_direct_jk_full_chain64(systems):
    """The 64-cell chain at full size (384 functions) against the oracle."""
    sysm, eng, orc = _engines(systems, "h_chain64", None)
    P = random_density(sysm.nbas, seed=11)
    J, K = eng.direct_JK(P)
    Jo, Ko, _ = orc.direct_jk(P)
    np.testing.assert_allclose(J, Jo, rtol=0, atol=TOL_JK)
    np.testing.assert_allclose(K, Ko, rtol=0, atol=TOL_JK)


def _lcg_sample(nshuc, nsh, nrand=50):
    """The self-check sample of fast_quad_self_check.f90:105-124 (0-based shells)."""
    seed = 12345
    out = [(i, i, i, i) for i in range(max(nshuc, 1))]
    for _ in range(nrand):
        q = []
        for m in (nshuc, nsh, nsh, nsh):
            seed = (seed * 1103515245 + 12345) % 2147483648
            q.append((seed // 16) % m)
        out.append(tuple(q))
    return out


def _lcg_v_sample(nshuc_first, nfuc, nbas, nrand=50, nv_rand=20):
    """The nuclear-attraction sample of fast_quad_self_check.f90:135-151 (0-based):
    the generator continues after the quartet sample's 4 nrand draws."""
    seed = 12345
    for _ in range(4 * nrand):
        seed = (seed * 1103515245 + 12345) % 2147483648
    out = [(f, f) for f in nshuc_first] or [(0, 0)]
    for r in range(2 * nv_rand):
        seed = (seed * 1103515245 + 12345) % 2147483648
        i = (seed // 16) % nfuc
        seed = (seed * 1103515245 + 12345) % 2147483648
        j = (seed // 16) % (nfuc if r < nv_rand else nbas)
        out.append((i, j))
    return out


@pytest.mark.parametrize("name,ncell", [("h_chain64", (8, 1, 1)), ("li_cube", (2, 2, 2))])
def test_fast_quad_self_check_nuclear_vs_oracle(systems, name, ncell):
    """Both halves of the gate: the ERI sample as in the test below, and the
    nuclear-attraction sample against the oracle's V with both rules."""
    import json
    import os
    import pyoracle
    from william_ci_b200.engine import Engine, fast_quad_self_check, fast_quad_self_check_nuc
    tab = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "quad_tables.json")))["128"]
    sysm = systems(name, ncell)
    fast = Engine(sysm)
    full = Engine(sysm, t_nodes=tab["t_val"], t_weights=tab["w_val"])
    d, dv, nq, nv, keep = fast_quad_self_check_nuc(fast, full)
    d0, nq0, _ = fast_quad_self_check(fast, full)
    assert d == d0 and nq == nq0
    o32 = pyoracle.Oracle(sysm)
    o128 = pyoracle.Oracle(sysm, t_nodes=tab["t_val"], t_weights=tab["w_val"])
    sh, _, _ = o32.shells()
    first = [f for f, _ in sh if f < sysm.nfuc]
    sample = _lcg_v_sample(first, sysm.nfuc, sysm.nbas)
    assert nv == len(sample)
    V32, V128 = o32.one_electron()[2], o128.one_electron()[2]
    dvref = max(abs(V32[i, j] - V128[i, j]) for i, j in sample)
    assert abs(dv - dvref) <= 1e-12, (dv, dvref)
    assert keep == (d <= 1e-10 and dvref <= 1e-10)


@pytest.mark.parametrize("name,ncell", [("h_chain64", (8, 1, 1)), ("li_cube", (2, 2, 2))])
def test_fast_quad_self_check_vs_oracle(systems, name, ncell):
    import json
    import os
    import pyoracle
    from william_ci_b200.engine import Engine, fast_quad_self_check
    tab = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "quad_tables.json")))["128"]
    sysm = systems(name, ncell)
    fast = Engine(sysm)
    full = Engine(sysm, t_nodes=tab["t_val"], t_weights=tab["w_val"])
    d, n, keep = fast_quad_self_check(fast, full)
    o32 = pyoracle.Oracle(sysm)
    o128 = pyoracle.Oracle(sysm, t_nodes=tab["t_val"], t_weights=tab["w_val"])
    sh, nshuc, _ = o32.shells()
    sample = _lcg_sample(nshuc, len(sh))
    assert n == len(sample)
    dref = max(np.abs(o32.shell_block(*q, mode=0) - o128.shell_block(*q, mode=0)).max() for q in sample)
    assert abs(d - dref) <= 1e-12, (d, dref)
    assert keep == (dref <= 1e-10)


def test_trexio_stream_from_the_device(systems):
    """tce_trexio_eri: the entry stream of the TREXIO export computed on the
    device from the full stored integrals equals the reference loop run on the
    same array (indices and values exactly), and the array equals the
    oracle's full integrals to 1e-10."""
    import pyoracle as po
    from william_ci_b200 import trexio_out as TX
    from william_ci_b200.engine import Engine
    sysm = systems("h_chain64", (4, 1, 1))
    with Engine(sysm, sao=False) as eng:
        E = eng.ERI_integral_toroidal()
        idx, val = eng.trexio_eri()
    ridx, rval = TX.reference_stream(E)
    assert np.array_equal(idx, ridx)
    assert np.array_equal(val, rval)
    Eo, _ = po.Oracle(sysm, sao=False).eri_stored()
    assert np.abs(E - Eo).max() < 1e-10
