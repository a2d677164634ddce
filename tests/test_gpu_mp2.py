"""DF-MP2 contraction and energy on the device (tce_dfmp2_energy) against the
numpy restatement of df_kMO's (ov|ov) loop and kMP2_calc (oracle/mp2_ref.py).

FP64 contraction: 1e-12 relative.  Split-BF16 tensor-core contraction with
FP32 accumulation: its error against FP64 is stated here and must stay below
2e-5 relative in the correlation energy."""
import numpy as np
import pytest

import mp2_ref

pytestmark = pytest.mark.gpu


def _case(ncl, no, nv, nau, seed, degenerate=False):
    rng = np.random.default_rng(seed)
    N = int(np.prod(ncl))
    L = (rng.standard_normal((no, nv, nau, N, N)) + 1j * rng.standard_normal((no, nv, nau, N, N))) * 0.05
    eo = -0.5 - rng.random((N, no))
    ev = 0.2 + rng.random((N, nv))
    oo = np.full((N, no), 2, dtype=np.int32)
    ovv = np.zeros((N, nv), dtype=np.int32)
    if degenerate:                          # a zero-gap pair: e_a + e_b = e_i + e_j for some terms
        ev[0, 0] = eo[0, 0]
        ev[:, 0] = eo[0, 0]
        eo[:, 0] = eo[0, 0]
    oo[1, no - 1] = 0                       # a partly filled band: occupation 0 in the occupied range
    return L, eo, oo, ev, ovv


@pytest.mark.parametrize("ncl,no,nv,nau", [((4, 1, 1), 2, 4, 16), ((2, 2, 2), 1, 6, 16), ((3, 1, 1), 2, 3, 12)])
def test_dfmp2_energy_vs_oracle(ncl, no, nv, nau):
    from william_ci_b200.engine import dfmp2_energy
    L, eo, oo, ev, ovv = _case(ncl, no, nv, nau, seed=no * 7 + nv)
    G = mp2_ref.ovov(L, ncl)
    ref = mp2_ref.kmp2(G, ncl, eo, oo, ev, ovv)
    d64 = dfmp2_energy(ncl, L, eo, oo, ev, ovv, mode=0)
    assert abs(d64["emp2"] - ref["emp2"]) <= 1e-12 * abs(ref["emp2"])
    assert abs(d64["e2d"] - ref["e2d"]) <= 1e-12 * abs(ref["e2d"])
    assert d64["nzero"] == ref["nzero"]
    d16 = dfmp2_energy(ncl, L, eo, oo, ev, ovv, mode=1)
    rel = abs(d16["emp2"] - ref["emp2"]) / abs(ref["emp2"])
    print("split-BF16 relative error of E_MP2: %.2e" % rel)
    assert rel < 2e-5
    assert d16["nzero"] == ref["nzero"]


def test_dfmp2_zero_gap_terms_left_out():
    from william_ci_b200.engine import dfmp2_energy
    ncl = (4, 1, 1)
    L, eo, oo, ev, ovv = _case(ncl, 2, 3, 16, seed=5, degenerate=True)
    ref = mp2_ref.kmp2(mp2_ref.ovov(L, ncl), ncl, eo, oo, ev, ovv)
    d = dfmp2_energy(ncl, L, eo, oo, ev, ovv, mode=0)
    assert ref["nzero"] > 0 and d["nzero"] == ref["nzero"]
    assert abs(d["gzero"] - ref["gzero"]) <= 1e-12 * ref["gzero"]
    assert abs(d["emp2"] - ref["emp2"]) <= 1e-12 * abs(ref["emp2"])
