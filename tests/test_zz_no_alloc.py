"""tce_shell_block_noalloc against tce_shell_block.

The allocation-free entry point serves callers whose device memory is
reserved up front by their own pool allocator, so the library must not
cudaMalloc during the call; its scratch is a file-scope device array shared by
all calls.  Checked here:

* every block equals the allocating entry point's block, on two calls in a row;
* the shared array keeps the previous call's contents, so a large (dd|dd)
  block alternates with smaller blocks: a stale tail of the large block must
  not leak into a later, smaller result;
* the calls allocate nothing: after one warm-up call the device's free memory
  (cudaMemGetInfo) and the handle's own device bytes stay the same across all
  of the allocation-free calls.

Runs alone in a fresh process or after every other test; collected last so
that a run stopping at the first failure has run the rest already.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_INT = 1e-10


def _free_bytes():
    import torch
    free, _ = torch.cuda.mem_get_info(0)
    return free


@pytest.mark.parametrize("name,ncell", [("h_chain64", (8, 1, 1)), ("h2_sheet", (2, 2, 1))])
def test_noalloc_block_matches_allocating_entry_point(systems, name, ncell):
    from william_ci_b200.engine import Engine
    sysm = systems(name, ncell)
    with Engine(sysm) as eng:
        sh = eng.shells()
        nshuc = eng.info()["nshuc"]
        rng = np.random.default_rng(42)
        # the largest block of the system (d shells: 6^4 integrals) alternating
        # with random, mostly smaller ones
        big = max(range(len(sh)), key=lambda s: sh[s][1])
        big_q = (big % nshuc, big, big, big)
        small = [tuple([int(rng.integers(0, nshuc))] + [int(x) for x in rng.integers(0, len(sh), 3)])
                 for _ in range(6)]
        quartets = []
        for q in small:
            quartets += [big_q, q]
        refs = {(q, mode): eng.ERI_shell_block(*q, mode=mode) for q in set(quartets) for mode in (0, 1, 2)}
        # warm-up: the first call on the device may still touch lazily loaded state
        eng.ERI_shell_block_noalloc(*big_q, mode=1)
        free0 = _free_bytes()
        dev0 = eng.info()["device_bytes"]
        for q in quartets:
            for mode in (0, 1, 2):
                first = eng.ERI_shell_block_noalloc(*q, mode=mode)
                second = eng.ERI_shell_block_noalloc(*q, mode=mode)
                ref = refs[(q, mode)]
                np.testing.assert_allclose(first, ref, rtol=0, atol=TOL_INT, err_msg=str((q, mode)))
                np.testing.assert_allclose(second, ref, rtol=0, atol=TOL_INT, err_msg=str((q, mode)))
        assert _free_bytes() == free0, "device free memory changed across allocation-free calls"
        assert eng.info()["device_bytes"] == dev0, "handle allocated device memory during allocation-free calls"
