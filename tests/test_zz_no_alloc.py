"""tce_shell_block_noalloc against tce_shell_block.

The allocation-free entry point serves callers whose device memory is
reserved up front by their own pool allocator, so the library must not
cudaMalloc during the call; its scratch is a file-scope device array shared by
all calls.  Two calls in a row must each reproduce the allocating entry
point's block (the shared array keeps the previous call's contents, which
must not leak into the next result).  Runs alone in a fresh process or after
every other test; collected last so that a run stopping at the first failure
has run the rest already.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_INT = 1e-10


@pytest.mark.parametrize("name,ncell", [("h_chain64", (8, 1, 1)), ("h2_sheet", (2, 2, 1))])
def test_noalloc_block_matches_allocating_entry_point(systems, name, ncell):
    from william_ci_b200.engine import Engine
    sysm = systems(name, ncell)
    with Engine(sysm) as eng:
        sh = eng.shells()
        nshuc = eng.info()["nshuc"]
        rng = np.random.default_rng(42)
        # the largest block of the system first (d shells: 6^4 integrals), then random ones
        big = max(range(len(sh)), key=lambda s: sh[s][1])
        quartets = [(big % nshuc, big, big, big)]
        quartets += [tuple([int(rng.integers(0, nshuc))] + [int(x) for x in rng.integers(0, len(sh), 3)])
                     for _ in range(6)]
        for q in quartets:
            for mode in (0, 1, 2):
                ref = eng.ERI_shell_block(*q, mode=mode)
                first = eng.ERI_shell_block_noalloc(*q, mode=mode)
                second = eng.ERI_shell_block_noalloc(*q, mode=mode)
                np.testing.assert_allclose(first, ref, rtol=0, atol=TOL_INT, err_msg=str((q, mode)))
                np.testing.assert_allclose(second, ref, rtol=0, atol=TOL_INT, err_msg=str((q, mode)))
