"""Multi-rank J/K (CPU, gloo, world size 2): the quartet list is split with the
library's cost-balanced planner (tce_shard_plan, host-only), each rank builds
partial J/K from its shard (oracle as the stand-in for the device kernel), and
one all-reduce of J and K reproduces the single-rank result.  This is the
exchange step of the multi-GPU path (bench.py under torchrun uses NCCL)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    sys.path.insert(0, os.path.dirname(here))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import pyoracle
        from conftest import make_system, random_density
        from william_ci_b200.engine import shard_plan
        sysm = make_system("h_chain64", (6, 1, 1))
        o = pyoracle.Oracle(sysm)
        items = o.items()
        # cost proxy: primitive quartets of the item (same for every rank)
        npr = np.diff(sysm.prim_off)
        sh, _, _ = o.shells()
        first = np.array([f for f, _ in sh])
        cost = np.prod(npr[first[items]], axis=1).astype(np.float64)
        owner = shard_plan(cost, world)
        mine = items[owner == rank]
        P = random_density(sysm.nbas, seed=9)
        J, K, nf = o.direct_jk_items(mine, P)
        tJ, tK = torch.from_numpy(J.copy()), torch.from_numpy(K.copy())
        dist.all_reduce(tJ)
        dist.all_reduce(tK)
        cnt = torch.tensor([float(len(mine)), float(nf)], dtype=torch.float64)
        dist.all_reduce(cnt)
        if rank == 0:
            Jf, Kf, _ = o.direct_jk(P)
            out.put((float(np.abs(tJ.numpy() - Jf).max()), float(np.abs(tK.numpy() - Kf).max()),
                     int(cnt[0]), len(items), int(cnt[1]), o.count()[1]))
    finally:
        dist.destroy_process_group()


def test_sharded_jk_allreduce_equals_full():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    dJ, dK, n_items_sum, n_items, nf_sum, nf = res
    assert n_items_sum == n_items          # every quartet on exactly one rank
    assert nf_sum == nf
    assert dJ < 1e-12 and dK < 1e-12


def test_shard_plan_balances():
    from william_ci_b200.engine import shard_plan
    rng = np.random.default_rng(0)
    cost = np.sort(rng.exponential(size=5000))[::-1]
    for n in (2, 3, 8):
        owner = shard_plan(cost, n)
        loads = np.array([cost[owner == r].sum() for r in range(n)])
        assert set(owner.tolist()) == set(range(n))
        assert loads.max() / loads.mean() < 1.01
