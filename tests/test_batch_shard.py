"""Host logic of the sharded batch (no GPU): the LPT assignment and the
gather of per-rank results with two gloo ranks on the CPU."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from amls_b200 import batch as B


def test_lpt_assignment_balances_and_covers():
    rng = np.random.default_rng(0)
    sizes = rng.integers(300, 6000, size=256)
    for ranks in (1, 2, 3, 8):
        parts = B.lpt_assign(sizes, ranks)
        assert sorted(i for p in parts for i in p) == list(range(256))
        loads = [float(np.sum(np.asarray(sizes)[p].astype(float) ** 3)) for p in parts]
        # LPT bound: max load <= 4/3 of the optimum, which is >= the mean
        assert max(loads) <= 4.0 / 3.0 * max(np.mean(loads), float(np.max(sizes)) ** 3) + 1.0
    assert B.lpt_assign([5, 5, 5], 2) == [[0, 2], [1]]


class _FakeSolver:
    """Stands in for the GPU solver: theta of pencil q is q + [0.1, 0.2]."""

    def solve_batch(self, Ks, Ms, opt):
        class S:
            pass
        out = []
        for K in Ks:
            s = S()
            s.theta = np.array([K + 0.1, K + 0.2])
            out.append(s)
        return out


class _P:
    def __init__(self, q, n):
        self.K = q
        self.M = q
        self.n = n


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ps = [_P(i, 100 + 37 * i % 900) for i in range(11)]
        got = B.solve_sharded(_FakeSolver(), ps, None, rank, world, dist)
        q.put((rank, None if got is None else [list(t) for t in got]))
    finally:
        dist.destroy_process_group()


def test_sharded_gather_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[1] is None
    assert res[0] == [[i + 0.1, i + 0.2] for i in range(11)]
