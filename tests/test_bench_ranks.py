"""The multi-rank path of bench.py on the host: two gloo ranks on 127.0.0.1.

With N GPUs the bench runs N independent replicas of the solve (the
single-pencil path does not shard) and reports every time as the slowest
rank's; the reference arm runs on rank 0 alone.  Both rules are host logic,
checked here without a GPU.
"""
import argparse
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        got = [bench.max_over_ranks(v, dist) for v in values[rank]]
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    values = [[0.5, 3.0, 2.0], [1.5, 1.0, 2.0]]    # per rank, three reductions
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, values, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1] == [1.5, 3.0, 2.0]


def test_max_over_ranks_single_process_is_identity():
    import bench
    assert bench.max_over_ranks(0.25, None) == 0.25


def test_reference_arm_runs_on_rank_zero_only():
    import bench
    args = argparse.Namespace(steps=1, warmup=0)
    assert bench.run_reference(args, 1, 2) is None


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
