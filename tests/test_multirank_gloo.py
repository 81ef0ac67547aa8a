"""The multi-rank paths of bench.py on CPU ranks (world size 2, gloo): the
max-over-ranks time, the whole-job replica rate, and the reference arm's
rank-0-only rule.  No GPU is touched."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import bench
    bench.torch = torch
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank                 # rank 1 is the slowest
        mx = bench.max_over_ranks(ms, device="cpu")
        rate = bench.replica_rate(world, 20, mx)
        dist.barrier()
        q.put((rank, mx, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [15.0, 15.0]
    assert all(abs(r[2] - 2 * 20 / 0.015) < 1e-9 for r in res)


def test_reference_arm_other_ranks_do_no_work(capsys):
    import bench

    class A:
        n = 256
        steps = 3
        warmup = 3
        ref_budget = 1.0
    bench.run_reference(A, rank=1, world=2)
    assert capsys.readouterr().out == ""
