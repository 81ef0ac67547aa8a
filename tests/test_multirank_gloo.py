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


def _ensemble_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    from dnsbox_b200.ensemble import CONFIG2_SIZES, gather_to_rank0, shard
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank reports a value that depends on the box only, for its
        # share of every size group of the 96-box ensemble
        local = {}
        for g in range(len(CONFIG2_SIZES)):
            for i in shard(32, rank, world):
                local[32 * g + i] = 0.5 * (32 * g + i) + 1.0
        q.put((rank, len(local), gather_to_rank0(local, world)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_ensemble_gathers_every_box_once(world):
    """Config-2 boxes split over the ranks with no collective but the final
    gather: every box is advanced by exactly one rank, shares differ by at most
    one box per size group, and rank 0 receives all 96 in index order."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_ensemble_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted((q.get(timeout=10) for _ in range(world)), key=lambda r: r[0])
    sizes = [r[1] for r in res]
    assert sum(sizes) == 96 and max(sizes) - min(sizes) <= 3
    merged = res[0][2]
    assert list(merged) == list(range(96)) and all(merged[i] == 0.5 * i + 1.0 for i in range(96))
    assert all(r[2] is None for r in res[1:])
