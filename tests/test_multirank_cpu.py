"""The N>1 path of bench.py on CPU ranks (gloo, world size 2): replicas build
bit-identical tables from the same seed, the job rate uses the slowest rank's
time, and a rank that fails is seen by the other through the store before any
collective (no GPU is involved)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from bigstickpublick_b200 import model
        T = model.build_tables(model.sd_model(3, 3, seed=2))
        digest = bench.table_checksum(T)
        got = [None] * world
        dist.all_gather_object(got, digest)
        t_rank = 1.0 + rank  # seconds this rank "took"
        tmax = bench.reduce_max(t_rank, dist)
        rate = bench.replica_rate(10, world, tmax)
        q.put((rank, got, tmax, rate))
    finally:
        dist.destroy_process_group()


def test_replicas_identical_and_rate_uses_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, digests, tmax, rate in res:
        assert len(set(digests)) == 1
        assert tmax == 2.0
        assert rate == pytest.approx(2 * 10 / 2.0)


def _failing_worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    store = dist.TCPStore("127.0.0.1", port, world, rank == 0, timeout=datetime.timedelta(seconds=30))
    if rank == 1:
        store.set("status/1", "failed: table validation")  # rank 1 fails before its first launch
        q.put((rank, "exited"))
        return
    store.wait(["status/1"], datetime.timedelta(seconds=30))
    q.put((rank, store.get("status/1").decode()))


def test_failed_rank_is_seen_through_the_store():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=60) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
    assert res[0].startswith("failed")
