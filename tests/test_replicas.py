"""The N > 1 path on CPU: two gloo ranks run the replica plumbing bench.py
uses on GPUs (disk sizes per rank, barrier, max over ranks, job rate)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from disco_b200.replicas import job_rate, max_over_ranks, rank_specs
        specs = rank_specs(rank, ndisk=8)
        units = sum(nr for nr, _, _ in specs)            # stands in for real cells
        ms = 10.0 + 5.0 * rank                           # rank 1 is the slow one
        dist.barrier()
        mx = max_over_ranks(ms, dist)
        rate = job_rate(world, units, 4, mx)
        # every rank sees the same maximum and the same job rate
        got = [None] * world
        dist.all_gather_object(got, (specs, mx, rate))
        if rank == 0:
            out.put(got)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (s0, m0, r0), (s1, m1, r1) = got
    assert [a[:2] for a in s0] == [a[:2] for a in s1]     # same sizes and Mach numbers
    assert not set(a[2] for a in s0) & set(a[2] for a in s1)   # own noise seeds
    assert m0 == m1 == 15.0                               # the slowest rank's time
    units = sum(nr for nr, _, _ in s0)
    assert r0 == r1 == pytest.approx(2 * units * 4 / 0.015)


def test_single_process_needs_no_group():
    from disco_b200.replicas import job_rate, max_over_ranks
    assert max_over_ranks(3.5) == 3.5
    assert job_rate(1, 1000, 10, 2.0) == pytest.approx(5e6)
