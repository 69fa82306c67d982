"""Replica sharding across ranks (the multi-GPU form of bench.py), as gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from libvc1_b200.replicas import clip_seed, whole_job_rate


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seconds = 2.0 if rank == 1 else 1.0  # rank 1 is the slow one
        rate = whole_job_rate(1000.0, seconds, world)
        q.put((rank, rate, clip_seed(rank)))
    finally:
        dist.destroy_process_group()


def test_whole_job_rate_is_all_units_over_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank reports the same whole-job figure: 2 ranks x 1000 units / 2 s
    assert [g[1] for g in got] == [pytest.approx(1000.0)] * 2
    # and analyses its own clip
    assert got[0][2] != got[1][2]


def test_single_rank_needs_no_process_group():
    assert whole_job_rate(500.0, 0.5, 1) == pytest.approx(1000.0)


def test_ranks_get_distinct_clips():
    from libvc1_b200 import synth

    a = synth.generate(64, 48, 2, clip_seed(0))
    b = synth.generate(64, 48, 2, clip_seed(1))
    assert (a.frame(1)[0] != b.frame(1)[0]).any()
