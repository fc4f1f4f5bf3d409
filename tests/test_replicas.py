"""Multi-rank replica path of bench.py, run as two gloo ranks on the CPU.

The reconstruction does not shard: each rank runs its own independent
reconstruction (same array and scene, its own noise seed) with no data-path
collective. The only exchange is the whole-job reduction after the timed
region: the slowest rank's time (max) and the work of all ranks (sum).
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        times, work = bench.combine_over_ranks([1.0 + rank, 5.0 - rank], [10.0 * (rank + 1), 3.0])
        seeds = bench.replica_seeds(rank)
        import gpair_b200 as g
        p = g.workload_problem("tiny", **seeds)
        q.put((rank, times, work, seeds, p.npow, p.nbis, p.nuv, float(np.sum(p.data))))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, times, work, seeds, *_ in res:
        assert times == [2.0, 5.0]  # max over ranks
        assert work == [30.0, 6.0]  # sum over ranks
    (_, _, _, s0, np0, nb0, nu0, d0), (_, _, _, s1, np1, nb1, nu1, d1) = res
    # same array and scene (same shapes and uv coverage), independent noise
    assert s0["scene_seed"] == s1["scene_seed"] and s0["array_seed"] == s1["array_seed"]
    assert s0["noise_seed"] != s1["noise_seed"]
    assert (np0, nb0, nu0) == (np1, nb1, nu1)
    assert d0 != d1


def test_reference_arm_other_ranks_exit_without_work(capsys):
    import bench

    class A:
        workload = "tiny"
        warmup = 1
        steps = 1
        gpus = 2

    bench.run_reference(A, rank=1)
    assert capsys.readouterr().out == ""
