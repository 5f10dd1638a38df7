"""The multi-GPU mode of bench.py (replicas: one independent proof per rank,
no collective on the data path) exercised with world_size 2 on CPU over gloo:
the per-rank timing reduction takes the slowest rank, the whole-job value
counts every rank's proof, each rank gets its own seeded polynomial, and the
reference arm runs on rank 0 only."""
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


def _rank_main(rank, world, port, out):
    import numpy as np
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    local = 10.0 + 5.0 * rank  # rank 1 is slower
    mx = bench.reduce_over_ranks(local, dist, "cpu")
    step_ms, value = bench.job_value(mx, 5, world)
    import __graft_entry__

    pkg = __graft_entry__.load_package()
    poly, point = bench.inputs(pkg.rng_koalabear, rank, 10)
    polys = [None] * world
    dist.all_gather_object(polys, poly[:8].tolist())
    out[rank] = (mx, step_ms, value, polys)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduction_and_inputs():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    for rank in range(world):
        mx, step_ms, value, polys = out[rank]
        assert mx == 15.0  # the slowest rank
        assert step_ms == 3.0 and value == 1.5  # 2 proofs per step over the job
        assert polys[0] != polys[1]  # independent inputs per replica


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import bench

    monkeypatch.setenv("RANK", "1")

    class A:
        steps, warmup, gpus = 1, 0, 2

    bench.run_reference(A())  # returns without any work on rank 1
    assert capsys.readouterr().out == ""
