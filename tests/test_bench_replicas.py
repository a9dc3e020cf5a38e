"""The multi-GPU bench path (replicas) with two gloo ranks on the CPU: the
slowest rank's time sets the whole-job throughput, and the reference arm does
its work on rank 0 only."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
        t = bench.max_over_ranks(ms, dist, device="cpu")
        dist.barrier()
        q.put((rank, t, bench.replica_throughput(world, 20, t), bench.dist_env()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, value, env in out:
        assert t == 150.0                       # max over ranks
        assert value == pytest.approx(2 * 20 / 0.150)  # both replicas' solves
        assert env == (rank, world, rank)


def test_single_process_keeps_its_own_time():
    assert bench.max_over_ranks(42.0) == 42.0
    assert bench.replica_throughput(1, 10, 1000.0) == pytest.approx(10.0)


def test_reference_arm_runs_on_rank0_only(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    import argparse
    ns = argparse.Namespace(gpus=2, steps=2, warmup=1, impl="reference", cpu_sample=1,
                            no_cpu=False, quick=True)
    assert bench.run_reference(ns) == 0     # returns at once, no solve, no output


def test_solve_bytes_counts_every_pass():
    """Per-solve algorithmic bytes: with unit-sized vectors and applies the
    count reduces to the passes of each solve, term by term."""
    n, nc, nrow = 1, 0, 0             # vectors of 4 / 8 bytes, no factors
    mixed, fp64 = bench.solve_bytes(n, nc, nrow, a32=0, a64=0, gcrk=2, steps=1, inner_iters=2,
                                    fp64_cycles=1)
    # mixed: initial 4*8; step: r32 (8+8) + res (8) + prec (12) + norm (4)
    # + iterations j=1,2: prec 12 + dots 4(j+1) + update 4(j+2) + xupdate 16
    # + x update 20 + residual 8 + norm 8
    it = sum(12 + 4 * (j + 1) + 4 * (j + 2) for j in (1, 2))
    assert mixed == 32 + 16 + 8 + 12 + 4 + it + 16 + 20 + 8 + 8
    # fp64: initial 32; cycle: prec 24 + norm 8 + scale 16 + 2 precs 48
    # + MGS (j=1: 16+24+16, j=2: 16+32+24) + xupdate 32 + residual 8 + norm 8
    assert fp64 == 32 + 24 + 8 + 16 + 48 + (16 + 24 + 16) + (16 + 32 + 24) + 32 + 8 + 8


def test_solve_bytes_counts_only_executed_iterations():
    """A cycle that stops early does not count its skipped step: with three
    iterations over two cycles (2 + 1) the count is one step j = 2 (prec 12,
    dots 12, update 16) and one x-update vector (4) below four (2 + 2)."""
    full, _ = bench.solve_bytes(1, 0, 0, a32=0, a64=0, gcrk=2, steps=2, inner_iters=4,
                                fp64_cycles=1)
    short, _ = bench.solve_bytes(1, 0, 0, a32=0, a64=0, gcrk=2, steps=2, inner_iters=3,
                                 fp64_cycles=1)
    assert full - short == 12 + 12 + 16 + 4
