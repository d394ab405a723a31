"""bench.py on N ranks: every rank runs its own replica of the step (the path is not
partitioned), the timed region is bracketed by a barrier on both sides and the reported
time is the maximum over ranks; the whole-job throughput counts every replica's steps.
Two gloo ranks on the CPU stand in for the NCCL ranks of the GPU box."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        r = bench.Ranks(ws, "cpu")
        r.barrier()
        local = 1.0 + rank  # rank 1 is the slow replica
        m = r.max(local)
        out[rank] = (m, r.throughput(10, m))
        r.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_throughput():
    ws = 2
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank, args=(ws, _port(), out), nprocs=ws, join=True)
        res = dict(out)
    assert res[0] == res[1] == (2.0, 10.0)  # 2 ranks x 10 steps / 2 s (the slower rank)


def test_single_rank_is_local():
    r = bench.Ranks(1, "cpu")
    r.barrier()
    assert r.max(3.5) == 3.5
    assert r.throughput(10, 2.0) == pytest.approx(5.0)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    """Under torchrun the reference arm prints from rank 0; the other ranks exit without work."""
    class A:
        workload, steps, warmup = "plate", 1, 0
    bench.bench_reference(A(), 2, 1)
    assert capsys.readouterr().out == ""
