"""Multi-GPU is replicas only: every rank renders its own frames, the job's
time is the maximum over ranks and the value counts all ranks' pixels.
These tests run the bench's rank plumbing as two gloo processes on the CPU
(no GPU): rendezvous, max-over-ranks, barrier, and the reference arm where
only rank 0 does work."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))


def _max_worker(rank, port, q):
    import sys
    sys.path.insert(0, ROOT)
    _env(rank, port)
    import torch.distributed as dist
    import bench
    ws, r, local = bench.dist_setup()
    t = bench.dist_max(0.5 + rank, ws)   # rank 1 is the slower one
    bench.dist_barrier(ws)
    q.put((r, ws, local, t))
    dist.destroy_process_group()


def _reference_worker(rank, port, q):
    import sys
    sys.path.insert(0, ROOT)
    _env(rank, port)
    import bench

    class Args:
        steps, warmup = 1, 1
    if rank == 1:
        q.put((rank, bench.run_reference_arm(Args)))
    else:
        # rank 0 would run the reference; here it only joins the rendezvous
        ws, r, _ = bench.dist_setup()
        q.put((rank, ws))


@pytest.mark.parametrize("worker", ["max"])
def test_two_ranks_max_and_barrier(worker):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_max_worker, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 2 for o in out)
    assert all(o[3] == 1.5 for o in out)   # both ranks see the slowest rank's time


def test_reference_arm_only_rank0_works():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_reference_worker, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert out[1] == 0     # rank 1 returns at once, without work
    assert out[0] == 2
