"""bench.py's multi-GPU path on CPU: two gloo ranks under the torchrun
environment contract (replicas, barrier, max over ranks, whole-job value)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup(backend="gloo")
    bench.barrier(w)
    ms = 10.0 + 5.0 * r  # rank 1 is the slow replica
    mx = bench.max_over_ranks(ms, w, local, device="cpu")
    value = bench.job_throughput(w, 1000, 4, mx)
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, w, mx, value))


def test_two_gloo_ranks_take_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for r, w, mx, value in res:
        assert w == 2 and mx == 15.0
        assert value == pytest.approx(2 * 1000 * 4 / 0.015)
