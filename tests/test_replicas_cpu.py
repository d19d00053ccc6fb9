"""Host logic of the N > 1 bench path on CPU: two gloo ranks, each timing its
own replica lattice; the job time is the max over ranks and the throughput
counts every rank's solves (replicas only: no collective on the data path)."""
import os
import socket
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    ms = 1000.0 + 250.0 * rank  # rank 1 is the slow one
    mx = bench.max_over_ranks(ms, world)
    theta, phi = bench.inputs(rank)
    q.put((rank, mx, bench.job_throughput(world, 4, mx), float(theta.sum()), float(np.abs(phi).sum())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas():
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
    for rank, mx, thr, _, _ in out:
        assert mx == 1250.0
        assert abs(thr - 2 * 4 / 1.25) < 1e-12
    # each rank draws its own lattice
    assert out[0][3] != out[1][3] and out[0][4] != out[1][4]


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_throughput(1, 5, 2000.0) == 2.5
