"""bench.py's multi-GPU path on CPU: two gloo ranks merge their measurements
the way the GPU ranks do (times: max over ranks; edges: sum), and every rank
takes the same collective steps."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    rep = bench.Replicas(dist, "cpu")
    rep.barrier()
    t = [1.0, 2.0][rank]       # this rank's device seconds
    e = [10.0, 30.0][rank]     # this rank's traversed edges
    out = (rep.max(t), rep.sum(e), rep.gteps(e * 1e9, t))
    rep.barrier()
    dist.destroy_process_group()
    q.put((rank, out))


def test_two_replicas_merge_like_the_gpu_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert res[r] == (2.0, 40.0, 40.0 / 2.0)


def test_single_process_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    rep = bench.Replicas(None)
    rep.barrier()
    assert rep.max(3.0) == 3.0 and rep.sum(4.0) == 4.0 and rep.gteps(8e9, 2.0) == 4.0
