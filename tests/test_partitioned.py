"""The partitioned single-root BFS (graph500_b200.partitioned) on CPU ranks:
the level loop, the partition, the top-down pair exchange, the bottom-up
bitmap all-gather and the pred combination, with each rank's device work
done by a CPU stand-in (tests/part_cpu_engine.py).  Ranks run in one process
(LocalComm) and as world-size-2 gloo processes (TorchComm).  Every root's
levels must equal the oracle's BFS, and the oracle's restatement of
validate.hpp must accept the combined pred."""
import json
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests"))


def _levels(pred):
    lv = ((pred >> 48) & 0xFFFF).astype(np.uint16)
    lv[pred == -1] = 0xFFFF
    return lv


def _graph(oracle_mod, scale, vr):
    edges = oracle_mod.generate_edges(scale, 16)
    return edges, oracle_mod.Graph(edges, vr)


def _check(oracle_mod, edges, og, root, pred):
    assert np.array_equal(_levels(pred), og.bfs_levels(root)), root
    ok, evc, rep = oracle_mod.validate(edges, og.info["max_used_vertex"] + 1, og.info["pred_size"], root, pred)
    assert ok, rep
    return evc


@pytest.mark.parametrize("nranks", [1, 2, 3])
@pytest.mark.parametrize("vr,alpha,beta", [(2, 2000.0, 8.0), (0, 2000.0, 8.0), (2, 1e-9, 8.0), (2, 1e9, 1e9)])
def test_partitioned_in_one_process(oracle_mod, nranks, vr, alpha, beta):
    """alpha 1e-9: top-down only (every level exchanges pairs); alpha 1e9, beta
    1e9: bottom-up from level 2 on; the reference thresholds switch both ways."""
    from graph500_b200.partitioned import LocalComm, PartitionedBFS
    from part_cpu_engine import CpuRank
    edges, og = _graph(oracle_mod, 9, vr)
    ranks = [CpuRank(og, r, nranks) for r in range(nranks)]
    bfs = PartitionedBFS(LocalComm(nranks), ranks, og.info["num_global_verts"], alpha, beta)
    for root in og.find_roots(3).tolist():
        pred = bfs.run_bfs(root).numpy()
        _check(oracle_mod, edges, og, root, pred)
        dirs = {fwd for fwd, _ in bfs.levels}
        if alpha == 1e-9:
            assert dirs == {True}
        if alpha == 1e9:
            assert [fwd for fwd, _ in bfs.levels][1:] == [False] * (len(bfs.levels) - 1)


def test_partitioned_root_without_edges(oracle_mod):
    from graph500_b200.partitioned import LocalComm, PartitionedBFS
    from part_cpu_engine import CpuRank
    edges, og = _graph(oracle_mod, 9, 2)
    lonely = int(np.nonzero(og.degree == 0)[0][0])
    ranks = [CpuRank(og, r, 2) for r in range(2)]
    pred = PartitionedBFS(LocalComm(2), ranks, og.info["num_global_verts"]).run_bfs(lonely).numpy()
    assert pred[lonely] == lonely and (np.delete(pred, lonely) == -1).all()


def _gloo_rank(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    import torch
    from graph500_b200.partitioned import PartitionedBFS, TorchComm
    from part_cpu_engine import CpuRank
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    edges = oracle.generate_edges(9, 16)
    og = oracle.Graph(edges, 2)
    bfs = PartitionedBFS(TorchComm(dist, torch.device("cpu")), [CpuRank(og, rank, world)],
                         og.info["num_global_verts"], 2000.0, 8.0)
    res = {}
    for root in og.find_roots(3).tolist():
        pred = bfs.run_bfs(root).numpy()
        res[root] = pred.tolist()
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_partitioned_over_gloo_world_size_2(oracle_mod, tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_gloo_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    edges, og = _graph(oracle_mod, 9, 2)
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    assert got[0] == got[1]  # every rank ends with the same pred
    for root, pred in got[0].items():
        _check(oracle_mod, edges, og, int(root), np.asarray(pred, np.int64))
