"""The partitioned single-root BFS with its CUDA rank work (g500_part_*): G
ranks emulated in one process on one GPU (LocalComm: the collectives are
copies between the ranks' buffers, made between the ranks' steps; no kernel
waits for another rank), and one rank over NCCL (TorchComm, world size 1).
Levels bit-exact against the oracle and the reference's SCALE 22 digests,
parents accepted by the device validator."""
import hashlib
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, load_golden_record

pytestmark = pytest.mark.gpu


def _levels16(pred):
    lv = ((pred >> 48) & 0xFFFF).astype(np.uint16)
    lv[pred == -1] = 0xFFFF
    return lv


@pytest.mark.parametrize("nranks", [1, 2, 3, 4, 8])
@pytest.mark.parametrize("scale,vr", [(12, 2), (14, 0)])
@pytest.mark.parametrize("alpha,beta", [(2000.0, 8.0), (1e-9, 8.0), (1e9, 1e9)])
def test_partitioned_levels_and_parents(g500, oracle_mod, nranks, scale, vr, alpha, beta):
    from graph500_b200.partitioned import CudaRank, LocalComm, PartitionedBFS
    edges = oracle_mod.generate_edges(scale, 16)
    og = oracle_mod.Graph(edges, vr)
    g = g500.Graph2DCSR.generate(scale, 16, vr)
    ranks = [CudaRank(g, r, nranks) for r in range(nranks)]
    bfs = PartitionedBFS(LocalComm(nranks), ranks, g.info.num_global_verts, alpha, beta)
    for root in g500.find_roots(g, 4).tolist():
        pred = bfs.run_bfs(root)
        assert np.array_equal(_levels16(pred.cpu().numpy()), og.bfs_levels(root)), (nranks, root)
        ok, evc, rep = g500.validate_bfs_result(g, root, pred)
        assert ok, rep
    lonely = int(np.nonzero(og.degree == 0)[0][0])
    pred = bfs.run_bfs(lonely).cpu().numpy()
    assert pred[lonely] == lonely and (np.delete(pred, lonely) == -1).all()
    bfs.close()
    g.close()


@pytest.mark.slow
def test_partitioned_matches_reference_at_scale_22(g500):
    """4 ranks on the SCALE 22 graph: the reference's level digests."""
    import torch
    from graph500_b200.partitioned import CudaRank, LocalComm, PartitionedBFS
    rec = load_golden_record(22, 2)
    g = g500.Graph2DCSR.generate(22, 16, 2)
    ranks = [CudaRank(g, r, 4) for r in range(4)]
    bfs = PartitionedBFS(LocalComm(4), ranks, g.info.num_global_verts, 2000.0, 8.0)
    for pr in rec["per_root"][:6]:
        pred = bfs.run_bfs(pr["root"])
        lv = _levels16(pred.cpu().numpy())
        assert hashlib.sha256(lv.tobytes()).hexdigest() == pr["levels_sha256"], pr["root"]
        ok, evc, _ = g500.validate_bfs_result(g, pr["root"], pred)
        assert ok and evc == pr["edge_visit_count"]
    bfs.close()
    g.close()
    torch.cuda.empty_cache()


def test_partitioned_over_nccl_one_rank(g500, tmp_path):
    """TorchComm over an NCCL process group of one rank (the multi-GPU path's
    collectives on this GPU), in a child process."""
    code = (
        "import os, sys, datetime, torch, numpy as np\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "import torch.distributed as dist, graph500_b200 as g5, oracle\n"
        "from graph500_b200.partitioned import CudaRank, PartitionedBFS, TorchComm\n"
        "os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=sys.argv[1], NCCL_NVLS_ENABLE='0')\n"
        "torch.cuda.set_device(0)\n"
        "dist.init_process_group('nccl', rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),\n"
        "                        device_id=torch.device('cuda', 0))\n"
        "g = g5.Graph2DCSR.generate(12, 16, 2)\n"
        "og = oracle.Graph(oracle.generate_edges(12, 16), 2)\n"
        "bfs = PartitionedBFS(TorchComm(dist, torch.device('cuda', 0)), [CudaRank(g, 0, 1)], g.info.num_global_verts)\n"
        "for r in g5.find_roots(g, 3).tolist():\n"
        "    p = bfs.run_bfs(r).cpu().numpy()\n"
        "    lv = ((p >> 48) & 0xFFFF).astype(np.uint16); lv[p == -1] = 0xFFFF\n"
        "    assert np.array_equal(lv, og.bfs_levels(r)), r\n"
        "bfs.close(); dist.destroy_process_group(); print('nccl ok')\n")
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-c", code, str(port)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "nccl ok" in r.stdout, r.stderr[-3000:]
