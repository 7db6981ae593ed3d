"""The CUDA path against the unmodified reference at the benchmark sizes.

1. Levels at Kronecker SCALE 22 and 24 (edgefactor 16, VERTEX_REORDERING 2,
   the 64 find_roots roots): for every root, the sha256 of the level array
   ((pred >> 48) & 0xFFFF per original vertex id, 0xFFFF when unreached), the
   level histogram and edge_visit_count equal the records of the reference's
   own run_bfs (mpi/bfs.hpp:2651-2940) and validator (mpi/validate.hpp:
   1008-1019), made by tests/golden/make_golden.py --large.  Checked for the
   plain BFS in every pred mode and for the 64-root multi-source launch.
2. Parents: the reference's compiled validate_bfs_result (oracle/_ref,
   ref_driver.cc ref_validate) accepts the GPU's pred arrays at SCALE 12-18,
   every pred mode, and counts the same edge_visit_count.  The reference keeps
   global state, so it runs in a child process per case (no GPU there).
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN_CASES, LARGE_GOLDEN_CASES, ROOT, load_golden, load_golden_record, pf_nedge

pytestmark = pytest.mark.gpu


def level_digest_u16(torch, pred):
    """(sha256, histogram) of the uint16 level array of a device pred."""
    lv = (pred >> 48) & 0xFFFF
    lv = torch.where(pred == -1, torch.full_like(lv, 0xFFFF), lv).to(torch.int32)
    host = lv.cpu().numpy().astype(np.uint16)
    hist = np.bincount(np.where(host == 0xFFFF, 0, host.astype(np.int64) + 1)).tolist()
    return hashlib.sha256(host.tobytes()).hexdigest(), hist


def ms_digest_u16(torch, lv8):
    """(sha256, histogram) of a multi-source uint8 level row (255 unreached) as uint16."""
    host = lv8.cpu().numpy().astype(np.uint16)
    host[host == 255] = 0xFFFF
    hist = np.bincount(np.where(host == 0xFFFF, 0, host.astype(np.int64) + 1)).tolist()
    return hashlib.sha256(host.tobytes()).hexdigest(), hist


@pytest.mark.slow
@pytest.mark.parametrize("scale,vr", LARGE_GOLDEN_CASES)
def test_levels_match_reference_at_benchmark_size(g500, scale, vr):
    import torch
    rec = load_golden_record(scale, vr)
    g = g500.Graph2DCSR.generate(scale, 16, vr)
    info = g.info
    assert [info.log_orig_global_verts, info.pred_size, info.num_local_verts, info.num_global_verts,
            info.num_global_edges, info.max_used_vertex] == [
        rec["info"][k] for k in ("log_orig_global_verts", "pred_size", "num_local_verts", "num_global_verts",
                                 "num_global_edges", "max_used_vertex")]
    roots = g500.find_roots(g, len(rec["roots"]))
    assert roots.tolist() == rec["roots"]
    bfs = g500.BfsOnGPU(reorder_mode=vr)
    bfs.graph_ = g
    bfs.prepare_bfs()
    pred = torch.empty(g.pred_size(), dtype=torch.int64, device="cuda")
    for mode in (1, 2, 3):  # as found, deferred 64-bit entries, deferred packed entries
        bfs.set_pred_mode(mode)
        for pr in rec["per_root"]:
            st = bfs.run_bfs(pr["root"], pred)
            d, hist = level_digest_u16(torch, pred)
            assert hist == pr["level_hist"], (scale, mode, pr["root"])
            assert d == pr["levels_sha256"], (scale, mode, pr["root"])
            if "edge_visit_count" in pr:
                assert st.nedge == pr["edge_visit_count"] == pf_nedge()[scale], (scale, mode, pr["root"])
    bfs.set_pred_mode(0)
    ms = g500.MultiSourceBFS(g, 64, 15.0, True)
    ms.run(roots)
    out = ms.device_levels(len(roots))
    for i, pr in enumerate(rec["per_root"]):
        d, hist = ms_digest_u16(torch, out[i])
        assert hist == pr["level_hist"], (scale, "multi-source", pr["root"])
        assert d == pr["levels_sha256"], (scale, "multi-source", pr["root"])
    ms.close()
    bfs.close()
    g.close()


@pytest.mark.parametrize("scale,vr", GOLDEN_CASES[1:])
def test_reference_validator_accepts_gpu_preds(g500, scale, vr):
    """The reference's own validator, run on the GPU's parents."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", f"libg500ref_vr{vr}.so")):
        pytest.skip("the reference was not compiled (oracle/_ref)")
    import torch
    rec, _ = load_golden(scale, vr)
    g = g500.Graph2DCSR.generate(scale, 16, vr)
    bfs = g500.BfsOnGPU(reorder_mode=vr)
    bfs.graph_ = g
    bfs.prepare_bfs()
    pred = torch.empty(g.pred_size(), dtype=torch.int64, device="cuda")
    roots = rec["roots"][:4]
    preds, want = {}, {}
    for mode in (1, 2, 3):
        bfs.set_pred_mode(mode)
        for r in roots:
            st = bfs.run_bfs(r, pred)
            preds[f"m{mode}_r{r}"] = pred.cpu().numpy()
            want[f"m{mode}_r{r}"] = (r, st.nedge)
    bfs.close()
    g.close()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "preds.npz")
        np.savez(path, **preds)
        env = dict(os.environ, NO_AFFINITY="1", CUDA_VISIBLE_DEVICES="")
        out = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "_ref_validate.py"), str(scale), str(vr),
                              path], capture_output=True, text=True, env=env, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    for key, (r, nedge) in want.items():
        ok, evc = res[key]
        assert ok, (scale, vr, key)
        assert evc == nedge, (scale, vr, key, evc, nedge)
        by_root = {p["root"]: p["edge_visit_count"] for p in rec["per_root"]}
        assert evc == by_root[r]
