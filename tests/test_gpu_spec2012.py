"""The spec-2012 generator on the GPU (g500_gen_edges_spec2012) against the
oracle's restatement and the reference's own edge lists
(generate_graph_spec2012, mpi/benchmark_helper.hpp:316-322): every 16-byte
WeightedEdge bit-exact, the N - 1 binary-tree initial edges first, the R-MAT
edges (A = .55, B = C = .01) after them, weight 0xBEEF."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def endpoints(e):
    return np.ascontiguousarray(e.view(np.uint32).reshape(-1, 4)[:, :3])


@pytest.mark.parametrize("scale", [1, 4, 10, 12, 16])
def test_spec2012_full_bit_exact(g500, oracle_mod, scale):
    got = g500.generate_edges_spec2012(scale)
    want = oracle_mod.generate_edges_spec2012(scale)
    assert len(got) == (1 << scale) * 17 - 1
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("scale", [4, 10, 12, 16])
def test_spec2012_matches_reference_fixture(g500, scale):
    rec = json.load(open(os.path.join(GOLDEN, f"ref_spec2012_s{scale}.json")))
    arr = dict(np.load(os.path.join(GOLDEN, f"ref_spec2012_s{scale}.npz")))
    e = g500.generate_edges_spec2012(scale)
    assert len(e) == rec["num_edges"]
    assert sha(endpoints(e)) == rec["endpoints_sha256"]
    assert np.array_equal(endpoints(e[:64]), endpoints(arr["edges_head"]))
    assert (e["weight"] == 0xBEEF).all()


@pytest.mark.parametrize("scale", [20, 22, 26])
def test_spec2012_sampled_ranges(g500, oracle_mod, scale):
    """Ranges across the tree / R-MAT boundary and deep into the R-MAT part."""
    n = 1 << scale
    m = n * 16 + n - 1
    rng = np.random.default_rng(scale)
    starts = [0, n - 1 - 2048, m - 4096] + [int(x) for x in rng.integers(0, m - 4096, 3)]
    for s in starts:
        got = g500.generate_edges_spec2012(scale, 16, s, s + 4096)
        want = oracle_mod.generate_edges_spec2012(scale, 16, s, s + 4096)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (scale, s)


def test_spec2012_into_device_memory_and_bounds(g500, oracle_mod):
    import torch
    n = 1 << 12
    m = n * 16 + n - 1
    buf = torch.zeros(m * 4, dtype=torch.int32, device="cuda")
    g500.generate_edges_spec2012(12, out=buf)
    host = buf.cpu().numpy().view(g500.WEDGE_DTYPE)
    assert np.array_equal(host.view(np.uint32), oracle_mod.generate_edges_spec2012(12).view(np.uint32))
    with pytest.raises(g500.G500Error) as e:
        g500.generate_edges_spec2012(12, 16, m - 10, m + 1)
    assert e.value.code == g500.G500_E_RANGE


def test_spec2012_graph_builds_and_traverses(g500, oracle_mod):
    """The spec-2012 endpoints (the weight dropped: the first 12 bytes are the
    packed layout) build a CSR and traverse like the oracle's BFS; the binary
    tree makes every vertex reachable from any root."""
    e = g500.generate_edges_spec2012(12)
    packed = np.ascontiguousarray(endpoints(e)).view(g500.EDGE_DTYPE).reshape(-1)
    g = g500.Graph2DCSR.build(packed, 2)
    og = oracle_mod.Graph(packed.view(oracle_mod.EDGE_DTYPE), 2)
    bfs = g500.BfsOnGPU()
    bfs.graph_ = g
    bfs.prepare_bfs()
    pred = np.zeros(g.pred_size(), np.int64)
    for r in g500.find_roots(g, 4):
        bfs.run_bfs(int(r), pred)
        lv = g500.levels_from_pred(pred)
        assert np.array_equal(lv, og.bfs_levels(int(r)))
        assert (lv[:1 << 12] != 0xFFFF).all()  # ids past 2^SCALE only pad pred_size
    bfs.close()
