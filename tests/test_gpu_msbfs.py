"""Batched multi-source BFS vs the oracle: per-root uint8 levels are the BFS
distances (255 = unreached), bit-exact, for every lane width, with and without
the CUDA graph, under push-only and pull-only level schedules."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def as_u8(levels16: np.ndarray) -> np.ndarray:
    out = levels16.astype(np.int64)
    out[levels16 == 0xFFFF] = 255
    assert out.max() <= 255
    return out.astype(np.uint8)


@pytest.fixture(scope="module")
def s13(g500, oracle_mod):
    edges = oracle_mod.generate_edges(13)
    og = oracle_mod.Graph(edges, 2)
    g = g500.Graph2DCSR.build(edges, 2)
    roots = og.find_roots(64)
    want = np.stack([as_u8(og.bfs_levels(int(r))) for r in roots])
    yield g, og, roots, want
    g.close()


@pytest.mark.parametrize("lane_width", [32, 64, 128])
@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("alpha", [1e-12, 15.0, 1e12])
def test_msbfs_levels_bit_exact(g500, s13, lane_width, use_graph, alpha):
    g, og, roots, want = s13
    ms = g500.MultiSourceBFS(g, lane_width, alpha, use_graph)
    for n in (len(roots), 7):
        got = ms.levels(roots[:n])
        assert np.array_equal(got, want[:n]), (lane_width, use_graph, alpha, n)
    ms.close()


@pytest.mark.parametrize("lane_width", [32, 64, 128])
@pytest.mark.parametrize("sparse,limit", [(False, 0), (True, 1), (True, 300), (True, 0), (True, 1 << 40)])
def test_msbfs_sparse_levels_keep_levels(g500, s13, lane_width, sparse, limit):
    """Dense levels only, sparse push levels for small frontiers (limits 1 and
    300 put the switch between the two inside the search), and every push
    level sparse: the same levels.  alpha 1e-12 pushes every level; 15 mixes
    push and pull levels."""
    g, og, roots, want = s13
    ms = g500.MultiSourceBFS(g, lane_width, 15.0, True)
    ms.set_sparse(sparse, limit)
    for alpha in (1e-12, 15.0):
        ms.set_params(lane_width, alpha, True)
        for n in (len(roots), 5):
            assert np.array_equal(ms.levels(roots[:n]), want[:n]), (lane_width, sparse, limit, alpha, n)
    with pytest.raises(g500.G500Error) as ei:
        ms.set_sparse(True, -1)
    assert ei.value.code == g500.G500_E_INVAL
    ms.close()


def test_msbfs_repeated_runs_and_device_output(g500, s13):
    import torch
    g, og, roots, want = s13
    ms = g500.MultiSourceBFS(g, 64, 15.0, True)
    out = torch.full((64, g.pred_size()), 7, dtype=torch.uint8, device="cuda")
    for _ in range(3):
        ms.run(roots, out)
        assert np.array_equal(out.cpu().numpy(), want)
    # a different root set reuses the captured graph
    other = roots[::-1].copy()
    assert np.array_equal(ms.levels(other), want[::-1])
    ms.close()


def test_msbfs_root_stats_match_validator(g500, oracle_mod, s13):
    g, og, roots, want = s13
    ms = g500.MultiSourceBFS(g, 64)
    ms.run(roots[:16])
    reached, nedge = ms.root_stats(16)
    edges = oracle_mod.generate_edges(13)
    for i, r in enumerate(roots[:16]):
        assert reached[i] == int((want[i] != 255).sum())
        ok, evc, _ = oracle_mod.validate(edges, og.info["max_used_vertex"] + 1, og.info["pred_size"], int(r),
                                         og.bfs_pred(int(r)))
        assert ok and nedge[i] == evc
    ms.close()


def test_msbfs_matches_reference_fixture_levels(g500):
    rec, arr = load_golden(18, 2)
    g = g500.Graph2DCSR.generate(18, 16, 2)
    roots = [rec["per_root"][0]["root"], rec["per_root"][1]["root"]]
    ms = g500.MultiSourceBFS(g, 32)
    got = ms.levels(np.array(roots))
    for i in range(2):
        assert np.array_equal(got[i], as_u8(arr[f"levels_{i}"]))
    ms.close()
    g.close()


def test_msbfs_duplicate_and_isolated_roots(g500, oracle_mod):
    pairs = [(1, 2), (2, 3), (3, 4), (10, 11), (40, 40), (5, 6)]
    edges = np.zeros(len(pairs), g500.EDGE_DTYPE)
    for i, (u, v) in enumerate(pairs):
        edges[i] = (u, v, 0)
    og = oracle_mod.Graph(edges, 2)
    g = g500.Graph2DCSR.build(edges, 2)
    roots = np.array([1, 1, 40, 11, 4, 0])  # duplicates, an isolated root with a self loop, a vertex without edges
    ms = g500.MultiSourceBFS(g, 32)
    got = ms.levels(roots)
    for i, r in enumerate(roots):
        assert np.array_equal(got[i], as_u8(og.bfs_levels(int(r)))), r
    ms.close()
    g.close()


def test_msbfs_autotune_keeps_levels(g500, s13):
    g, og, roots, want = s13
    ms = g500.MultiSourceBFS(g, 64)
    tune = ms.autotune(roots, reps=1)
    assert tune["lane_width"] in (32, 64, 128) and tune["configs_tried"] == 15
    assert np.array_equal(ms.levels(roots), want)
    ms.close()


@pytest.fixture(scope="module")
def star(g500, oracle_mod):
    """A star whose centre has more than 2^20 neighbours (a hub row for both
    the pull and the push phase), a 40-vertex path hanging off one leaf, and
    2000 random edges among the leaves."""
    leaves = (1 << 20) + 300
    rng = np.random.default_rng(7)
    pairs = [np.stack([np.zeros(leaves, np.int64), np.arange(1, leaves + 1)], 1)]
    path = np.arange(leaves + 1, leaves + 41)
    pairs.append(np.stack([np.concatenate([[5], path[:-1]]), path], 1))
    pairs.append(rng.integers(1, leaves + 1, (2000, 2)))
    pr = np.concatenate(pairs)
    edges = np.zeros(len(pr), g500.EDGE_DTYPE)
    edges["v0_low"], edges["v1_low"] = pr[:, 0], pr[:, 1]
    og = oracle_mod.Graph(edges, 2)
    g = g500.Graph2DCSR.build(edges, 2)
    roots = np.array([0, 5, int(path[-1]), int(path[20]), 17, 123456, leaves], np.int64)
    want = np.stack([as_u8(og.bfs_levels(int(r))) for r in roots])
    yield g, roots, want
    g.close()


@pytest.mark.parametrize("lane_width", [32, 128])
@pytest.mark.parametrize("alpha", [1e-12, 1e12])
@pytest.mark.parametrize("sparse", [False, True])
def test_msbfs_hub_rows_keep_levels(g500, star, lane_width, alpha, sparse):
    """Rows longer than the hub thresholds are split into chunks that several
    warps take (push: over 256 entries, pull: over 2^20); alpha 1e-12 pushes
    every level and 1e12 pulls every level after the first."""
    g, roots, want = star
    ms = g500.MultiSourceBFS(g, lane_width, alpha, True)
    ms.set_sparse(sparse, 0)
    assert np.array_equal(ms.levels(roots), want), (lane_width, alpha, sparse)
    ms.close()


def test_msbfs_refuses_depth_beyond_uint8(g500):
    n = 300
    edges = np.zeros(n - 1, g500.EDGE_DTYPE)
    for i in range(n - 1):
        edges[i] = (i, i + 1, 0)
    g = g500.Graph2DCSR.build(edges, 0)
    ms = g500.MultiSourceBFS(g, 32)
    with pytest.raises(g500.G500Error) as ei:
        ms.run(np.array([0]))
    assert ei.value.code == g500.G500_E_RANGE
    # the handle stays usable for shallow searches
    assert ms.levels(np.array([150]))[0][150] == 0
    ms.close()
    g.close()
