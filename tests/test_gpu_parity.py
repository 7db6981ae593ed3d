"""CUDA path vs the oracle and the reference fixtures, through the C ABI.

Bit-exact for everything: edges, CSR, reorder maps, roots, levels; parents
are accepted iff both the device validator and the oracle's restatement of
validate.hpp accept them.
"""
import hashlib

import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden, pf_nedge

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# ----------------------------------------------------------------- generator
@pytest.mark.parametrize("scale", [1, 4, 10, 12, 16])
def test_generator_full_bit_exact(g500, oracle_mod, scale):
    assert np.array_equal(g500.generate_edges(scale).view(np.uint32),
                          oracle_mod.generate_edges(scale).view(np.uint32))


@pytest.mark.parametrize("scale,ef", [(20, 16), (22, 16), (26, 16), (14, 3)])
def test_generator_sampled_ranges(g500, oracle_mod, scale, ef):
    m = (1 << scale) * ef
    rng = np.random.default_rng(scale * 100 + ef)
    starts = [0, m - 4096] + [int(x) for x in rng.integers(0, m - 4096, 4)]
    for s in starts:
        dev = g500.generate_edges(scale, ef, s, s + 4096)
        ref = oracle_mod.generate_edges(scale, ef, s, s + 4096)
        assert np.array_equal(dev.view(np.uint32), ref.view(np.uint32)), (scale, s)


@pytest.mark.parametrize("scale,vr", GOLDEN_CASES)
def test_generator_matches_reference_fixture(g500, scale, vr):
    rec, arr = load_golden(scale, vr)
    e = g500.generate_edges(scale)
    assert sha(e) == rec["edges_sha256"]
    assert np.array_equal(e[:64], arr["edges_head"])


def test_generator_into_device_memory(g500, oracle_mod):
    import torch
    buf = torch.zeros((1 << 12) * 16 * 3, dtype=torch.int32, device="cuda")
    g500.generate_edges(12, out=buf)
    host = buf.cpu().numpy().view(g500.EDGE_DTYPE)
    assert np.array_equal(host.view(np.uint32), oracle_mod.generate_edges(12).view(np.uint32))


# -------------------------------------------------------------- construction
@pytest.mark.parametrize("scale", [8, 12, 14])
@pytest.mark.parametrize("vr", [0, 1, 2])
def test_csr_bit_exact(g500, oracle_mod, scale, vr):
    edges = oracle_mod.generate_edges(scale)
    og = oracle_mod.Graph(edges, vr)
    dg = g500.Graph2DCSR.build(edges, vr)
    info = dg.info
    assert [info.log_orig_global_verts, info.pred_size, info.num_local_verts, info.num_global_verts,
            info.num_global_edges, info.max_used_vertex] == list(og.info.values())
    csr = dg.copy_csr()
    assert np.array_equal(csr["offsets"], og.offsets)
    assert np.array_equal(csr["cols"], og.cols)
    assert np.array_equal(csr["reorder_map"], og.reorder_map)
    dg.close()


@pytest.mark.parametrize("scale,vr", GOLDEN_CASES)
def test_graph_info_and_roots_match_reference(g500, scale, vr):
    rec, _ = load_golden(scale, vr)
    g = g500.Graph2DCSR.generate(scale, 16, vr)
    got = [g.info.log_orig_global_verts, g.info.pred_size, g.info.num_local_verts, g.info.num_global_verts,
           g.info.num_global_edges, g.info.max_used_vertex]
    assert got == [rec["info"][k] for k in ("log_orig_global_verts", "pred_size", "num_local_verts",
                                           "num_global_verts", "num_global_edges", "max_used_vertex")]
    assert g500.find_roots(g, len(rec["roots"])).tolist() == rec["roots"]
    for v in rec["roots"][:4]:
        assert g.has_edge(v)
    g.close()


# ----------------------------------------------------------------------- BFS
@pytest.mark.parametrize("pred_mode", [1, 2, 3])  # pred written as found / deferred to one final pass / packed
@pytest.mark.parametrize("scale,vr", GOLDEN_CASES)
def test_bfs_levels_and_validation(g500, oracle_mod, scale, vr, pred_mode):
    rec, arr = load_golden(scale, vr)
    bfs = g500.BfsOnGPU(reorder_mode=vr)
    bfs.construct(g500.EdgeList(None, scale, 16))
    bfs.prepare_bfs()
    bfs.set_pred_mode(pred_mode)
    edges = oracle_mod.generate_edges(scale) if scale <= 16 else None
    pred = np.zeros(bfs.graph_.pred_size(), np.int64)
    for i, pr in enumerate(rec["per_root"]):
        st = bfs.run_bfs(pr["root"], pred)
        lv = g500.levels_from_pred(pred)
        assert sha(lv) == pr["levels_sha256"], (scale, vr, pr["root"])
        if f"levels_{i}" in arr:
            assert np.array_equal(lv, arr[f"levels_{i}"])
        ok, evc, rep = g500.validate_bfs_result(bfs.graph_, pr["root"], pred)
        assert ok, rep
        assert evc == pr["edge_visit_count"]
        assert st.nedge == evc and st.reached == int((lv != 0xFFFF).sum())
        if edges is not None and i < 3:
            ok2, evc2, rep2 = oracle_mod.validate(edges, bfs.graph_.info.max_used_vertex + 1,
                                                  bfs.graph_.pred_size(), pr["root"], pred)
            assert ok2 and evc2 == evc, rep2
    bfs.close()


@pytest.mark.parametrize("vr", [0, 2])
def test_level_counters_match_oracle_schedule(g500, oracle_mod, vr):
    """Per-level direction, frontier, discovered, scanned and the bytes-model
    counts equal the oracle's replay of bfs.hpp's direction rule."""
    scale = 14
    edges = oracle_mod.generate_edges(scale)
    og = oracle_mod.Graph(edges, vr)
    bfs = g500.BfsOnGPU(reorder_mode=vr)
    bfs.construct(edges)
    bfs.prepare_bfs(count_edges=True)
    pred = np.zeros(bfs.graph_.pred_size(), np.int64)
    for root in og.find_roots(6):
        bfs.run_bfs(int(root), pred)
        dev = bfs.level_stats()
        ref = og.dobfs_schedule(int(root))
        assert len(dev) == len(ref)
        for d, r in zip(dev, ref):
            assert d["direction"] == r["direction"]
            assert d["discovered"] == r["discovered"]
            if r["direction"] == 1:
                assert d["frontier"] == r["frontier"]
            else:
                assert d["scanned"] == r["scanned"]
            assert d["edges_examined"] == r["edges_examined"], (d, r)
            assert d["edge_sectors"] == r["edge_sectors"]
    bfs.close()


@pytest.mark.parametrize("policy,alpha,beta", [(0, 1e18, 8.0), (0, 1e-9, 1e-9), (0, 2000.0, 1e9), (0, 30.0, 2.0),
                                               (1, 15.0, 24.0), (1, 1e-9, 1e9), (1, 1e18, 1.0), (1, 2.0, 1e-9)])
def test_levels_independent_of_switch_thresholds(g500, oracle_mod, policy, alpha, beta):
    edges = oracle_mod.generate_edges(13)
    og = oracle_mod.Graph(edges, 2)
    bfs = g500.BfsOnGPU(reorder_mode=2)
    bfs.construct(edges)
    bfs.prepare_bfs(alpha, beta, policy=policy)
    pred = np.zeros(bfs.graph_.pred_size(), np.int64)
    for root in og.find_roots(4):
        bfs.run_bfs(int(root), pred)
        assert np.array_equal(g500.levels_from_pred(pred), og.bfs_levels(int(root)))
        assert g500.validate_bfs_result(bfs.graph_, int(root), pred)[0]
    bfs.close()


def test_autotune_keeps_results_identical(g500, oracle_mod):
    edges = oracle_mod.generate_edges(14)
    og = oracle_mod.Graph(edges, 2)
    bfs = g500.BfsOnGPU(reorder_mode=2)
    bfs.construct(edges)
    bfs.prepare_bfs()
    roots = og.find_roots(6)
    tune = bfs.autotune(roots[:3], reps=1)
    assert tune["configs_tried"] >= 8 and tune["best_ms"] <= tune["reference_ms"] + 1e-9
    pred = np.zeros(bfs.graph_.pred_size(), np.int64)
    for r in roots:
        bfs.run_bfs(int(r), pred)
        assert np.array_equal(g500.levels_from_pred(pred), og.bfs_levels(int(r)))
        assert g500.validate_bfs_result(bfs.graph_, int(r), pred)[0]
    bfs.close()


def test_pred_in_device_memory(g500, oracle_mod):
    import torch
    bfs = g500.BfsOnGPU(reorder_mode=2)
    bfs.construct(g500.EdgeList(None, 12, 16))
    bfs.prepare_bfs()
    rec, _ = load_golden(12, 2)
    pred = torch.empty(bfs.graph_.pred_size(), dtype=torch.int64, device="cuda")
    pred.fill_(12345)
    root = rec["per_root"][0]["root"]
    bfs.run_bfs(root, pred)
    torch.cuda.synchronize()
    host = pred.cpu().numpy()
    assert sha(g500.levels_from_pred(host)) == rec["per_root"][0]["levels_sha256"]
    ok, evc, _ = g500.validate_bfs_result(bfs.graph_, root, pred)
    assert ok and evc == rec["per_root"][0]["edge_visit_count"]
    bfs.close()


@pytest.mark.parametrize("scale,vr", [(16, 0), (18, 2)])
def test_host_pred_transfers(g500, oracle_mod, scale, vr):
    """A pageable host pred crosses PCIe as packed 32-bit entries that host
    threads expand; a pinned one, or any with packing off, as int64.  Every
    entry must be written (the buffer starts as garbage), the levels must be
    the reference's and the parents must validate.  (Parents are compared by
    validation, not entry by entry: two runs may pick different valid ones.)"""
    import ctypes
    rec, _ = load_golden(scale, vr)
    bfs = g500.BfsOnGPU(reorder_mode=vr)
    bfs.construct(g500.EdgeList(None, scale, 16))
    bfs.prepare_bfs()
    n = bfs.graph_.pred_size()
    hp = ctypes.c_void_p()
    g500.check(g500.lib().g500_host_alloc(8 * n, ctypes.byref(hp)))
    pinned = np.ctypeslib.as_array((ctypes.c_int64 * n).from_address(hp.value))
    edges = oracle_mod.generate_edges(scale)
    nglob = bfs.graph_.info.max_used_vertex + 1
    for pr in rec["per_root"][:3]:
        root = pr["root"]
        for on, kind in ((True, "pageable"), (False, "pageable"), (True, "pinned")):
            bfs.set_host_pack(on)
            host = np.empty(n, np.int64) if kind == "pageable" else pinned
            host[:] = 0x5A5A5A5A5A5A5A5A
            st = bfs.run_bfs(root, host)
            assert sha(g500.levels_from_pred(host)) == pr["levels_sha256"], (scale, vr, root, on, kind)
            ok, evc, rep = oracle_mod.validate(edges, nglob, n, root, host)
            assert ok and evc == pr["edge_visit_count"] == st.nedge, (rep, on, kind)
    bfs.set_host_pack(True)
    g500.check(g500.lib().g500_host_free(hp))
    bfs.close()


def _edges_from_pairs(g500, pairs):
    a = np.zeros(len(pairs), g500.EDGE_DTYPE)
    for i, (u, v) in enumerate(pairs):
        a[i] = (u & 0xFFFFFFFF, v & 0xFFFFFFFF, ((u >> 32) & 0xFFFF) | (((v >> 32) & 0xFFFF) << 16))
    return a


@pytest.mark.parametrize("pred_mode", [1, 2, 3])  # 3 on the path graph: deeper than the packed field
@pytest.mark.parametrize("name", ["path", "star", "big_star", "two_components", "self_loops_dups", "high_ids",
                                  "isolated_root"])
@pytest.mark.parametrize("vr", [0, 1, 2])
def test_small_graphs(g500, oracle_mod, name, vr, pred_mode):
    rng = np.random.default_rng(7)
    if name == "path":
        n = 3000  # depth > 255 levels
        pairs = [(i, i + 1) for i in range(n - 1)]
        root = 0
    elif name == "star":
        pairs = [(0, i) for i in range(1, 5000)]
        root = 17
    elif name == "big_star":  # a hub row of 30000 edges reached top-down: listed whole, spread over the warps
        pairs = [(0, i) for i in range(1, 30000)] + [(i, i + 30000) for i in range(1, 30000, 7)]
        root = 17
    elif name == "two_components":
        pairs = [(int(a), int(b)) for a, b in rng.integers(0, 500, (3000, 2))]
        pairs += [(int(a) + 1000, int(b) + 1000) for a, b in rng.integers(0, 300, (1000, 2))]
        root = pairs[0][0] if pairs[0][0] != pairs[0][1] else pairs[1][0]
    elif name == "self_loops_dups":
        pairs = [(5, 5), (5, 6), (6, 5), (5, 6), (6, 7), (7, 7), (7, 8), (9, 9)]
        root = 5
    elif name == "high_ids":
        pairs = [(70000, 3), (3, 131071), (131071, 99999), (12, 13)]
        root = 99999
    else:  # isolated root: only a self loop
        pairs = [(1, 2), (2, 3), (40, 40)]
        root = 40
    edges = _edges_from_pairs(g500, pairs)
    og = oracle_mod.Graph(edges, vr)
    bfs = g500.BfsOnGPU(reorder_mode=vr)
    bfs.construct(edges)
    info = bfs.graph_.info
    assert [info.log_orig_global_verts, info.pred_size, info.num_local_verts, info.num_global_verts,
            info.num_global_edges, info.max_used_vertex] == list(og.info.values())
    bfs.prepare_bfs()
    bfs.set_pred_mode(pred_mode)
    pred = np.full(bfs.graph_.pred_size(), 777, np.int64)
    st = bfs.run_bfs(root, pred)
    lv = g500.levels_from_pred(pred)
    assert np.array_equal(lv, og.bfs_levels(root))
    nglob = info.max_used_vertex + 1
    if root < nglob:
        ok_o, evc_o, rep_o = oracle_mod.validate(edges, nglob, info.pred_size, root, pred)
        ok_d, evc_d, rep_d = g500.validate_bfs_result(bfs.graph_, root, pred)
        assert ok_o and ok_d, (rep_o, rep_d)
        assert evc_o == evc_d == st.nedge
    bfs.close()


# ---------------------------------------------------------------- validation
@pytest.mark.parametrize("mutation", ["none", "level", "parent_not_edge", "self_parent", "range", "unreached",
                                      "root", "depth_gap"])
def test_device_validator_matches_oracle(g500, oracle_mod, mutation):
    rec, arr = load_golden(12, 0)
    edges = oracle_mod.generate_edges(12)
    g = g500.Graph2DCSR.build(edges, 0)
    root = rec["roots"][0]
    pred = arr["pred_0"].copy()
    reached = np.nonzero((pred != -1) & (np.arange(len(pred)) != root))[0]
    v = int(reached[len(reached) // 3])
    lvl = (pred >> 48) & 0xFFFF
    v0, v1 = oracle_mod.edge_endpoints(edges)
    if mutation == "level":
        pred[v] = (pred[v] & 0xFFFFFFFFFFFF) | ((int(lvl[v]) + 1) << 48)
    elif mutation == "parent_not_edge":
        nbrs = set(v1[v0 == v].tolist()) | set(v0[v1 == v].tolist())
        u = next(int(u) for u in reached if lvl[u] == lvl[v] - 1 and int(u) not in nbrs)
        pred[v] = u | (int(lvl[v]) << 48)
    elif mutation == "self_parent":
        pred[v] = v | (int(lvl[v]) << 48)
    elif mutation == "range":
        pred[v] = (1 << 40) | (int(lvl[v]) << 48)
    elif mutation == "unreached":
        pred[v] = -1
    elif mutation == "root":
        pred[root] = int(reached[0])
    elif mutation == "depth_gap":
        pred[v] = (pred[v] & 0xFFFFFFFFFFFF) | ((int(lvl[v]) + 2) << 48)
    ok_o, evc_o, _ = oracle_mod.validate(edges, g.info.max_used_vertex + 1, g.info.pred_size, root, pred)
    ok_d, evc_d, rep = g500.validate_bfs_result(g, root, pred, edges)
    assert ok_o == ok_d == (mutation == "none"), rep
    if ok_d:
        assert evc_d == evc_o == pf_nedge()[12]
    g.close()
