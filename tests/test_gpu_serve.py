"""Serving loop (g500_server_*): queries on several resident graphs, batched
into multi-source launches as they arrive.  Every query's levels must equal
the oracle's BFS distances for its root, bit-exact, whether it ran alone or
inside a mix of concurrent queries on every graph; the per-query edge count
must equal the validator's edge_visit_count."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRAPHS = [(10, 2), (12, 2), (13, 0)]  # (SCALE, VERTEX_REORDERING)


def as_u8(levels16: np.ndarray) -> np.ndarray:
    out = levels16.astype(np.int64)
    out[levels16 == 0xFFFF] = 255
    return out.astype(np.uint8)


@pytest.fixture(scope="module")
def served(g500, oracle_mod):
    graphs, oracles, edges = [], [], []
    for scale, vr in GRAPHS:
        e = oracle_mod.generate_edges(scale)
        edges.append(e)
        oracles.append(oracle_mod.Graph(e, vr))
        graphs.append(g500.Graph2DCSR.build(e, vr))
    yield graphs, oracles, edges
    for g in graphs:
        g.close()


def pick_queries(graphs, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        gi = int(rng.integers(len(graphs)))
        roots = g500_roots(graphs[gi])
        out.append((gi, int(roots[int(rng.integers(len(roots)))])))
    return out


_roots_cache = {}


def g500_roots(graph):
    key = id(graph)
    if key not in _roots_cache:
        import graph500_b200 as g5
        _roots_cache[key] = g5.find_roots(graph, 64)
    return _roots_cache[key]


def run_alone(g500, graphs, queries, **cfg):
    srv = g500.Server(graphs, **cfg)
    out = {}
    for gi, r in queries:
        buf = np.full(graphs[gi].pred_size(), 7, np.uint8)
        qid = srv.submit(gi, r, levels=buf)
        srv.drain()
        res = srv.poll()
        assert len(res) == 1 and res[0]["id"] == qid and res[0]["status"] == 0
        assert res[0]["batch_size"] == 1
        out[(gi, r)] = (buf, res[0])
    srv.close()
    return out


# plain_below: calibrated, never plain, always plain; batch_target 32: a second launch of a graph
# waits until 32 of its queries wait (0, the default: no holding)
@pytest.mark.parametrize("plain_below,batch_target", [(-1, 0), (0, 0), (1000, 0), (0, 32)])
def test_serve_levels_alone_and_in_mix(g500, served, plain_below, batch_target):
    graphs, oracles, _ = served
    alone_q = pick_queries(graphs, 9, seed=1)
    alone = run_alone(g500, graphs, alone_q)
    for (gi, r), (buf, res) in alone.items():
        want = as_u8(oracles[gi].bfs_levels(r))
        assert np.array_equal(buf, want), (gi, r)
        assert res["reached"] == int((want != 255).sum())

    # the mix: every alone query again, plus many more on every graph, submitted back to back
    mix_q = alone_q + pick_queries(graphs, 400, seed=2) + alone_q
    srv = g500.Server(graphs, max_batch=128, max_workers_per_graph=2, plain_below=plain_below,
                      batch_target=batch_target)
    bufs, ids = [], []
    for gi, r in mix_q:
        b = np.full(graphs[gi].pred_size(), 7, np.uint8)
        bufs.append(b)
        ids.append(srv.submit(gi, r, tag=len(ids), levels=b))
    srv.drain()
    results = {}
    while True:
        got = srv.poll(1024)
        if not got:
            break
        for x in got:
            results[x["id"]] = x
    assert len(results) == len(mix_q)
    info = srv.info()
    srv.close()
    if plain_below == 0:
        assert info["launches"] < len(mix_q), "queries were not batched"
        assert max(x["batch_size"] for x in results.values()) > 1
    if plain_below == 1000:
        assert all(x["batch_size"] == 1 and x["lane_width"] == 0 for x in results.values())
    for k, (gi, r) in enumerate(mix_q):
        res = results[ids[k]]
        assert res["status"] == 0 and res["tag"] == k and res["graph"] == gi and res["root"] == r
        want = as_u8(oracles[gi].bfs_levels(r))
        assert np.array_equal(bufs[k], want), (k, gi, r)
        if (gi, r) in alone:
            abuf, ares = alone[(gi, r)]
            assert np.array_equal(bufs[k], abuf)
            assert (res["reached"], res["nedge"]) == (ares["reached"], ares["nedge"])


def test_serve_edge_counts_match_validator(g500, oracle_mod, served):
    graphs, oracles, edges = served
    qs = pick_queries(graphs, 12, seed=3)
    srv = g500.Server(graphs)
    for gi, r in qs:
        srv.submit(gi, r)
    srv.drain()
    res = srv.poll(64)
    srv.close()
    assert len(res) == len(qs)
    for x in res:
        og = oracles[x["graph"]]
        ok, evc, _ = oracle_mod.validate(edges[x["graph"]], og.info["max_used_vertex"] + 1, og.info["pred_size"],
                                         x["root"], og.bfs_pred(x["root"]))
        assert ok and x["nedge"] == evc


def test_serve_plain_mode_matches(g500, served):
    graphs, oracles, _ = served
    qs = pick_queries(graphs, 6, seed=4)
    srv = g500.Server(graphs, mode=g500.SERVE_PLAIN)
    bufs = []
    for gi, r in qs:
        b = np.zeros(graphs[gi].pred_size(), np.uint8)
        bufs.append(b)
        srv.submit(gi, r, levels=b)
    srv.drain()
    res = srv.poll(64)
    srv.close()
    assert len(res) == len(qs) and all(x["status"] == 0 and x["batch_size"] == 1 for x in res)
    for (gi, r), b in zip(qs, bufs):
        assert np.array_equal(b, as_u8(oracles[gi].bfs_levels(r)))


def test_serve_admission_by_free_memory(g500, served):
    graphs, _, _ = served
    qs = pick_queries(graphs, 600, seed=5)
    # a reserve larger than any device: no launch slot beyond the first per graph
    srv = g500.Server(graphs, max_workers_per_graph=4, hbm_reserve_bytes=1 << 60)
    for gi, r in qs:
        srv.submit(gi, r)
    srv.drain()
    assert len(srv.poll(1024)) == len(qs)
    assert srv.info()["workers"] == len(graphs)
    srv.close()


def test_serve_poisson_report(g500, served):
    graphs, _, _ = served
    srv = g500.Server(graphs)
    rep = srv.run_poisson(5000.0, 600, seed=2026, warmup=100)
    srv.close()
    assert rep["failed"] == 0 and rep["queries"] == 500
    assert 0 < rep["p50_ms"] <= rep["p99_ms"] <= rep["max_ms"]
    assert rep["gteps"] > 0 and rep["mean_batch"] >= 1 and rep["launches"] >= 1


@pytest.mark.parametrize("mode", ["DELIVER_DEVICE", "DELIVER_HOST"])
def test_serve_poisson_with_delivery(g500, served, mode):
    """Each load-generator query's levels are copied to a buffer of its own before
    it completes; the buffers are a bounded ring, so queries wait for a free one."""
    graphs, _, _ = served
    srv = g500.Server(graphs, max_batch=16, max_workers_per_graph=1)
    srv.set_delivery(getattr(g500, mode))
    rep = srv.run_poisson(20000.0, 600, seed=2026, warmup=100)
    assert rep["failed"] == 0 and rep["queries"] == 500 and rep["delivery"] == getattr(g500, mode)
    srv.set_delivery(g500.DELIVER_NONE)
    rep2 = srv.run_poisson(20000.0, 300, seed=7)
    assert rep2["failed"] == 0 and rep2["delivery"] == g500.DELIVER_NONE
    with pytest.raises(g500.G500Error):
        srv.set_delivery(7)
    srv.close()


def test_serve_rejects_bad_queries(g500, served):
    graphs, _, _ = served
    srv = g500.Server(graphs)
    with pytest.raises(g500.G500Error) as e:
        srv.submit(len(graphs), 0)
    assert e.value.code == g500.G500_E_INVAL
    with pytest.raises(g500.G500Error):
        srv.submit(0, graphs[0].pred_size())
    srv.close()


def test_msbfs_async_launch_and_small_grid(g500, served):
    graphs, oracles, _ = served
    g, og = graphs[1], oracles[1]
    roots = g500_roots(g)[:40]
    ms = g500.MultiSourceBFS(g, 64)
    ms.set_root_stats(True)
    for blocks in (0, 24):
        ms.set_grid(blocks)
        ms.launch(roots)
        while not ms.poll():
            pass
        ms.wait()
        lv = ms.device_levels(len(roots)).cpu().numpy()
        for i, r in enumerate(roots):
            assert np.array_equal(lv[i], as_u8(og.bfs_levels(int(r))))
        reached, _ = ms.root_stats(len(roots))
        assert list(reached) == [int((lv[i] != 255).sum()) for i in range(len(roots))]
    assert ms.grid(64)[0] == 24
    ms.close()
