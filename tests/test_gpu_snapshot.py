"""A graph saved to a snapshot and loaded back is the same graph: CSR, maps,
scalars, roots, and BFS results (levels bit-exact, parents valid against the
kept edge list)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("vr", [0, 2])
def test_snapshot_round_trip(g500, tmp_path, vr):
    g = g500.Graph2DCSR.generate(13, 16, vr)
    path = str(tmp_path / "s13.g500")
    g.save(path)
    h = g500.Graph2DCSR.load(path)
    fields = [f[0] for f in g500.GraphInfo._fields_]
    assert [getattr(g.info, f) for f in fields] == [getattr(h.info, f) for f in fields]
    a, b = g.copy_csr(), h.copy_csr()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    ra, rb = g500.find_roots(g, 16), g500.find_roots(h, 16)
    assert np.array_equal(ra, rb)
    for v in range(0, g.pred_size(), 97):
        assert g.has_edge(v) == h.has_edge(v)
    ba, bb = g500.BfsOnGPU(), g500.BfsOnGPU()
    ba.graph_, bb.graph_ = g, h
    ba.prepare_bfs()
    bb.prepare_bfs()
    pa = np.zeros(g.pred_size(), np.int64)
    pb = np.zeros(h.pred_size(), np.int64)
    for r in ra[:4]:
        ba.run_bfs(int(r), pa)
        bb.run_bfs(int(r), pb)
        assert np.array_equal(g500.levels_from_pred(pa), g500.levels_from_pred(pb))
        ok, evc, _ = g500.validate_bfs_result(h, int(r), pb)  # the loaded graph's own edge list
        assert ok and evc == g500.validate_bfs_result(g, int(r), pa)[1]
    ba.close()
    bb.close()


def test_truncated_snapshot_is_refused(g500, tmp_path):
    g = g500.Graph2DCSR.generate(11, 16, 2)
    path = str(tmp_path / "s11.g500")
    g.save(path)
    g.close()
    size = os.path.getsize(path)
    with open(path, "r+b") as f:
        f.truncate(size - 100)
    with pytest.raises(g500.G500Error) as e:
        g500.Graph2DCSR.load(path)
    assert e.value.code == g500.G500_E_IO
