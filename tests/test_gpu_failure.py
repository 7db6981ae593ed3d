"""Failure detection on the GPU without a fault: a persistent kernel's grid
barrier whose waits run out (one block never arrives) reports a timeout, and
the context stays usable for the next launch and for a BFS."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_barrier_wait_runs_out_and_context_recovers(g500):
    t, r = C.c_int32(), C.c_int32()
    g500.check(g500.lib().g500_selftest_barrier_timeout(0, C.byref(t), C.byref(r)))
    assert t.value == 1 and r.value == 1
    bfs = g500.BfsOnGPU()
    bfs.construct(g500.EdgeList(None, 10, 16))
    bfs.prepare_bfs()
    pred = np.zeros(bfs.graph_.pred_size(), np.int64)
    root = int(g500.find_roots(bfs.graph_, 1)[0])
    bfs.run_bfs(root, pred)
    assert g500.validate_bfs_result(bfs.graph_, root, pred)[0]
    bfs.close()
