"""g500_validate_noalloc: Graph500 validation that allocates no device memory.

It serves callers that cannot call cudaMalloc -- a host framework that owns
all device memory through its own arena or caching allocator, or a serving
loop that forbids allocation once it is running.  Its scratch is a fixed
device array inside libg500.so, so this test checks it against the
allocating entry point (g500_validate) on the same inputs, on calls made back
to back (the shared scratch must not carry state from one call to the next).

The file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(g5, eptr, m, nglob, nloc, root, pred):
    evc, ok, rep = C.c_int64(), C.c_int(), g5.ValidateReport()
    pptr, on_dev = g5._ptr(pred)
    assert on_dev
    g5.check(g5.lib().g500_validate_noalloc(eptr, m, nglob, nloc, int(root), pptr, None, C.byref(evc), C.byref(ok),
                                           C.byref(rep)))
    return bool(ok.value), evc.value, {f[0]: getattr(rep, f[0]) for f in g5.ValidateReport._fields_}


def test_noalloc_validation_matches_allocating_validation(g500):
    import torch

    bfs = g500.BfsOnGPU(reorder_mode=2)
    bfs.construct(g500.EdgeList(None, 14, 16))
    bfs.prepare_bfs()
    g = bfs.graph_
    eptr, m = g.device_edges()
    assert eptr and m == (1 << 14) * 16
    nglob, nloc = g.info.max_used_vertex + 1, g.pred_size()
    roots = g500.find_roots(g, 3)
    pred = torch.empty(nloc, dtype=torch.int64, device="cuda")

    for r in roots[:2]:
        bfs.run_bfs(int(r), pred)
        want = g500.validate_bfs_result(g, int(r), pred)
        first = _noalloc(g500, eptr, m, nglob, nloc, r, pred)
        second = _noalloc(g500, eptr, m, nglob, nloc, r, pred)
        assert want[0] and first == second == want

    # a wrong level planted in the result (host side), then a valid result again:
    # the second call must not see the first call's counters or flags
    r = int(roots[2])
    bfs.run_bfs(r, pred)
    host = pred.cpu().numpy()
    reached = np.nonzero((host != -1) & (np.arange(len(host)) != r))[0]
    v = int(reached[len(reached) // 2])
    bad = host.copy()
    bad[v] = (bad[v] & 0xFFFFFFFFFFFF) | ((((int(bad[v]) >> 48) & 0xFFFF) + 1) << 48)
    bad_dev = torch.from_numpy(bad).cuda()
    want_bad = g500.validate_bfs_result(g, r, bad_dev)
    got_bad = _noalloc(g500, eptr, m, nglob, nloc, r, bad_dev)
    assert not want_bad[0] and got_bad == want_bad
    want_ok = g500.validate_bfs_result(g, r, pred)
    got_ok = _noalloc(g500, eptr, m, nglob, nloc, r, pred)
    assert want_ok[0] and got_ok == want_ok
    bfs.close()


def test_noalloc_refuses_sizes_beyond_its_scratch(g500):
    import torch

    L = g500.lib()
    limit = 1 << 22  # G500_VALIDATE_STATIC_MAX_VERTS
    pred = torch.full((8,), -1, dtype=torch.int64, device="cuda")
    evc, ok = C.c_int64(), C.c_int()
    rc = L.g500_validate_noalloc(None, 0, 1, limit + 1, 0, pred.data_ptr(), None, C.byref(evc), C.byref(ok), None)
    assert rc == g500.G500_E_RANGE
    assert b"at most" in L.g500_last_error()


def test_noalloc_refuses_buffers_off_the_current_device(g500):
    """pred (or the edge list) that is not memory of the current device is refused
    before any kernel runs; a host array stands in for another device's buffer."""
    L = g500.lib()
    host_pred = np.full(64, -1, dtype=np.int64)
    evc, ok = C.c_int64(), C.c_int()
    rc = L.g500_validate_noalloc(None, 0, 1, 64, 0, host_pred.ctypes.data, None, C.byref(evc), C.byref(ok), None)
    assert rc == g500.G500_E_INVAL
    assert b"device memory" in L.g500_last_error()
