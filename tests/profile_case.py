"""A small, self-contained run of every kernel on the path, for profilers
(a profiling case kept beside the tests; pytest does not collect it).

    python tests/profile_case.py SCALE [ALPHA BETA [NROOTS]]

Generates and builds a Kronecker graph on the GPU (VERTEX_REORDERING 2), runs
the plain BFS from the first NROOTS find_roots roots with the given direction
thresholds, validates the last one on the device, and runs one multi-source
launch over 64 roots (lane width 64, alpha 6, no CUDA graph, so a profiler
sees each kernel launch).  It prints one line and exits 0.
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main(argv):
    import torch

    import graph500_b200 as g5
    scale = int(argv[1])
    alpha = float(argv[2]) if len(argv) > 2 else 2000.0
    beta = float(argv[3]) if len(argv) > 3 else 8.0
    nroots = int(argv[4]) if len(argv) > 4 else 3
    bfs = g5.BfsOnGPU()
    bfs.construct(g5.EdgeList(None, scale, 16))
    bfs.prepare_bfs(alpha, beta)
    roots = g5.find_roots(bfs.graph_, 64)
    pred = torch.empty(bfs.graph_.pred_size(), dtype=torch.int64, device="cuda")
    st = None
    for r in roots[:nroots]:
        st = bfs.run_bfs(int(r), pred)
    ok, evc, _ = g5.validate_bfs_result(bfs.graph_, int(roots[nroots - 1]), pred)
    ms = g5.MultiSourceBFS(bfs.graph_, 64, 6.0, False)
    ms.run(roots)
    torch.cuda.synchronize()
    ms.close()
    bfs.close()
    print(f"profile case SCALE {scale}: valid {ok}, edge_visit_count {evc}, last BFS {st.device_ms:.3f} ms")
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main(sys.argv))
