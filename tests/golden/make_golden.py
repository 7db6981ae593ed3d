"""Generate the golden fixtures of tests/golden/ from the UNMODIFIED reference.

Runs the reference CPU path (suzumura/graph500, compiled here by
oracle/Makefile against a single-rank MPI stand-in) through oracle.Reference
and stores, per (SCALE, VERTEX_REORDERING) case:
  - a digest of the whole generated edge list plus its first/last 64 edges,
  - the graph scalars (graph_constructor.hpp), the find_roots roots,
  - per root: edge_visit_count, a digest of the level array ((pred>>48)&0xFFFF),
    the level histogram, and for two roots the full level array,
  - one reference predecessor array (SCALE 12, VR 0, first root).
The benchmark sizes (SCALE 22 and 24, VR 2, the 64 find_roots roots) keep the
per-root records only: no full level arrays, and the reference validator runs
on the first VALIDATE_LARGE roots (every root's edge_visit_count still comes
from it for those; the rest carry the reached count from the level histogram).
pf_nedge.json restates the reference's known-answer table pf_nedge[]
(mpi/utils.hpp:3663-3707, edgefactor 16, seeds 2/3).

Each (SCALE, VR) case runs in its own process because the reference keeps
global state.  Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASES = [(10, 0, 16), (12, 0, 16), (12, 2, 16), (16, 0, 16), (16, 2, 16), (18, 2, 8)]
# the benchmark sizes (Kronecker SCALE 22 and 24, edgefactor 16, VR 2, 64 roots)
LARGE_CASES = [(22, 2, 64), (24, 2, 64)]
VALIDATE_LARGE = 64

# mpi/utils.hpp:3663-3699: expected traversed edges for edgefactor 16, seeds (2, 3)
PF_NEDGE = [-1, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16383, 32767, 65535, 131070, 262144, 524285,
            1048570, 2097137, 4194250, 8388513, 16776976, 33553998, 67108130, 134216177, 268432547, 536865258,
            1073731075, 2147462776, 4294927670, 8589858508, 17179724952, 34359466407, 68718955183, 137437972330,
            274876029861, 549752273512, 1099505021204]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def one_case(scale: int, vr: int, nroots: int) -> None:
    import oracle as O
    large = scale >= 20
    ref = O.Reference(vr)
    ref.generate(scale, 16)
    edges = ref.edges()
    ref.construct()
    roots = ref.find_roots(nroots)
    ref.prepare_bfs()
    rec = {"scale": scale, "vr": vr, "info": ref.info, "roots": roots.tolist(), "num_edges": len(edges),
           "edges_sha256": digest(edges), "per_root": []}
    head, tail = edges[:64].copy(), edges[-64:].copy()
    if large:
        del edges
    full = {}
    for i, r in enumerate(roots):
        pred, t = ref.run_bfs(int(r))
        entry = {"root": int(r)}
        if not large or i < VALIDATE_LARGE:
            ok, evc = ref.validate(int(r), pred)
            assert ok, (scale, vr, r)
            entry["edge_visit_count"] = evc
        lv = ((pred >> 48) & 0xFFFF).astype(np.uint16)
        lv[pred == -1] = 0xFFFF
        hist = np.bincount(np.where(lv == 0xFFFF, 0, lv.astype(np.int64) + 1)).tolist()
        entry.update({"levels_sha256": digest(lv), "level_hist": hist})
        rec["per_root"].append(entry)
        if large:
            print(f"SCALE {scale} root {i} {int(r)} bfs {t:.3f}s", file=sys.stderr, flush=True)
        elif i < 2:
            full[f"levels_{i}"] = lv
        if scale == 12 and vr == 0 and i == 0:
            full["pred_0"] = pred
    name = f"ref_s{scale}_vr{vr}"
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(rec, f, indent=1)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), edges_head=head, edges_tail=tail, **full)
    print("wrote", name, file=sys.stderr)


# spec-2012 generator fixtures (generate_graph_spec2012, benchmark_helper.hpp:316-322)
SPEC2012_SCALES = [4, 10, 12, 16]


def spec2012_case(scale: int) -> None:
    import oracle as O
    ref = O.Reference(0)
    e = ref.generate_spec2012(scale, 16)
    # the digest covers the endpoints (the first 12 bytes of each 16-byte
    # WeightedEdge).  The reference's weights are racy: generateWeight's
    # per-thread loop (graph_generator.hpp:488-503) has no barrier before the
    # master thread copies the chunk out (benchmark_helper.hpp:270-284, the
    # barrier is compiled for the Intel compiler only), so a weight is 0xBEEF or
    # whatever the chunk buffer held; the count of 0xBEEF weights is recorded
    ends = np.ascontiguousarray(e.view(np.uint32).reshape(-1, 4)[:, :3])
    rec = {"scale": scale, "edgefactor": 16, "num_edges": len(e), "endpoints_sha256": digest(ends),
           "weights_0xBEEF": int((e["weight"] == 0xBEEF).sum())}
    name = f"ref_spec2012_s{scale}"
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(rec, f, indent=1)
    n = 1 << scale
    np.savez_compressed(os.path.join(HERE, name + ".npz"), edges_head=e[:64], edges_tail=e[-64:],
                        edges_tree_end=e[n - 33:n + 31])
    print("wrote", name, file=sys.stderr)


def main() -> None:
    """No arguments: the small cases.  ``--large``: the benchmark sizes (minutes
    of reference construction and validation each).  ``--spec2012``: the
    spec-2012 generator's edge lists.  ``SCALE VR NROOTS``: one case."""
    if len(sys.argv) == 4:
        one_case(int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]))
        return
    if sys.argv[1:2] == ["--spec2012"]:
        if len(sys.argv) == 3:
            spec2012_case(int(sys.argv[2]))
            return
        for scale in SPEC2012_SCALES:
            subprocess.run([sys.executable, __file__, "--spec2012", str(scale)], check=True,
                           env=dict(os.environ, NO_AFFINITY="1"), stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL)
        return
    if sys.argv[1:] == ["--large"]:
        env = dict(os.environ, NO_AFFINITY="1")
        for scale, vr, nroots in LARGE_CASES:
            subprocess.run([sys.executable, __file__, str(scale), str(vr), str(nroots)], check=True, env=env,
                           stdout=subprocess.DEVNULL)
        return
    with open(os.path.join(HERE, "pf_nedge.json"), "w") as f:
        json.dump({"source": "mpi/utils.hpp:3663-3707 (edgefactor 16, seeds 2/3)", "pf_nedge": PF_NEDGE}, f,
                  indent=1)
    env = dict(os.environ, NO_AFFINITY="1")
    for scale, vr, nroots in CASES:
        subprocess.run([sys.executable, __file__, str(scale), str(vr), str(nroots)], check=True, env=env,
                       stdout=subprocess.DEVNULL)


if __name__ == "__main__":
    main()
