"""Child process of tests/test_gpu_reference_pinned.py: runs the unmodified
reference's validate_bfs_result (mpi/validate.hpp:1008-1019, through
oracle/ref_driver.cc ref_validate) on parent arrays read from an .npz file.

  python tests/_ref_validate.py SCALE VR PREDS.npz

Each key of the .npz is "m<mode>_r<root>"; the result is one JSON object
{key: [ok, edge_visit_count]} on stdout.  The reference keeps global MPI and
graph state, hence one process per (SCALE, VR).  Uses no GPU.
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import oracle  # noqa: E402


def main() -> None:
    scale, vr, path = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3]
    ref = oracle.Reference(vr)
    ref.generate(scale, 16)
    ref.construct()
    out = {}
    with np.load(path) as preds:
        for key in preds.files:
            root = int(key.split("_r")[1])
            ok, evc = ref.validate(root, preds[key])
            out[key] = [ok, evc]
    print(json.dumps(out))


if __name__ == "__main__":
    main()
