import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA library")
    config.addinivalue_line("markers", "slow: large-scale case (SCALE >= 20)")


def _gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _gpu_available()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def load_golden(scale: int, vr: int):
    with open(os.path.join(GOLDEN, f"ref_s{scale}_vr{vr}.json")) as f:
        rec = json.load(f)
    arrays = dict(np.load(os.path.join(GOLDEN, f"ref_s{scale}_vr{vr}.npz")))
    return rec, arrays


def pf_nedge() -> list:
    with open(os.path.join(GOLDEN, "pf_nedge.json")) as f:
        return json.load(f)["pf_nedge"]


GOLDEN_CASES = [(10, 0), (12, 0), (12, 2), (16, 0), (16, 2), (18, 2)]


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def g500():
    import graph500_b200
    graph500_b200.lib()
    return graph500_b200


# the benchmark sizes, pinned by per-root records of the unmodified reference
# (tests/golden/make_golden.py --large)
LARGE_GOLDEN_CASES = [(22, 2), (24, 2)]


def load_golden_record(scale: int, vr: int):
    with open(os.path.join(GOLDEN, f"ref_s{scale}_vr{vr}.json")) as f:
        return json.load(f)
