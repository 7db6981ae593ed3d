"""The main.cc-style driver (graph500_b200/g500_main, host C++ over the C ABI):
it builds, links against libg500.so and parses its arguments without a GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "graph500_b200", "g500_main")


@pytest.fixture(scope="module")
def driver(g500):
    assert os.path.exists(DRIVER), "g500_main is built with the library (python -m graph500_b200.build)"
    return DRIVER


def test_driver_usage(driver):
    r = subprocess.run([driver, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "usage: g500_main SCALE" in r.stderr


@pytest.mark.parametrize("args", [[], ["0"], ["12", "--roots", "65"], ["12", "--reorder", "3"]])
def test_driver_rejects_bad_arguments(driver, args):
    r = subprocess.run([driver] + args, capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def test_cpp_header_compiles(tmp_path):
    """include/g500_bfs.hpp (the BfsOnGPU class main.cc would use) compiles on its own."""
    src = tmp_path / "t.cc"
    src.write_text('#include "g500_bfs.hpp"\nint main(){g500cpp::BfsOnGPU b(2); (void)b; return 0;}\n')
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)], check=True,
                   env={k: v for k, v in os.environ.items() if k not in ("CC", "CXX")})


def _write_log(path, runs, scale=22, ef=16):
    """A resume file in the LogFileFormat layout (mpi/logfile.h:109-124)."""
    import struct
    data = struct.pack("<4i3d", scale, ef, 1, len(runs), 1.25, 20.5, 0.0)
    for t, v, e in runs:
        data += struct.pack("<ddq", t, v, e)
    data += b"\0" * (24 * (64 - len(runs)))
    with open(path, "wb") as f:
        f.write(data)


def _block(text):
    """The statistics lines of a result block (min_time .. stddev_validate)."""
    lines = [ln for ln in text.splitlines() if ":" in ln]
    names = [ln.split(":")[0] for ln in lines]
    i = names.index("min_time")
    return lines[i:i + 28]


@pytest.mark.parametrize("n", [64, 16, 7])
def test_result_block_matches_reference(driver, oracle_mod, tmp_path, n):
    """The driver's result block, printed from fixed run times and edge counts
    (--print-result), is character for character the reference's
    print_bfs_result (logfile.h:49-107) on the same runs, and its harmonic mean
    equals the oracle's restated statistics."""
    import json
    import sys
    import numpy as np
    if not oracle_mod.ref_available(0):
        pytest.skip("the reference was not compiled (oracle/_ref)")
    rng = np.random.default_rng(n)
    bfs = (rng.random(n) * 1e-3 + 1e-4).round(9)
    bfs[n // 3] = bfs[n // 2]  # a tie
    val = rng.random(n) * 0.05
    edges = np.full(n, 67108130, dtype=np.int64)
    edges[::5] = 67108130 - rng.integers(0, 1000, len(edges[::5]))
    runs = list(zip(bfs.tolist(), val.tolist(), edges.tolist()))
    log = tmp_path / "log.bin"
    _write_log(str(log), runs)
    ours = subprocess.run([driver, "--print-result", str(log)], capture_output=True, text=True)
    assert ours.returncode == 0, ours.stderr
    child = (
        "import ctypes as C, json, sys\n"
        f"L = C.CDLL({os.path.join(ROOT, 'oracle', '_ref', 'libg500ref_vr0.so')!r})\n"
        "b, v, e = json.loads(sys.stdin.read())\n"
        "D = C.c_double * len(b)\n"
        "L.ref_print_bfs_result(len(b), D(*b), D(*v), D(*[float(x) for x in e]), 1)\n")
    ref = subprocess.run([sys.executable, "-c", child], input=json.dumps([bfs.tolist(), val.tolist(), edges.tolist()]),
                         capture_output=True, text=True, env=dict(os.environ, NO_AFFINITY="1"))
    assert ref.returncode == 0, ref.stderr
    assert _block(ours.stdout) == _block(ref.stdout)
    hm = [ln for ln in _block(ours.stdout) if ln.startswith("harmonic_mean_TEPS")][0]
    st = oracle_mod.statistics(bfs / edges)
    assert abs(float(hm.split(":")[1]) - 1.0 / st["mean"]) <= 1e-9 * (1.0 / st["mean"])
