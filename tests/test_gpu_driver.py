"""The main.cc-style driver end to end on the GPU: the Graph500 result block,
validation of every root, and the LOGFILE resume log (an interrupted run
resumes at its first unfinished root; a log of another run is refused)."""
import os
import re
import struct
import subprocess

import pytest

from conftest import pf_nedge

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "graph500_b200", "g500_main")
LOG_FORMAT = "<iiiiddd" + "ddq" * 64  # LogFileFormat (logfile.h:109-124)


def run(args, logfile=None):
    env = dict(os.environ)
    env.pop("LOGFILE", None)
    if logfile:
        env["LOGFILE"] = str(logfile)
    return subprocess.run([DRIVER] + [str(a) for a in args], capture_output=True, text=True, env=env, timeout=300)


def result_block(out):
    block = out.split("============= Result ==============")[1]
    return {m.group(1): float(m.group(2)) for m in re.finditer(r"^(\w+):\s+(\S+)$", block, re.M)}


def test_driver_result_block(g500):
    r = run([12, "--roots", 8])
    assert r.returncode == 0, r.stderr
    res = result_block(r.stdout)
    assert res["SCALE"] == 12 and res["edgefactor"] == 16 and res["NBFS"] == 8
    want = pf_nedge()[12]
    assert res["min_nedge"] == res["max_nedge"] == want
    teps = [float(x) for x in re.findall(r"TEPS for BFS \d+ is (\S+)", r.stdout)]
    assert len(teps) == 8
    hm = len(teps) / sum(1.0 / t for t in teps)
    assert abs(res["harmonic_mean_TEPS"] / hm - 1) < 1e-3
    assert res["min_time"] <= res["median_time"] <= res["max_time"]


def test_driver_resume_log(g500, tmp_path):
    log = tmp_path / "g500.log"
    r = run([12, "--roots", 8, "--max-runs", 3], logfile=log)
    assert r.returncode == 0 and "stopped after 3 of 8" in r.stdout, r.stdout + r.stderr
    raw = log.read_bytes()
    assert len(raw) == struct.calcsize(LOG_FORMAT)
    f = struct.unpack(LOG_FORMAT, raw)
    assert f[:4] == (12, 16, 1, 3)
    r = run([12, "--roots", 8], logfile=log)
    assert r.returncode == 0, r.stderr
    assert "Resume from 3 th run" in r.stdout
    assert "Running BFS 2 " not in r.stdout and "Running BFS 3 " in r.stdout
    res = result_block(r.stdout)
    assert res["NBFS"] == 8 and res["min_nedge"] == res["max_nedge"] == pf_nedge()[12]
    assert struct.unpack(LOG_FORMAT, log.read_bytes())[3] == 8
    # a log of another run is refused, as the reference does
    r = run([13, "--roots", 8], logfile=log)
    assert r.returncode == 1 and "Log file is not match" in r.stderr
