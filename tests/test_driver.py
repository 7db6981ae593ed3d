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
