"""The C-ABI library loads, exports every symbol include/g500.h declares, and
its host-side pieces agree with the oracle.  No GPU needed."""
import ctypes
import os
import subprocess

import pytest

from conftest import HAS_GPU, ROOT


def test_library_loads_and_exports_header_symbols(g500):
    names = g500.header_functions()
    assert len(names) >= 20
    L = g500.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.g500_abi_version() == 1


def test_symbols_are_plain_c(g500):
    """Exported g500_* names are unmangled C symbols."""
    out = subprocess.run(["nm", "-D", "--defined-only", g500.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    for n in g500.header_functions():
        assert n in exported, n


def test_struct_layout_matches_header(g500, tmp_path):
    """ctypes mirrors have the sizes the C compiler gives the header's structs."""
    src = tmp_path / "sz.c"
    src.write_text('#include "g500.h"\n#include <stdio.h>\nint main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
                   'sizeof(g500_graph_info),sizeof(g500_level_stats),sizeof(g500_bfs_stats),'
                   'sizeof(g500_validate_report),sizeof(g500_packed_edge),sizeof(g500_tune_result),'
                   'sizeof(g500_msbfs_stats),sizeof(g500_msbfs_tune),sizeof(g500_msbfs_level),'
                   'sizeof(g500_server_config),sizeof(g500_query_result),sizeof(g500_server_info_t),'
                   'sizeof(g500_serve_report));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True,
                   env={k: v for k, v in os.environ.items() if k not in ("CC", "CXX")})
    sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert sizes == [ctypes.sizeof(g500.GraphInfo), ctypes.sizeof(g500.LevelStats), ctypes.sizeof(g500.BfsStats),
                     ctypes.sizeof(g500.ValidateReport), g500.EDGE_DTYPE.itemsize, ctypes.sizeof(g500.TuneResult),
                     ctypes.sizeof(g500.MsStats), ctypes.sizeof(g500.MsTune), ctypes.sizeof(g500.MsLevel),
                     ctypes.sizeof(g500.ServerConfig), ctypes.sizeof(g500.QueryResult), ctypes.sizeof(g500.ServerInfo),
                     ctypes.sizeof(g500.ServeReport)]


def test_scramble_values_match_oracle(g500, oracle_mod):
    for s in (10, 16, 26):
        assert g500.scramble_values(s) == oracle_mod.scramble_values(s)
    assert g500.scramble_values(20, 7, 11) == oracle_mod.scramble_values(20, 7, 11)


def test_invalid_arguments_return_status(g500):
    L = g500.lib()
    assert L.g500_graph_info_get(None, None) == g500.G500_E_INVAL
    assert b"null" in L.g500_last_error()
    assert L.g500_gen_edges(0, 16, 2, 3, 0, 10, None, 1, None) == g500.G500_E_INVAL
    assert L.g500_gen_edges(10, 16, 2, 3, 0, (1 << 10) * 16 + 1, None, 1, None) == g500.G500_E_RANGE
    assert L.g500_bfs_run(None, 0, None, 0, None) == g500.G500_E_INVAL
    for setter in (L.g500_bfs_set_pred_mode, L.g500_bfs_set_host_pack, L.g500_bfs_set_grid):
        assert setter(None, 0) == g500.G500_E_INVAL


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device error path")
def test_no_device_fails_loudly(g500):
    """Without a GPU the library reports a device error; it never falls back to the CPU."""
    with pytest.raises(g500.G500Error) as ei:
        g500.Graph2DCSR.generate(10)
    assert ei.value.code in (g500.G500_E_DEVICE, g500.G500_E_NOMEM)


def test_product_does_not_reference_oracle():
    """The CUDA library and the package never load the checker."""
    pkg = os.path.join(ROOT, "graph500_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp", ".cc")):
                text = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in text and "liboracle" not in text and "g500_oracle" not in text, f


class _FakeCudaArray:
    """An object exposing __cuda_array_interface__ (no GPU memory behind it)."""

    def __init__(self, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (0, False), "version": 3,
                                         "strides": None}


def test_edge_count_comes_from_byte_size(g500):
    """A 3*m int32 device buffer holds m packed edges, not 3*m."""
    assert g500._num_edges(_FakeCudaArray((30,), "<i4")) == 10
    assert g500._num_edges(_FakeCudaArray((5, 3), "<u4")) == 5
    import numpy as np
    assert g500._num_edges(np.zeros(7, g500.EDGE_DTYPE)) == 7
    with pytest.raises(ValueError):
        g500._num_edges(_FakeCudaArray((31,), "<i4"))
