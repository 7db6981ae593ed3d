"""ctypes bindings for the checker: the C restatement (liboracle.so) and, when
it was built, the unmodified reference CPU path (``_ref/libg500ref_vrN.so``).

TEST INFRASTRUCTURE.  Only tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of bench.py import this package; the CUDA product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
USERSEED1, USERSEED2 = 2, 3  # mpi/parameters.h:190-191
EDGE_DTYPE = np.dtype([("v0_low", "<u4"), ("v1_low", "<u4"), ("high", "<u4")])
WEDGE_DTYPE = np.dtype([("v0_low", "<u4"), ("v1_low", "<u4"), ("high", "<u4"), ("weight", "<i4")])

INFO_NAMES = ("log_orig_global_verts", "pred_size", "num_local_verts",
              "num_global_verts", "num_global_edges", "max_used_vertex")

_lib = None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference tree is present)."""
    targets = ["oracle"]
    if os.path.isdir(os.environ.get("G500_REFERENCE", "/root/reference")):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, "-j8"] + targets, check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.c_void_p
        i64, u64, i32 = C.c_int64, C.c_uint64, C.c_int
        L.orc_generate_edges.argtypes = [i32, i32, u64, u64, i64, i64, P]
        L.orc_generate_edges_spec2012.argtypes = [i32, i32, u64, u64, i64, i64, P]
        L.orc_scramble_values.argtypes = [i32, u64, u64, P, P]
        L.orc_make_random_numbers.argtypes = [i64, u64, u64, i64, P]
        L.orc_mrg_skip_matrix.argtypes = [i32, i32, P]
        L.orc_graph_build.argtypes = [P, i64, i32]
        L.orc_graph_build.restype = P
        L.orc_graph_free.argtypes = [P]
        L.orc_graph_info.argtypes = [P, P]
        for f in ("orc_graph_offsets", "orc_graph_cols", "orc_graph_reorder_map",
                  "orc_graph_invert_map", "orc_graph_degree"):
            getattr(L, f).argtypes = [P]
            getattr(L, f).restype = P
        L.orc_graph_has_edge.argtypes = [P, i64]
        L.orc_find_roots.argtypes = [P, i32, u64, u64, P]
        L.orc_find_max_used_vertex.argtypes = [P]
        L.orc_find_max_used_vertex.restype = i64
        L.orc_bfs_levels.argtypes = [P, i64, P]
        L.orc_bfs_pred.argtypes = [P, i64, P]
        L.orc_dobfs_schedule.argtypes = [P, i64, C.c_double, C.c_double, P, i32]
        L.orc_validate.argtypes = [P, i64, i64, i64, i64, P, P, P]
        L.orc_statistics.argtypes = [P, i32, P]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def generate_edges(scale: int, edgefactor: int = 16, start: int = 0, end: int | None = None,
                   seed1: int = USERSEED1, seed2: int = USERSEED2) -> np.ndarray:
    """Packed 12-byte edges [start, end) (generator/graph_generator.hpp:612-627)."""
    if end is None:
        end = (1 << scale) * edgefactor
    out = np.zeros(end - start, dtype=EDGE_DTYPE)
    lib().orc_generate_edges(scale, edgefactor, seed1, seed2, start, end, _p(out))
    return out


def generate_edges_spec2012(scale: int, edgefactor: int = 16, start: int = 0, end: int | None = None,
                            seed1: int = USERSEED1, seed2: int = USERSEED2) -> np.ndarray:
    """Weighted edges [start, end) of generate_graph_spec2012
    (mpi/benchmark_helper.hpp:316-322): N - 1 binary-tree edges, then R-MAT
    edges with A = .55, B = C = .01; weight 0xBEEF."""
    n = 1 << scale
    if end is None:
        end = n * edgefactor + n - 1
    out = np.zeros(end - start, dtype=WEDGE_DTYPE)
    lib().orc_generate_edges_spec2012(scale, edgefactor, seed1, seed2, start, end, _p(out))
    return out


def edge_endpoints(edges: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(v0, v1) int64 arrays of packed edges (mpi/primitives.hpp:61-62)."""
    hi = edges["high"].astype(np.int64)
    v0 = edges["v0_low"].astype(np.int64) | ((hi & 0xFFFF) << 32)
    v1 = edges["v1_low"].astype(np.int64) | ((hi >> 16) << 32)
    return v0, v1


def scramble_values(scale: int, seed1: int = USERSEED1, seed2: int = USERSEED2) -> tuple[int, int]:
    a, b = np.zeros(1, np.uint64), np.zeros(1, np.uint64)
    lib().orc_scramble_values(scale, seed1, seed2, _p(a), _p(b))
    return int(a[0]), int(b[0])


def skip_matrix(byte_index: int, val: int) -> np.ndarray:
    out = np.zeros(25, np.uint32)
    lib().orc_mrg_skip_matrix(byte_index, val, _p(out))
    return out.reshape(5, 5)


def random_numbers(n: int, position: int, seed1: int = USERSEED1, seed2: int = USERSEED2) -> np.ndarray:
    out = np.zeros(n, np.float64)
    lib().orc_make_random_numbers(n, seed1, seed2, position, _p(out))
    return out


class Graph:
    """One-rank CSR restated from mpi/graph_constructor.hpp."""

    def __init__(self, edges: np.ndarray, reorder_mode: int):
        self._edges = np.ascontiguousarray(edges)
        self.h = lib().orc_graph_build(_p(self._edges), len(self._edges), reorder_mode)
        info = np.zeros(6, np.int64)
        lib().orc_graph_info(self.h, _p(info))
        self.info = dict(zip(INFO_NAMES, (int(x) for x in info)))
        nlv, nolv = self.info["num_local_verts"], self.info["pred_size"]
        ne = self.info["num_global_edges"]

        def view(fn, dtype, n):
            ptr = getattr(lib(), fn)(self.h)
            if n == 0:
                return np.zeros(0, dtype)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))), (n,))

        self.offsets = view("orc_graph_offsets", np.uint64, nlv + 1)
        self.cols = view("orc_graph_cols", np.uint32, ne)
        self.reorder_map = view("orc_graph_reorder_map", np.uint32, nolv)
        self.invert_map = view("orc_graph_invert_map", np.uint32, nolv)
        self.degree = view("orc_graph_degree", np.int64, nolv)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_graph_free(self.h)
            self.h = None

    def has_edge(self, v: int) -> bool:
        return bool(lib().orc_graph_has_edge(self.h, v))

    def find_roots(self, n: int, seed1: int = USERSEED1, seed2: int = USERSEED2) -> np.ndarray:
        out = np.zeros(n, np.int64)
        k = lib().orc_find_roots(self.h, n, seed1, seed2, _p(out))
        return out[:k]

    def bfs_levels(self, root: int) -> np.ndarray:
        out = np.zeros(self.info["pred_size"], np.uint16)
        lib().orc_bfs_levels(self.h, root, _p(out))
        return out

    def bfs_pred(self, root: int) -> np.ndarray:
        out = np.zeros(self.info["pred_size"], np.int64)
        lib().orc_bfs_pred(self.h, root, _p(out))
        return out

    def dobfs_schedule(self, root: int, alpha: float = 2000.0, beta: float = 8.0) -> np.ndarray:
        dt = np.dtype([("direction", "<i4"), ("pad", "<i4"), ("frontier", "<i8"), ("discovered", "<i8"),
                       ("scanned", "<i8"), ("edge_sectors", "<i8"), ("edges_examined", "<i8")])
        out = np.zeros(512, dt)
        n = lib().orc_dobfs_schedule(self.h, root, alpha, beta, _p(out), 512)
        return out[:n]


def validate(edges: np.ndarray, nglobalverts: int, nlocalverts: int, root: int,
             pred: np.ndarray) -> tuple[bool, int, dict]:
    """validate.hpp:506-802 on one rank -> (ok, edge_visit_count, error counts)."""
    edges = np.ascontiguousarray(edges)
    pred = np.ascontiguousarray(pred, dtype=np.int64)
    evc = np.zeros(1, np.int64)
    rep = np.zeros(6, np.int64)
    ok = lib().orc_validate(_p(edges), len(edges), nglobalverts, nlocalverts, root, _p(pred),
                            _p(evc), _p(rep))
    names = ("range", "root", "self_parent", "depth", "edge", "missing_parent_edge")
    return bool(ok), int(evc[0]), dict(zip(names, (int(x) for x in rep)))


def statistics(x) -> dict:
    """get_statistics (mpi/logfile.h:19-44)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    r = np.zeros(7, np.float64)
    lib().orc_statistics(_p(x), len(x), _p(r))
    return dict(zip(("min", "q1", "median", "q3", "max", "mean", "std"), (float(v) for v in r)))


# ---------------------------------------------------------------------------
# the unmodified reference, compiled here (oracle/_ref)
# ---------------------------------------------------------------------------

def ref_available(reorder_mode: int) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libg500ref_vr{reorder_mode}.so"))


class Reference:
    """The reference CPU path (mpi/main.cc call sequence) through ref_driver.cc.

    One instance per process and reordering mode: the reference keeps global
    MPI/graph state.
    """

    def __init__(self, reorder_mode: int):
        os.environ.setdefault("NO_AFFINITY", "1")
        L = C.CDLL(os.path.join(REF_DIR, f"libg500ref_vr{reorder_mode}.so"))
        P, i64, i32 = C.c_void_p, C.c_int64, C.c_int
        L.ref_generate.argtypes = [i32, i32]
        L.ref_generate.restype = C.c_double
        L.ref_copy_edges.argtypes = [P, i64, i64]
        L.ref_copy_edges.restype = i64
        L.ref_construct.restype = C.c_double
        L.ref_graph_info.argtypes = [P]
        L.ref_has_edge.argtypes = [i64]
        L.ref_find_roots.argtypes = [i32, P]
        L.ref_run_bfs.argtypes = [i64, P]
        L.ref_run_bfs.restype = C.c_double
        L.ref_validate.argtypes = [i64, P, P]
        self.L = L
        self.reorder_mode = reorder_mode

    def generate(self, scale: int, edgefactor: int = 16) -> float:
        self.scale, self.edgefactor = scale, edgefactor
        return self.L.ref_generate(scale, edgefactor)

    def generate_spec2012(self, scale: int, edgefactor: int = 16) -> np.ndarray:
        """The reference's generate_graph_spec2012 edge list (weighted, 16 bytes per edge)."""
        L = self.L
        L.ref_generate_spec2012.argtypes = [C.c_int, C.c_int]
        L.ref_generate_spec2012.restype = C.c_int64
        L.ref_copy_edges_spec2012.argtypes = [C.c_void_p, C.c_int64, C.c_int64]
        L.ref_copy_edges_spec2012.restype = C.c_int64
        n = L.ref_generate_spec2012(scale, edgefactor)
        out = np.zeros(n, WEDGE_DTYPE)
        got = L.ref_copy_edges_spec2012(_p(out), 0, n)
        return out[:got]

    def edges(self, start: int = 0, count: int | None = None) -> np.ndarray:
        if count is None:
            count = (1 << self.scale) * self.edgefactor - start
        out = np.zeros(count, EDGE_DTYPE)
        n = self.L.ref_copy_edges(_p(out), start, count)
        return out[:n]

    def construct(self) -> float:
        t = self.L.ref_construct()
        info = np.zeros(6, np.int64)
        self.L.ref_graph_info(_p(info))
        self.info = dict(zip(INFO_NAMES, (int(x) for x in info)))
        return t

    def find_roots(self, n: int) -> np.ndarray:
        out = np.zeros(n, np.int64)
        k = self.L.ref_find_roots(n, _p(out))
        return out[:k]

    def prepare_bfs(self) -> None:
        self.L.ref_prepare_bfs()

    def run_bfs(self, root: int) -> tuple[np.ndarray, float]:
        pred = np.zeros(self.info["pred_size"], np.int64)
        t = self.L.ref_run_bfs(root, _p(pred))
        return pred, t

    def validate(self, root: int, pred: np.ndarray) -> tuple[bool, int]:
        evc = np.zeros(1, np.int64)
        p = np.ascontiguousarray(pred, dtype=np.int64).copy()
        ok = self.L.ref_validate(root, _p(p), _p(evc))
        return bool(ok), int(evc[0])

    def end_bfs(self) -> None:
        self.L.ref_end_bfs()
