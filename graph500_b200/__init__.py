"""graph500_b200 -- B200-native Graph500 BFS behind the reference's BfsBase interface.

Python mirror of the suzumura/graph500 driver-facing API (mpi/main.cc and
mpi/bfs.hpp), bound to libg500.so through its C ABI (include/g500.h):

    edge_list = generate_graph_spec2010(SCALE, edgefactor)      # benchmark_helper.hpp:308
    bfs = BfsOnGPU(); bfs.construct(edge_list)                   # bfs.hpp:102
    roots = find_roots(bfs.graph_, 64)                           # benchmark_helper.hpp:475
    bfs.prepare_bfs()                                            # bfs.hpp:115
    bfs.run_bfs(root, pred)                                      # bfs.hpp:120
    ok, nedge = validate_bfs_result(edge_list, max_used_vertex(bfs.graph_) + 1,
                                    bfs.graph_.pred_size(), root, pred)   # validate.hpp:1008
    bfs.end_bfs()                                                # bfs.hpp:126

There is no CPU fallback: every call runs the CUDA library, and importing a
function whose library is missing raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libg500.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "g500.h")
USERSEED1, USERSEED2 = 2, 3  # mpi/parameters.h:190-191
EDGE_DTYPE = np.dtype([("v0_low", "<u4"), ("v1_low", "<u4"), ("high", "<u4")])
WEDGE_DTYPE = np.dtype([("v0_low", "<u4"), ("v1_low", "<u4"), ("high", "<u4"), ("weight", "<i4")])

(G500_OK, G500_E_INVAL, G500_E_NOMEM, G500_E_DEVICE, G500_E_TIMEOUT, G500_E_RANGE, G500_E_STATE,
 G500_E_VALIDATION, G500_E_IO) = range(9)


class G500Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[g500 status {code}] {msg}")
        self.code = code


class GraphInfo(C.Structure):
    _fields_ = [("log_orig_global_verts", C.c_int64), ("pred_size", C.c_int64), ("num_local_verts", C.c_int64),
                ("num_global_verts", C.c_int64), ("num_global_edges", C.c_int64), ("max_used_vertex", C.c_int64),
                ("num_input_edges", C.c_int64), ("device_bytes", C.c_int64), ("reorder_mode", C.c_int32),
                ("device", C.c_int32)]


class LevelStats(C.Structure):
    _fields_ = [("direction", C.c_int32), ("level", C.c_int32), ("frontier", C.c_int64),
                ("discovered", C.c_int64), ("scanned", C.c_int64), ("edge_sectors", C.c_int64),
                ("edges_examined", C.c_int64), ("device_ms", C.c_double),
                ("device_ms_tail", C.c_double)]


class BfsStats(C.Structure):
    _fields_ = [("device_ms", C.c_double), ("host_ms", C.c_double), ("reached", C.c_int64), ("nedge", C.c_int64),
                ("num_levels", C.c_int32), ("td_levels", C.c_int32), ("bu_levels", C.c_int32),
                ("kernel_launches", C.c_int32), ("init_ms", C.c_double), ("search_ms", C.c_double)]


class TuneResult(C.Structure):
    _fields_ = [("policy", C.c_int32), ("configs_tried", C.c_int32), ("alpha", C.c_double), ("beta", C.c_double),
                ("best_ms", C.c_double), ("reference_ms", C.c_double)]


DIR_REFERENCE, DIR_EDGES = 0, 1


class MsStats(C.Structure):
    _fields_ = [("device_ms", C.c_double), ("host_ms", C.c_double), ("num_levels", C.c_int32),
                ("pull_levels", C.c_int32), ("lane_width", C.c_int32), ("batches", C.c_int32),
                ("kernel_launches", C.c_int32), ("pad", C.c_int32), ("init_ms", C.c_double),
                ("search_ms", C.c_double)]


class MsTune(C.Structure):
    _fields_ = [("lane_width", C.c_int32), ("configs_tried", C.c_int32), ("alpha", C.c_double),
                ("best_ms", C.c_double)]


class MsLevel(C.Structure):
    _fields_ = [("level", C.c_int32), ("pull", C.c_int32), ("discovered", C.c_int64), ("device_ms", C.c_double),
                ("expand_ms", C.c_double), ("rows_read", C.c_int64), ("sectors", C.c_int64)]


class ServerConfig(C.Structure):
    _fields_ = [("max_batch", C.c_int32), ("max_workers_per_graph", C.c_int32), ("mode", C.c_int32),
                ("vertices_per_block", C.c_int32), ("hbm_reserve_bytes", C.c_uint64), ("alpha", C.c_double),
                ("max_grid_fraction", C.c_double), ("plain_below", C.c_int32), ("batch_target", C.c_int32)]


class QueryResult(C.Structure):
    _fields_ = [("id", C.c_int64), ("tag", C.c_uint64), ("graph", C.c_int32), ("status", C.c_int32),
                ("root", C.c_int64), ("reached", C.c_int64), ("nedge", C.c_int64), ("arrival_us", C.c_double),
                ("start_us", C.c_double), ("done_us", C.c_double), ("batch_size", C.c_int32),
                ("lane_width", C.c_int32)]


class ServerInfo(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("finished", C.c_int64), ("launches", C.c_int64),
                ("queries_launched", C.c_int64), ("workers", C.c_int32), ("max_in_flight", C.c_int32),
                ("block_capacity", C.c_int32), ("pad", C.c_int32)]


class ServeReport(C.Structure):
    _fields_ = [("rate_qps", C.c_double), ("queries", C.c_int64), ("failed", C.c_int64), ("wall_s", C.c_double),
                ("achieved_qps", C.c_double), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_ms", C.c_double), ("max_ms", C.c_double), ("gteps", C.c_double), ("nedge", C.c_int64),
                ("mean_batch", C.c_double), ("launches", C.c_int64), ("max_in_flight", C.c_int32),
                ("workers", C.c_int32), ("delivery", C.c_int32), ("pad", C.c_int32)]


SERVE_BATCHED, SERVE_PLAIN = 0, 1
DELIVER_NONE, DELIVER_DEVICE, DELIVER_HOST = 0, 1, 2


class ValidateReport(C.Structure):
    _fields_ = [("range_errors", C.c_int64), ("root_errors", C.c_int64), ("self_parent_errors", C.c_int64),
                ("depth_errors", C.c_int64), ("edge_errors", C.c_int64),
                ("missing_parent_edge_errors", C.c_int64)]


_lib = None


def header_functions() -> list[str]:
    """Names of the functions include/g500.h declares."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(g500_\w+)\s*\(", text, re.M)))


def lib() -> C.CDLL:
    """Load libg500.so (raise if it was not built: there is no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m graph500_b200.build`")
    L = C.CDLL(LIB_PATH)
    P, i64, u64, i32 = C.c_void_p, C.c_int64, C.c_uint64, C.c_int
    sig = {
        "g500_last_error": ([], C.c_char_p),
        "g500_abi_version": ([], i32),
        "g500_host_alloc": ([u64, C.POINTER(P)], i32),
        "g500_host_free": ([P], i32),
        "g500_scramble_values": ([i32, u64, u64, C.POINTER(u64), C.POINTER(u64)], i32),
        "g500_gen_edges": ([i32, i32, u64, u64, i64, i64, P, i32, P], i32),
        "g500_gen_edges_spec2012": ([i32, i32, u64, u64, i64, i64, P, i32, P], i32),
        "g500_graph_build": ([P, i64, i32, i32, i32, i32, C.POINTER(P)], i32),
        "g500_graph_generate": ([i32, i32, u64, u64, i32, i32, C.POINTER(P)], i32),
        "g500_graph_info_get": ([P, C.POINTER(GraphInfo)], i32),
        "g500_graph_has_edge": ([P, i64, C.POINTER(i32)], i32),
        "g500_graph_find_roots": ([P, i32, u64, u64, P, C.POINTER(i32)], i32),
        "g500_graph_edges": ([P, C.POINTER(P), C.POINTER(i64)], i32),
        "g500_graph_copy_csr": ([P, P, P, P], i32),
        "g500_graph_save": ([P, C.c_char_p], i32),
        "g500_graph_load": ([C.c_char_p, i32, C.POINTER(P)], i32),
        "g500_graph_timings": ([P, C.POINTER(C.c_double), C.POINTER(C.c_double)], i32),
        "g500_graph_destroy": ([P], i32),
        "g500_bfs_create": ([P, C.POINTER(P)], i32),
        "g500_bfs_set_params": ([P, C.c_double, C.c_double, i32], i32),
        "g500_bfs_set_stream": ([P, P], i32),
        "g500_bfs_set_pred_mode": ([P, i32], i32),
        "g500_bfs_set_host_pack": ([P, i32], i32),
        "g500_bfs_set_grid": ([P, i32], i32),
        "g500_bfs_set_policy": ([P, i32], i32),
        "g500_bfs_autotune": ([P, P, i32, i32, C.POINTER(TuneResult)], i32),
        "g500_bfs_run": ([P, i64, P, i32, C.POINTER(BfsStats)], i32),
        "g500_bfs_level_stats": ([P, P, i32, C.POINTER(i32)], i32),
        "g500_bfs_device_pred": ([P, C.POINTER(P)], i32),
        "g500_bfs_destroy": ([P], i32),
        "g500_validate": ([P, P, i64, i32, i64, P, i32, C.POINTER(i64), C.POINTER(i32), C.POINTER(ValidateReport)],
                          i32),
        "g500_msbfs_create": ([P, C.POINTER(P)], i32),
        "g500_msbfs_set_params": ([P, i32, C.c_double, i32], i32),
        "g500_msbfs_run": ([P, P, i32, P, i32, C.POINTER(MsStats)], i32),
        "g500_msbfs_root_stats": ([P, P, P], i32),
        "g500_msbfs_device_levels": ([P, C.POINTER(P)], i32),
        "g500_msbfs_level_info": ([P, i32, C.POINTER(MsLevel), i32, C.POINTER(i32)], i32),
        "g500_msbfs_launch": ([P, P, i32], i32),
        "g500_msbfs_poll": ([P, C.POINTER(i32)], i32),
        "g500_msbfs_wait": ([P, C.POINTER(MsStats)], i32),
        "g500_msbfs_set_root_stats": ([P, i32], i32),
        "g500_msbfs_set_grid": ([P, i32], i32),
        "g500_msbfs_set_sparse": ([P, i32, i64], i32),
        "g500_msbfs_set_count": ([P, i32], i32),
        "g500_msbfs_get_grid": ([P, i32, C.POINTER(i32), C.POINTER(i32)], i32),
        "g500_msbfs_workspace_bytes": ([P, C.POINTER(u64)], i32),
        "g500_selftest_barrier_timeout": ([i32, C.POINTER(i32), C.POINTER(i32)], i32),
        "g500_server_default_config": ([C.POINTER(ServerConfig)], i32),
        "g500_server_create": ([P, i32, C.POINTER(ServerConfig), C.POINTER(P)], i32),
        "g500_server_submit": ([P, i32, i64, u64, P, C.POINTER(i64)], i32),
        "g500_server_poll": ([P, C.POINTER(QueryResult), i32, C.POINTER(i32), i32], i32),
        "g500_server_drain": ([P, i32], i32),
        "g500_server_info": ([P, C.POINTER(ServerInfo)], i32),
        "g500_server_run_poisson": ([P, C.c_double, i64, u64, i64, C.POINTER(ServeReport)], i32),
        "g500_server_destroy": ([P], i32),
        "g500_server_set_delivery": ([P, i32], i32),
        "g500_msbfs_autotune": ([P, P, i32, i32, C.POINTER(MsTune)], i32),
        "g500_msbfs_destroy": ([P], i32),
        "g500_validate_noalloc": ([P, i64, i64, i64, i64, P, P, C.POINTER(i64), C.POINTER(i32),
                                   C.POINTER(ValidateReport)], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(status: int) -> None:
    if status != G500_OK:
        raise G500Error(status, lib().g500_last_error().decode(errors="replace"))


def _ptr(obj) -> tuple[int, bool]:
    """(address, on_device) of a numpy array or a CUDA array (e.g. a torch tensor)."""
    if isinstance(obj, np.ndarray):
        if not obj.flags.c_contiguous:
            raise ValueError("array must be C-contiguous")
        return obj.ctypes.data, False
    cai = getattr(obj, "__cuda_array_interface__", None)
    if cai is not None:
        if cai.get("strides") not in (None, ()):
            raise ValueError("CUDA array must be contiguous")
        return int(cai["data"][0]), True
    raise TypeError(f"unsupported buffer type {type(obj)!r}")


def _nbytes(obj) -> int:
    """Size in bytes of a numpy array or a contiguous CUDA array."""
    if isinstance(obj, np.ndarray):
        return obj.nbytes
    cai = obj.__cuda_array_interface__
    n = 1
    for d in cai["shape"]:
        n *= int(d)
    return n * int(np.dtype(cai["typestr"]).itemsize)


def _num_edges(edges) -> int:
    """Packed 12-byte edges held by a buffer (the count is derived from its
    byte size, never from its element count)."""
    nb = _nbytes(edges)
    if nb % EDGE_DTYPE.itemsize:
        raise ValueError(f"edge buffer of {nb} bytes is not a whole number of 12-byte packed edges")
    return nb // EDGE_DTYPE.itemsize


# ---------------------------------------------------------------------------
# (a) generation
# ---------------------------------------------------------------------------
class EdgeList:
    """The generated edge list (EdgeListStorage, generator/graph_generator.hpp:35-319).

    Host edges are a numpy array of 12-byte packed edges; a device-resident
    list belongs to a graph built by ``generate_graph_spec2010(..., device=True)``.
    """

    def __init__(self, edges: np.ndarray | None = None, scale: int | None = None, edgefactor: int = 16):
        self.edges = edges
        self.scale = scale
        self.edgefactor = edgefactor

    def num_local_edges(self) -> int:
        return len(self.edges) if self.edges is not None else (1 << self.scale) * self.edgefactor


def generate_edges(scale: int, edgefactor: int = 16, start: int = 0, end: int | None = None,
                   seed1: int = USERSEED1, seed2: int = USERSEED2, out=None):
    """Edges [start, end) of the spec-2010 Kronecker graph, generated on the GPU."""
    if end is None:
        end = (1 << scale) * edgefactor
    if out is None:
        out = np.zeros(end - start, dtype=EDGE_DTYPE)
    ptr, dev = _ptr(out)
    if _nbytes(out) < (end - start) * EDGE_DTYPE.itemsize:
        raise ValueError("output buffer too small for the requested edge range")
    check(lib().g500_gen_edges(scale, edgefactor, seed1, seed2, start, end, ptr, int(dev), None))
    return out


def generate_edges_spec2012(scale: int, edgefactor: int = 16, start: int = 0, end: int | None = None,
                            seed1: int = USERSEED1, seed2: int = USERSEED2, out=None):
    """Weighted edges [start, end) of generate_graph_spec2012
    (mpi/benchmark_helper.hpp:316-322), generated on the GPU: 2^scale - 1
    binary-tree edges, then R-MAT edges (A = .55, B = C = .01); weight 0xBEEF."""
    n = 1 << scale
    if end is None:
        end = n * edgefactor + n - 1
    if out is None:
        out = np.zeros(end - start, dtype=WEDGE_DTYPE)
    ptr, dev = _ptr(out)
    if _nbytes(out) < (end - start) * WEDGE_DTYPE.itemsize:
        raise ValueError("output buffer too small for the requested edge range")
    check(lib().g500_gen_edges_spec2012(scale, edgefactor, seed1, seed2, start, end, ptr, int(dev), None))
    return out


def generate_graph_spec2010(scale: int, edgefactor: int = 16) -> EdgeList:
    """generate_graph_spec2010 (mpi/benchmark_helper.hpp:308-314) into host memory."""
    return EdgeList(generate_edges(scale, edgefactor), scale, edgefactor)


def scramble_values(scale: int, seed1: int = USERSEED1, seed2: int = USERSEED2) -> tuple[int, int]:
    a, b = C.c_uint64(), C.c_uint64()
    check(lib().g500_scramble_values(scale, seed1, seed2, C.byref(a), C.byref(b)))
    return a.value, b.value


# ---------------------------------------------------------------------------
# (b) construction
# ---------------------------------------------------------------------------
class Graph2DCSR:
    """Device-resident graph (mpi/graph_constructor.hpp:24-143) for one GPU."""

    def __init__(self, handle: int):
        self.h = C.c_void_p(handle)
        info = GraphInfo()
        check(lib().g500_graph_info_get(self.h, C.byref(info)))
        self.info = info
        self.log_orig_global_verts_ = info.log_orig_global_verts
        self.num_local_verts_ = info.num_local_verts
        self.num_global_verts_ = info.num_global_verts
        self.num_global_edges_ = info.num_global_edges
        self.reorder_mode = info.reorder_mode

    @classmethod
    def build(cls, edges: np.ndarray, reorder_mode: int = 2, keep_edges: bool = True, device: int = 0):
        ptr, dev = _ptr(edges)
        h = C.c_void_p()
        check(lib().g500_graph_build(ptr, _num_edges(edges), int(dev), reorder_mode, int(keep_edges), device,
                                     C.byref(h)))
        return cls(h.value)

    @classmethod
    def generate(cls, scale: int, edgefactor: int = 16, reorder_mode: int = 2, device: int = 0,
                 seed1: int = USERSEED1, seed2: int = USERSEED2):
        h = C.c_void_p()
        check(lib().g500_graph_generate(scale, edgefactor, seed1, seed2, reorder_mode, device, C.byref(h)))
        return cls(h.value)

    def save(self, path: str) -> None:
        """Write the constructed graph to a snapshot file (g500_graph_save)."""
        check(lib().g500_graph_save(self.h, os.fsencode(path)))

    @classmethod
    def load(cls, path: str, device: int = 0):
        """A graph read back from a snapshot file onto `device` (g500_graph_load)."""
        h = C.c_void_p()
        check(lib().g500_graph_load(os.fsencode(path), device, C.byref(h)))
        return cls(h.value)

    def pred_size(self) -> int:
        return self.info.pred_size

    def log_orig_global_verts(self) -> int:
        return self.info.log_orig_global_verts

    def has_edge(self, v: int) -> bool:
        out = C.c_int()
        check(lib().g500_graph_has_edge(self.h, v, C.byref(out)))
        return bool(out.value)

    def timings(self) -> tuple[float, float]:
        a, b = C.c_double(), C.c_double()
        check(lib().g500_graph_timings(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def device_edges(self) -> tuple[int, int]:
        p, m = C.c_void_p(), C.c_int64()
        check(lib().g500_graph_edges(self.h, C.byref(p), C.byref(m)))
        return (p.value or 0), m.value

    def copy_csr(self) -> dict:
        nlv, nge, nolv = self.info.num_local_verts, self.info.num_global_edges, self.info.pred_size
        offsets = np.zeros(nlv + 1, np.uint64)
        cols = np.zeros(max(nge, 1), np.uint32)
        rmap = np.zeros(nolv, np.uint32)
        check(lib().g500_graph_copy_csr(self.h, offsets.ctypes.data, cols.ctypes.data, rmap.ctypes.data))
        return {"offsets": offsets, "cols": cols[:nge], "reorder_map": rmap}

    def close(self) -> None:
        if self.h is not None and self.h.value:
            check(lib().g500_graph_destroy(self.h))
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def find_roots(graph: Graph2DCSR, num_roots: int, seed1: int = USERSEED1, seed2: int = USERSEED2) -> np.ndarray:
    """find_roots (mpi/benchmark_helper.hpp:475-508)."""
    out = np.zeros(num_roots, np.int64)
    n = C.c_int()
    check(lib().g500_graph_find_roots(graph.h, num_roots, seed1, seed2, out.ctypes.data, C.byref(n)))
    return out[:n.value]


def find_max_used_vertex(graph: Graph2DCSR) -> int:
    """find_max_used_vertex (mpi/benchmark_helper.hpp:510-528)."""
    return graph.info.max_used_vertex


# ---------------------------------------------------------------------------
# (c) BFS -- the BfsBase method set
# ---------------------------------------------------------------------------
class BfsOnGPU:
    """BfsBase (mpi/bfs.hpp:29-2649) on one B200.

    construct -> prepare_bfs -> run_bfs(root, pred) / get_pred -> end_bfs, as
    mpi/main.cc drives BfsOnCPU.
    """

    def __init__(self, device: int = 0, reorder_mode: int = 2):
        self.device = device
        self.reorder_mode = reorder_mode
        self.graph_: Graph2DCSR | None = None
        self.h = None
        self.last_stats = BfsStats()

    # bfs.hpp:102-113
    def construct(self, edge_list, keep_edges: bool = True) -> None:
        if isinstance(edge_list, EdgeList) and edge_list.edges is None:
            self.graph_ = Graph2DCSR.generate(edge_list.scale, edge_list.edgefactor, self.reorder_mode, self.device)
        else:
            edges = edge_list.edges if isinstance(edge_list, EdgeList) else edge_list
            self.graph_ = Graph2DCSR.build(edges, self.reorder_mode, keep_edges, self.device)

    # bfs.hpp:115-118
    def prepare_bfs(self, alpha: float = 2000.0, beta: float = 8.0, count_edges: bool = False,
                    policy: int = DIR_REFERENCE) -> None:
        if self.graph_ is None:
            raise G500Error(G500_E_STATE, "construct() first")
        h = C.c_void_p()
        check(lib().g500_bfs_create(self.graph_.h, C.byref(h)))
        self.h = h
        self.set_params(alpha, beta, count_edges, policy)

    def set_params(self, alpha: float = 2000.0, beta: float = 8.0, count_edges: bool = False,
                   policy: int | None = None) -> None:
        check(lib().g500_bfs_set_params(self.h, alpha, beta, int(count_edges)))
        if policy is not None:
            check(lib().g500_bfs_set_policy(self.h, policy))

    def set_pred_mode(self, mode: int = 0) -> None:
        """0 by pred size, 1 pred written as vertices are found, 2 deferred (one pass at the end),
        3 deferred with 32-bit entries (a search deeper than 31 levels reruns in mode 2)."""
        check(lib().g500_bfs_set_pred_mode(self.h, mode))

    def set_host_pack(self, on: bool = True) -> None:
        """A pageable host pred crosses PCIe as packed 32-bit entries expanded by host threads (default),
        or always as int64; a pinned pred is always one int64 DMA copy."""
        check(lib().g500_bfs_set_host_pack(self.h, int(on)))

    def autotune(self, roots, reps: int = 2) -> dict:
        """Pick the direction policy and thresholds on sample roots (kept on the handle)."""
        r = np.ascontiguousarray(roots, dtype=np.int64)
        out = TuneResult()
        check(lib().g500_bfs_autotune(self.h, r.ctypes.data, len(r), reps, C.byref(out)))
        return {f[0]: getattr(out, f[0]) for f in TuneResult._fields_}

    # bfs.hpp:120, :2651-2940
    def run_bfs(self, root: int, pred) -> BfsStats:
        if self.h is None:
            raise G500Error(G500_E_STATE, "prepare_bfs() first")
        ptr, dev = _ptr(pred)
        if _nbytes(pred) < 8 * self.graph_.pred_size():
            raise ValueError(f"pred holds fewer than pred_size() = {self.graph_.pred_size()} int64 entries")
        st = BfsStats()
        check(lib().g500_bfs_run(self.h, int(root), ptr, int(dev), C.byref(st)))
        self.last_stats = st
        return st

    # bfs.hpp:122-124 (no-op in the reference too: run_bfs already wrote pred)
    def get_pred(self, pred) -> None:
        return None

    def level_stats(self) -> list[dict]:
        arr = (LevelStats * 4096)()
        n = C.c_int()
        check(lib().g500_bfs_level_stats(self.h, arr, 4096, C.byref(n)))
        keys = [f[0] for f in LevelStats._fields_]
        return [{k: getattr(arr[i], k) for k in keys} for i in range(min(n.value, 4096))]

    def device_pred_ptr(self) -> int:
        p = C.c_void_p()
        check(lib().g500_bfs_device_pred(self.h, C.byref(p)))
        return p.value or 0

    # bfs.hpp:126-128
    def end_bfs(self) -> None:
        if self.h is not None:
            check(lib().g500_bfs_destroy(self.h))
            self.h = None

    def close(self) -> None:
        self.end_bfs()
        if self.graph_ is not None:
            self.graph_.close()
            self.graph_ = None


# ---------------------------------------------------------------------------
# batched multi-source BFS
# ---------------------------------------------------------------------------
class MultiSourceBFS:
    """Many roots per launch (bit-lanes of 32/64/128-bit masks per vertex)."""

    def __init__(self, graph: Graph2DCSR, lane_width: int = 64, alpha: float = 15.0, use_cuda_graph: bool = True):
        self.graph = graph
        h = C.c_void_p()
        check(lib().g500_msbfs_create(graph.h, C.byref(h)))
        self.h = h
        self.set_params(lane_width, alpha, use_cuda_graph)

    def set_params(self, lane_width: int = 64, alpha: float = 15.0, use_cuda_graph: bool = True) -> None:
        check(lib().g500_msbfs_set_params(self.h, lane_width, alpha, int(use_cuda_graph)))

    def run(self, roots, levels=None) -> MsStats:
        """levels: None (stay on the device), or a host/device buffer of
        len(roots) * pred_size bytes (root-major, 255 = unreached)."""
        r = np.ascontiguousarray(roots, dtype=np.int64)
        st = MsStats()
        if levels is None:
            check(lib().g500_msbfs_run(self.h, r.ctypes.data, len(r), None, 0, C.byref(st)))
        else:
            ptr, dev = _ptr(levels)
            if _nbytes(levels) < len(r) * self.graph.pred_size():
                raise ValueError("levels buffer smaller than len(roots) * pred_size bytes")
            check(lib().g500_msbfs_run(self.h, r.ctypes.data, len(r), ptr, int(dev), C.byref(st)))
        return st

    def levels(self, roots) -> np.ndarray:
        """Run and return a (len(roots), pred_size) uint8 host array."""
        out = np.empty((len(roots), self.graph.pred_size()), np.uint8)
        self.run(roots, out)
        return out

    def root_stats(self, n: int) -> tuple[np.ndarray, np.ndarray]:
        reached, nedge = np.zeros(n, np.int64), np.zeros(n, np.int64)
        check(lib().g500_msbfs_root_stats(self.h, reached.ctypes.data, nedge.ctypes.data))
        return reached, nedge

    def launch(self, roots) -> None:
        """Enqueue a call and return at once (g500_msbfs_launch); levels stay on the device."""
        self._launched = np.ascontiguousarray(roots, dtype=np.int64)
        check(lib().g500_msbfs_launch(self.h, self._launched.ctypes.data, len(self._launched)))

    def poll(self) -> bool:
        done = C.c_int32()
        check(lib().g500_msbfs_poll(self.h, C.byref(done)))
        return bool(done.value)

    def wait(self) -> MsStats:
        st = MsStats()
        check(lib().g500_msbfs_wait(self.h, C.byref(st)))
        return st

    def set_root_stats(self, on: bool = True) -> None:
        check(lib().g500_msbfs_set_root_stats(self.h, int(on)))

    def set_count(self, on: bool = True) -> None:
        """Counting runs: level_info() then carries rows_read and sectors per level (untimed use)."""
        check(lib().g500_msbfs_set_count(self.h, int(on)))

    def set_grid(self, blocks: int = 0) -> None:
        check(lib().g500_msbfs_set_grid(self.h, blocks))

    def set_sparse(self, on: bool = True, limit: int = 0) -> None:
        """Sparse push levels up to a last-frontier degree sum of `limit` (0 = nlv / 8); levels are the same."""
        check(lib().g500_msbfs_set_sparse(self.h, int(on), limit))

    def grid(self, lane_width: int = 64) -> tuple[int, int]:
        b, mx = C.c_int32(), C.c_int32()
        check(lib().g500_msbfs_get_grid(self.h, lane_width, C.byref(b), C.byref(mx)))
        return b.value, mx.value

    def device_levels(self, nroots: int):
        """The device output of the last call as a (nroots, pred_size) uint8 torch tensor view."""
        import torch
        p = C.c_void_p()
        check(lib().g500_msbfs_device_levels(self.h, C.byref(p)))
        n = nroots * self.graph.pred_size()
        return _device_u8(p.value, n).view(nroots, self.graph.pred_size())

    def level_info(self, batch: int = 0) -> list[dict]:
        """Per level of launch `batch` of the last run: direction, discovered
        (vertex, root) pairs and device milliseconds."""
        buf = (MsLevel * 256)()
        n = C.c_int32()
        check(lib().g500_msbfs_level_info(self.h, batch, buf, 256, C.byref(n)))
        return [{f[0]: getattr(buf[i], f[0]) for f in MsLevel._fields_} for i in range(min(n.value, 256))]

    def autotune(self, roots, reps: int = 2) -> dict:
        r = np.ascontiguousarray(roots, dtype=np.int64)
        out = MsTune()
        check(lib().g500_msbfs_autotune(self.h, r.ctypes.data, len(r), reps, C.byref(out)))
        return {f[0]: getattr(out, f[0]) for f in MsTune._fields_}

    def close(self) -> None:
        if self.h is not None:
            check(lib().g500_msbfs_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# (d) validation
# ---------------------------------------------------------------------------
def validate_bfs_result(graph: Graph2DCSR, root: int, pred, edge_list=None) -> tuple[bool, int, dict]:
    """validate_bfs_result (mpi/validate.hpp:1008-1019) on the GPU.

    nglobalverts = max_used_vertex + 1 and nlocalverts = pred_size, as
    mpi/main.cc:129-133 calls it.  edge_list None uses the graph's resident
    edge list.  Returns (ok, edge_visit_count, per-stage error counts).
    """
    pptr, pdev = _ptr(pred)
    if _nbytes(pred) < 8 * graph.pred_size():
        raise ValueError(f"pred holds fewer than pred_size() = {graph.pred_size()} int64 entries")
    eptr, edev, m = None, 1, 0
    if edge_list is not None:
        edges = edge_list.edges if isinstance(edge_list, EdgeList) else edge_list
        eptr, d = _ptr(edges)
        edev, m = int(d), _num_edges(edges)
    evc, ok, rep = C.c_int64(), C.c_int(), ValidateReport()
    check(lib().g500_validate(graph.h, eptr, m, edev, int(root), pptr, int(pdev), C.byref(evc), C.byref(ok),
                              C.byref(rep)))
    return bool(ok.value), evc.value, {f[0]: getattr(rep, f[0]) for f in ValidateReport._fields_}


def levels_from_pred(pred: np.ndarray) -> np.ndarray:
    """(pred >> 48) & 0xFFFF with 0xFFFF for unreached (validate.hpp:813)."""
    lv = ((pred >> 48) & 0xFFFF).astype(np.uint16)
    lv[pred == -1] = 0xFFFF
    return lv


def _device_u8(ptr: int, n: int):
    """A torch uint8 CUDA tensor over n bytes of library-owned device memory (no copy)."""
    import torch

    class _Arr:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3}
    return torch.as_tensor(_Arr(), device="cuda")


# ---------------------------------------------------------------------------
# serving
# ---------------------------------------------------------------------------
class Server:
    """Request loop over resident graphs (g500_server_*): queries are batched
    into multi-source launches as they arrive (continuous batching)."""

    def __init__(self, graphs, **config):
        cfg = ServerConfig()
        check(lib().g500_server_default_config(C.byref(cfg)))
        for k, v in config.items():
            if not hasattr(cfg, k):
                raise TypeError(f"unknown server option {k}")
            setattr(cfg, k, v)
        self.graphs = list(graphs)
        arr = (C.c_void_p * len(self.graphs))(*[g.h.value if isinstance(g.h, C.c_void_p) else g.h
                                                 for g in self.graphs])
        h = C.c_void_p()
        check(lib().g500_server_create(arr, len(self.graphs), C.byref(cfg), C.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, graph: int, root: int, tag: int = 0, levels=None) -> int:
        """levels: None or a buffer of pred_size bytes (host or device) for the query's levels."""
        ptr = None
        if levels is not None:
            if _nbytes(levels) < self.graphs[graph].pred_size():
                raise ValueError("levels buffer smaller than pred_size bytes")
            ptr, _ = _ptr(levels)
        qid = C.c_int64()
        check(lib().g500_server_submit(self.h, graph, int(root), tag, ptr, C.byref(qid)))
        if levels is not None:
            self._keep[qid.value] = levels
        return qid.value

    def poll(self, max_results: int = 1024, wait_us: int = 0) -> list[dict]:
        buf = (QueryResult * max_results)()
        n = C.c_int32()
        check(lib().g500_server_poll(self.h, buf, max_results, C.byref(n), wait_us))
        out = [{f[0]: getattr(buf[i], f[0]) for f in QueryResult._fields_} for i in range(n.value)]
        for r in out:
            self._keep.pop(r["id"], None)
        return out

    def drain(self, timeout_ms: int = 60000) -> None:
        check(lib().g500_server_drain(self.h, timeout_ms))

    def info(self) -> dict:
        i = ServerInfo()
        check(lib().g500_server_info(self.h, C.byref(i)))
        return {f[0]: getattr(i, f[0]) for f in ServerInfo._fields_}

    def set_delivery(self, mode: int) -> None:
        """DELIVER_NONE, DELIVER_DEVICE or DELIVER_HOST for the load generator's queries."""
        check(lib().g500_server_set_delivery(self.h, int(mode)))

    def run_poisson(self, rate_qps: float, num_queries: int, seed: int = 2026, warmup: int = 0) -> dict:
        rep = ServeReport()
        check(lib().g500_server_run_poisson(self.h, rate_qps, num_queries, seed, warmup, C.byref(rep)))
        return {f[0]: getattr(rep, f[0]) for f in ServeReport._fields_}

    def close(self) -> None:
        if self.h is not None:
            check(lib().g500_server_destroy(self.h))
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
