// Internal declarations shared by the CUDA translation units of libg500.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>
#include <string>
#include <vector>

#include "../../include/g500.h"

namespace g500 {

// ------------------------------------------------------------------ errors
int set_error(int code, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what, const char* file, int line);

#define G500_CUDA(call)                                                        \
  do {                                                                         \
    cudaError_t e__ = (call);                                                  \
    if (e__ != cudaSuccess) return ::g500::cuda_error(e__, #call, __FILE__, __LINE__); \
  } while (0)

#define G500_TRY(call)                                                         \
  do {                                                                         \
    int s__ = (call);                                                          \
    if (s__ != G500_OK) return s__;                                            \
  } while (0)

constexpr unsigned FULL_MASK = 0xFFFFFFFFu;
constexpr int64_t LOCAL_VERTS_UNIT = 65536;  // max(11, 16) bits, bfs.hpp:109 + graph_constructor.hpp:557
constexpr int TD_CHUNK = 128;                // edges per top-down work item (one warp pass)
constexpr uint32_t NO_VERTEX = 0xFFFFFFFFu;
// first[v] of a row with more than one edge carries FIRST_MORE (when the graph
// has first_flags: every reordered id then fits in 31 bits), so that a
// bottom-up miss on a one-edge row needs no further scan
constexpr uint32_t FIRST_MORE = 0x80000000u;
constexpr uint32_t FIRST_ID = 0x7FFFFFFFu;

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t roundup(int64_t a, int64_t b) { return ceil_div(a, b) * b; }
inline int msb_index(uint64_t v) { return 63 - __builtin_clzll(v); }
inline int bits_for(uint64_t n) {  // smallest b with (1 << b) >= n
  int b = 0;
  while ((uint64_t(1) << b) < n) ++b;
  return b;
}

int num_sms();

// device allocation helpers (set the library error on failure)
int dev_alloc(void** p, size_t bytes, const char* what);
template <typename T>
int dev_alloc_n(T** p, int64_t n, const char* what) {
  return dev_alloc(reinterpret_cast<void**>(p), sizeof(T) * (size_t)(n > 0 ? n : 1), what);
}
void dev_free(void* p);

// ------------------------------------------------------------- primitives
// Exclusive prefix sum of n values (uint32 or uint64 input) into uint64
// out[0..n]; out[n] = total.  tmp: scan_tmp_bytes(n) bytes of device memory.
size_t scan_tmp_bytes(int64_t n);
int exclusive_scan_u32(const uint32_t* in, uint64_t* out, int64_t n, void* tmp, cudaStream_t s);
int exclusive_scan_u64(const uint64_t* in, uint64_t* out, int64_t n, void* tmp, cudaStream_t s);

// Stable LSD radix sort of 64-bit keys on bits [lo_bit, hi_bit), 8 bits a
// pass.  Sorts keys (n) using alt (n) as the ping-pong buffer; *result is the
// buffer holding the sorted keys (keys or alt).  tmp: sort_tmp_bytes(n).
size_t sort_tmp_bytes(int64_t n);
int radix_sort_u64(uint64_t* keys, uint64_t* alt, int64_t n, int lo_bit, int hi_bit,
                   void* tmp, cudaStream_t s, uint64_t** result);

// -------------------------------------------------------------- generator
struct GenPlan;  // defined in gen.cu
int gen_edges_device(int scale, uint64_t seed1, uint64_t seed2, int64_t start, int64_t end,
                     g500_packed_edge* out, cudaStream_t s);
int gen_edges_spec2012_device(int scale, uint64_t seed1, uint64_t seed2, int64_t start, int64_t end,
                              g500_weighted_edge* out, cudaStream_t s);

// 5x5 transition matrices mod 2^31-1 on the host
struct Mat5 { uint32_t m[25]; };
void mrg_skip_matrix_host(int byte_index, int val, Mat5* out);
void mat5_mul_host(const Mat5& a, const Mat5& b, Mat5* r);
void mrg_seed_host(uint64_t s1, uint64_t s2, uint32_t z[5]);
void mrg_skip_host(uint32_t z[5], uint64_t hi, uint64_t mid, uint64_t lo);
uint32_t mrg_next_host(uint32_t z[5]);
void scramble_values_host(uint64_t s1, uint64_t s2, uint64_t* v0, uint64_t* v1);

}  // namespace g500

// --------------------------------------------------------------- handles
struct g500_graph {
  int device = 0;
  cudaStream_t stream = nullptr;
  int reorder_mode = 0;
  int log_bits = 0;                 // bits of a reordered id used in sort keys
  int64_t log_orig_global_verts = 0;
  int64_t nolv = 0;                 // pred_size / num_orig_local_verts
  int64_t nlv = 0;                  // num_local_verts (multiple of 65536)
  int64_t ngv = 0;                  // vertices with >= 1 edge
  int64_t nge = 0;                  // directed CSR entries
  int64_t max_used_vertex = 0;
  int64_t device_bytes = 0;
  double gen_seconds = 0, build_seconds = 0;

  uint64_t* d_offsets = nullptr;    // [nlv + 1]
  uint32_t* d_cols = nullptr;       // [nge]   reordered targets, ascending per row
  uint32_t* d_first = nullptr;      // [nlv]   first (smallest) neighbour (| FIRST_MORE) or NO_VERTEX
  bool first_flags = false;         // first[] carries FIRST_MORE (nlv <= FIRST_ID)
  uint32_t* d_reorder = nullptr;    // [nolv]  original -> reordered
  uint32_t* d_invert = nullptr;     // [nolv]  reordered -> original
  uint32_t* d_vis_init = nullptr;   // [nlv/32] ~has_edge in reordered space
  uint32_t* d_endp = nullptr;       // [nolv]  input endpoint occurrences per reordered vertex
  g500_packed_edge* d_edges = nullptr;  // resident input edge list (optional)
  int64_t num_edges = 0;
  bool owns_edges = false;

  std::vector<uint32_t> h_has_edge_orig;  // bitmap over original ids
};

// Per-phase counters of the persistent BFS kernel (3 rotating slots).
// C_MF: degree sum of new top-down discoveries; C_BIG: rows listed whole for the next top-down level
enum BfsCounter { C_QITEMS = 0, C_DISC, C_SCAN, C_EDGES, C_SECT, C_FRONT, C_SKIP, C_MF, C_BIG, C_NUM };

// Top-down work item: one chunk (<= TD_CHUNK edges) of a frontier row.
struct __align__(16) TdItem {
  unsigned long long begin;  // first adjacency index of the chunk
  uint32_t orig;             // original id of the row's vertex (the parent written to pred)
  uint32_t len;              // chunk length; bit 31 marks the row's first chunk
};
enum BfsErr { BFS_ERR_QUEUE = 1, BFS_ERR_TIMEOUT = 2, BFS_ERR_DEPTH = 4, BFS_ERR_PACK = 8 };
constexpr unsigned GRID_ERR_TIMEOUT = 2;  // same bit as BFS_ERR_TIMEOUT

// State of a grid-wide barrier of a cooperative kernel (device memory, zeroed
// before each launch): arrivals of every barrier of the launch so far, sticky
// error bits.
struct GridBarrier {
  unsigned count;
  unsigned reserved;
  unsigned err;
  unsigned pad;
};

// Append positions of a phase (found list / work items, listed long rows),
// three rotating slots like the counters
enum BfsPos { P_ITEMS = 0, P_BIG, P_NUM };

// Control block of one run, in device memory.
struct BfsCtl {
  unsigned long long cnt[3][C_NUM];
  unsigned long long pos[3][P_NUM];
  GridBarrier bar;
  unsigned num_levels;
  int final_vis;
  int root_has_edges;
  unsigned long long t0_ns;
  unsigned long long t_init_ns;  // pred/visited initialised and root seeded
  unsigned long long t_end_ns;
  unsigned long long reach[2];  // reached vertices, 2 * nedge (filled by reach_kernel)
  unsigned pad_overflow;        // host copy of the levels-overflow flag of an asynchronous run
};

// One record per level, written by the kernel.
struct LevelRecord {
  int32_t direction;
  int32_t level;
  unsigned long long frontier, discovered, scanned, edges, sectors;
  unsigned long long t_mid_ns;  // %globaltimer after the level's first barrier (TD expand / BU pass A)
  unsigned long long t_ns;      // %globaltimer when the level's last barrier completed
};

constexpr int MAX_LEVELS = 0xFFFE;

namespace g500 {
class PredExpander;
}

struct g500_bfs {
  g500_graph* g = nullptr;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  double alpha = 2000.0, beta = 8.0;
  int policy = 0;                    // G500_DIR_REFERENCE or G500_DIR_EDGES
  int count_edges = 0;
  unsigned grid = 0;                 // co-resident blocks of the persistent kernel

  int64_t* d_pred = nullptr;         // [nolv]
  int64_t* d_pred_r = nullptr;       // [nlv] deferred mode: pred entries by reordered id
  uint8_t* d_levels = nullptr;       // [nolv] levels of an asynchronous run (serving)
  unsigned* d_overflow = nullptr;    // a level over 254 in d_levels
  cudaEvent_t ev_done = nullptr;
  int in_flight = 0;
  unsigned grid_full = 0;            // every co-resident block of the device
  int pred_mode = 0;                 // 0 by pred size, 1 direct, 2 deferred, 3 deferred packed
  int pack_off = 0;                  // a search outgrew the packed level field: deferred runs stay unpacked
  uint8_t* last_levels_dst = nullptr;  // levels destination of the run in flight (a rerun writes it again)
  // a host pred crosses PCIe as packed 32-bit entries, expanded by host threads
  int pack_host_off = 0;
  uint32_t* d_pack = nullptr;        // [nolv]
  unsigned* d_pack_ovf = nullptr;
  uint32_t* h_pack = nullptr;        // pinned [nolv + 64]
  cudaEvent_t ev_chunk[8] = {};
  g500::PredExpander* expander = nullptr;
  uint32_t* d_vis[2] = {nullptr, nullptr};
  TdItem* d_queue[2] = {nullptr, nullptr};
  int64_t queue_cap = 0;
  BfsCtl* d_ctl = nullptr;
  BfsCtl* h_ctl = nullptr;           // pinned copy after each run
  LevelRecord* d_rec = nullptr;      // [MAX_LEVELS]
  TdItem* d_big = nullptr;           // [BIG_ROWS] long frontier rows, listed whole
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int64_t last_root = -1;
};

namespace g500 {
// Asynchronous plain BFS for the serving loop: the run from `root`, its uint8
// levels (255 unreached) into levels_dst (host or device, may be null), the
// reached / edge counts, all enqueued on the handle's stream.
int bfs_launch_levels(g500_bfs* b, int64_t root, uint8_t* levels_dst);
int bfs_poll(g500_bfs* b, int* done);
int bfs_complete(g500_bfs* b, int64_t* reached, int64_t* nedge);

// Copy the run's pred (b->d_pred) to host_pred as packed entries, expanded by
// host threads chunk by chunk; *packed = false when the graph or the run
// does not fit the packed form (the caller then copies the int64 entries).
// Enqueued on s after the run; returns when host_pred is complete.
int pred_to_host_packed(g500_bfs* b, int64_t* host_pred, cudaStream_t s, bool* packed);
void pred_expander_free(g500_bfs* b);

// g500_msbfs_launch that also copies each root's level row (pred_size bytes)
// to root_dsts[i] when it is not null, before the launch's completion event.
int msbfs_launch_to(g500_msbfs* m, const int64_t* roots, int nroots, uint8_t* const* root_dsts);
}  // namespace g500

namespace g500 {
// An empty graph handle on `device` with its own stream (build.cu).
int new_graph(int device, int reorder_mode, g500_graph** out);
int graph_destroy_internal(g500_graph* g);
}  // namespace g500
