/*
 * g500.h -- C ABI of the B200-native Graph500 BFS hot path (libg500.so).
 *
 * Plain C types only: pointers, sizes, status codes.  Every function returns
 * G500_OK (0) or a G500_E_* status; g500_last_error() gives the message of the
 * calling thread's last failure.  No exception crosses this boundary.
 *
 * Each entry point replaces one step of the suzumura/graph500 reference,
 * cited below as path:line inside that project.  Vertex ids at this boundary
 * are the reference's ORIGINAL (scrambled, int64) ids; the reordered ids the
 * kernels use internally never leave the library.
 *
 * Threading: a handle is used by one host thread at a time.  All work of a
 * handle is ordered on that handle's CUDA stream.  Handles of different
 * graphs are independent.
 */
#ifndef G500_H
#define G500_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define G500_ABI_VERSION 1

enum g500_status {
  G500_OK = 0,
  G500_E_INVAL = 1,    /* bad argument (null handle, out-of-range root, ...) */
  G500_E_NOMEM = 2,    /* device or pinned-host allocation failed */
  G500_E_DEVICE = 3,   /* a CUDA call failed (message has the CUDA error) */
  G500_E_TIMEOUT = 4,  /* a bounded device-side wait gave up */
  G500_E_RANGE = 5,    /* size beyond what the format or a fixed buffer holds */
  G500_E_STATE = 6,    /* call out of order (e.g. run before create) */
  G500_E_VALIDATION = 7,
  G500_E_IO = 8        /* a file could not be read or written, or is not what it claims */
};

/* The reference's packed edge: 48-bit endpoints in 12 bytes
 * (mpi/primitives.hpp:51-81, UnweightedPackedEdge). */
typedef struct g500_packed_edge {
  uint32_t v0_low;
  uint32_t v1_low;
  uint32_t high; /* v0[47:32] | v1[47:32] << 16 */
} g500_packed_edge;

typedef struct g500_graph g500_graph;
typedef struct g500_bfs g500_bfs;
typedef struct g500_msbfs g500_msbfs;

/* Scalars of the built graph (mpi/graph_constructor.hpp:24-143, Graph2DCSR). */
typedef struct g500_graph_info {
  int64_t log_orig_global_verts; /* estimated SCALE (graph_constructor.hpp:754-759) */
  int64_t pred_size;             /* pred[] length = num_orig_local_verts (:64) */
  int64_t num_local_verts;       /* reordered range, multiple of 65536 (:338-346) */
  int64_t num_global_verts;      /* vertices with >= 1 edge (:1444-1464) */
  int64_t num_global_edges;      /* directed CSR entries after dedup (:1438-1441) */
  int64_t max_used_vertex;       /* largest original id with an edge (benchmark_helper.hpp:510) */
  int64_t num_input_edges;       /* length of the resident edge list (0 if not kept) */
  int64_t device_bytes;          /* device memory held by the graph */
  int32_t reorder_mode;          /* VERTEX_REORDERING 0/1/2 (parameters.h:37-41) */
  int32_t device;
} g500_graph_info;

/* ------------------------------------------------------------------ misc */
const char* g500_last_error(void);
int g500_abi_version(void);
/* Pinned host memory for fast host<->device copies (cudaHostAlloc). */
int g500_host_alloc(uint64_t bytes, void** out);
int g500_host_free(void* p);

/* ------------------------------------------------------ (a) generation */
/* The two scramble words of the generator (graph_generator.hpp:375-384). */
int g500_scramble_values(int scale, uint64_t userseed1, uint64_t userseed2,
                         uint64_t* val0, uint64_t* val1);

/* Edges [start, end) of the spec-2010 Kronecker graph, bit-exact to
 * RmatGraphGenerator<..,5700,1900>::generateRange (graph_generator.hpp:612-627,
 * called from generate_graph_spec2010, benchmark_helper.hpp:308-314).
 * out: end-start packed edges, device memory if out_on_device else host
 * memory.  stream: a cudaStream_t or NULL for the library's own stream. */
int g500_gen_edges(int scale, int edgefactor, uint64_t userseed1, uint64_t userseed2,
                   int64_t start, int64_t end, g500_packed_edge* out, int out_on_device,
                   void* stream);

/* WeightedEdge (mpi/primitives.hpp:87-106): the packed edge and an int weight. */
typedef struct g500_weighted_edge {
  uint32_t v0_low;
  uint32_t v1_low;
  uint32_t high;
  int32_t weight;
} g500_weighted_edge;

/* Edges [start, end) of the spec-2012 graph, bit-exact to
 * generate_graph_spec2012 (benchmark_helper.hpp:316-322):
 * RmatGraphGenerator<WeightedEdge, 5500, 100> (A = .55, B = C = .01) with
 * InitialEdgeType::BINARY_TREE, i.e. 2^scale * edgefactor + 2^scale - 1 edges,
 * of which edge i < 2^scale - 1 is (scramble(i + 1), scramble((i + 1) / 2))
 * (graph_generator.hpp:385-392, :513-520) and every later edge the R-MAT edge
 * of its index's stream (:612-627).  The weight is the reference's constant
 * 0xBEEF (generateWeight, :495-503, whose random draw is disabled); its SSSP
 * (run_sssp, bfs.hpp:2569-2571) is an empty stub, so nothing consumes the
 * weights.  out, out_on_device, stream as for g500_gen_edges. */
int g500_gen_edges_spec2012(int scale, int edgefactor, uint64_t userseed1, uint64_t userseed2,
                            int64_t start, int64_t end, g500_weighted_edge* out, int out_on_device,
                            void* stream);

/* ---------------------------------------------------- (b) construction */
/* BfsBase::construct(EdgeList*) (mpi/bfs.hpp:102-113 ->
 * GraphConstructor2DCSR::construct, graph_constructor.hpp:554-574).
 * edges may be host or device memory.  keep_edges != 0 keeps a device copy of
 * the edge list for on-device validation.  reorder_mode: VERTEX_REORDERING
 * 0 identity, 1 vertices with edges first, 2 degree descending; ties in
 * degree are ordered by ascending original id. */
int g500_graph_build(const g500_packed_edge* edges, int64_t num_edges, int edges_on_device,
                     int reorder_mode, int keep_edges, int device, g500_graph** out);

/* Generation + construction on the device in one call, edge list kept
 * resident (main.cc:45-60: generate_graph_spec2010 then construct). */
int g500_graph_generate(int scale, int edgefactor, uint64_t userseed1, uint64_t userseed2,
                        int reorder_mode, int device, g500_graph** out);

int g500_graph_info_get(const g500_graph* g, g500_graph_info* info);
/* Graph2DCSR::has_edge (graph_constructor.hpp:101-110), original id. */
int g500_graph_has_edge(const g500_graph* g, int64_t v, int* out);
/* find_roots (benchmark_helper.hpp:475-508); *found = roots written. */
int g500_graph_find_roots(const g500_graph* g, int num_roots, uint64_t userseed1,
                          uint64_t userseed2, int64_t* roots, int* found);
/* The resident device edge list, if kept (NULL otherwise). */
int g500_graph_edges(const g500_graph* g, const g500_packed_edge** dev_edges, int64_t* num_edges);
/* Host copies of the CSR for inspection: offsets[num_local_verts+1],
 * cols[num_global_edges] (reordered ids), reorder_map[pred_size] (original ->
 * reordered).  Any pointer may be NULL. */
int g500_graph_copy_csr(const g500_graph* g, uint64_t* offsets, uint32_t* cols,
                        uint32_t* reorder_map);
/* CSR snapshots: the constructed graph (CSR, maps, bitmaps and the kept edge
 * list, if any) written to a file and read back onto `device`, so that a
 * serving process loads resident graphs without regenerating them.  No
 * counterpart in the reference (its TMPFILE spill holds only the edge list,
 * graph_generator.hpp:67-83).  Errors: G500_E_IO for unreadable, truncated or
 * foreign files. */
int g500_graph_save(const g500_graph* g, const char* path);
int g500_graph_load(const char* path, int device, g500_graph** out);
/* Seconds spent on the device in generation and construction. */
int g500_graph_timings(const g500_graph* g, double* generation_s, double* construction_s);
int g500_graph_destroy(g500_graph* g);

/* ------------------------------------------------------------ (c) BFS */
/* Per-level record of a run (bfs.hpp:2831-2887 prints the same quantities). */
typedef struct g500_level_stats {
  int32_t direction;       /* 1 top-down, 0 bottom-up */
  int32_t level;
  int64_t frontier;        /* TD: frontier vertices */
  int64_t discovered;      /* vertices found at this level */
  int64_t scanned;         /* BU: unvisited vertices with edges scanned */
  int64_t edge_sectors;    /* TD: sum ceil(deg/8); BU: sum ceil(k/8) (if counting on) */
  int64_t edges_examined;  /* TD: sum deg; BU: sum k (if counting on) */
  double device_ms;        /* device time of the level (%globaltimer between level barriers) */
  double device_ms_tail;   /* part after the level's first barrier: BU miss pass / TD row chunking */
} g500_level_stats;

typedef struct g500_bfs_stats {
  double device_ms;        /* CUDA-event time of the whole run on the device */
  double host_ms;          /* host wall time of the call (includes any D2H copy) */
  int64_t reached;         /* vertices with a level */
  int64_t nedge;           /* input edges inside the reached component */
  int32_t num_levels;
  int32_t td_levels;
  int32_t bu_levels;
  int32_t kernel_launches; /* kernels this library launched for the run */
  double init_ms;          /* device global timer: kernel start to the first level */
  double search_ms;        /* device global timer: the levels (and the deferred pred pass) */
} g500_bfs_stats;

/* BfsBase::prepare_bfs / allocate_memory (bfs.hpp:115-118, :151-239). */
int g500_bfs_create(g500_graph* g, g500_bfs** out);
/* alpha / beta: denominators of the direction switch (DENOM_TOPDOWN_TO_BOTTOMUP
 * 2000, DEMON_BOTTOMUP_TO_TOPDOWN 8; parameters.h:87-88, bfs.hpp:2799-2829).
 * count_edges != 0 records edge_sectors/edges_examined per level (slower). */
int g500_bfs_set_params(g500_bfs* b, double alpha, double beta, int count_edges);
/* Direction policy.  G500_DIR_REFERENCE is the reference's rule (bfs.hpp:
 * 2799-2829): TD -> BU when growing and nq > num_global_verts / alpha; BU -> TD
 * when unvisited < num_global_verts / beta.  G500_DIR_EDGES compares edges
 * instead (Beamer, Asanovic, Patterson, SC'12): TD -> BU when the new
 * frontier's degree sum m_f > (degree sum of unvisited vertices) / alpha;
 * BU -> TD when the frontier shrinks below num_global_verts / beta.  Levels are
 * the same under every policy; only the parents and the speed differ. */
enum g500_dir_policy { G500_DIR_REFERENCE = 0, G500_DIR_EDGES = 1 };
int g500_bfs_set_policy(g500_bfs* b, int policy);
/* Use this stream for the runs (NULL = the handle's own stream). */
int g500_bfs_set_stream(g500_bfs* b, void* stream);
/* How run writes pred: 0 (default) by its size, 1 at random as vertices are
 * discovered, 2 deferred: entries by reordered id during the search, then one
 * sequential pass in original-id order, 3 deferred with 32-bit entries (graphs
 * of at most 2^27 vertex ids; a search deeper than 31 levels is run again
 * with mode 2, which the handle then keeps).  Results are identical. */
int g500_bfs_set_pred_mode(g500_bfs* b, int mode);
/* A pageable host pred (g500_bfs_run with pred_on_device = 0, memory not
 * pinned) crosses PCIe as 32-bit packed entries (parent id in 27 bits, level
 * in 5) into pinned staging, in chunks that host threads expand into the
 * caller's int64 array while the next chunk is copied: about twice as fast
 * as the runtime's pageable copy.  A pinned pred gets one DMA copy of the
 * int64 entries, as do graphs of more than 2^27 vertex ids and runs deeper
 * than 30 levels.  on = 1 (default) or 0 (always copy the int64 entries);
 * the values are the same. */
int g500_bfs_set_host_pack(g500_bfs* b, int on);
/* Blocks of the persistent kernel (0 = every co-resident block of the device);
 * fewer leave SMs to kernels of other handles running at the same time. */
int g500_bfs_set_grid(g500_bfs* b, int blocks);

/* Autotuner: time every (policy, alpha, beta) of a built-in grid on the given
 * roots (device pred, best of `reps` runs per root), keep the fastest on the
 * handle and report it.  No counterpart in the reference (its thresholds are
 * compile-time constants, parameters.h:87-88). */
typedef struct g500_tune_result {
  int32_t policy;
  int32_t configs_tried;
  double alpha;
  double beta;
  double best_ms;          /* mean device time per BFS of the chosen setting */
  double reference_ms;     /* the same for the reference setting (policy 0, 2000, 8) */
} g500_tune_result;
int g500_bfs_autotune(g500_bfs* b, const int64_t* roots, int num_roots, int reps, g500_tune_result* out);
/* BfsBase::run_bfs(root, pred) (bfs.hpp:120, :2651-2940): writes EVERY entry
 * of pred[pred_size]: parent | level << 48 for reached vertices, root = root,
 * -1 otherwise.  pred is device memory if pred_on_device else host memory
 * (the call then returns after the device-to-host copy).  stats may be NULL. */
int g500_bfs_run(g500_bfs* b, int64_t root, int64_t* pred, int pred_on_device,
                 g500_bfs_stats* stats);
/* Per-level records of the last run. */
int g500_bfs_level_stats(const g500_bfs* b, g500_level_stats* out, int max_levels, int* num_levels);
/* The device pred[] of the last run (valid until the next run or destroy). */
int g500_bfs_device_pred(const g500_bfs* b, const int64_t** dev_pred);
/* BfsBase::end_bfs / deallocate_memory (bfs.hpp:126-128). */
int g500_bfs_destroy(g500_bfs* b);

/* ------------------------------------------------------ (d) validation */
typedef struct g500_validate_report {
  int64_t range_errors;                /* validate.hpp:822-839 */
  int64_t root_errors;                 /* :529-537, :930-933 */
  int64_t self_parent_errors;          /* :542-571 */
  int64_t depth_errors;                /* :920-995 */
  int64_t edge_errors;                 /* :688-702 */
  int64_t missing_parent_edge_errors;  /* :780-792 */
} g500_validate_report;

/* validate_bfs_result (validate.hpp:1008-1019) with nglobalverts =
 * max_used_vertex + 1 and nlocalverts = pred_size, as main.cc:129-133 calls
 * it.  edges == NULL uses the graph's resident edge list.  *ok = 1 when the
 * result is valid; *edge_visit_count = the traversed-edge count TEPS uses. */
int g500_validate(g500_graph* g, const g500_packed_edge* edges, int64_t num_edges,
                  int edges_on_device, int64_t root, const int64_t* pred, int pred_on_device,
                  int64_t* edge_visit_count, int* ok, g500_validate_report* report);

/* ------------------------------------------- batched multi-source BFS */
/* Many roots per launch: one bit-lane per root in 32/64/128-bit masks per
 * vertex, a persistent cooperative kernel per launch, the launch sequence
 * captured as a CUDA graph.  No counterpart in the reference, which runs one
 * root at a time (main.cc:105-160); each root's levels equal the plain BFS's
 * (pred >> 48) (bfs.hpp:1203, :2470). */
typedef struct g500_msbfs_stats {
  double device_ms;        /* CUDA-event time of all launches of the call */
  double host_ms;          /* wall time of the call */
  int32_t num_levels;      /* deepest launch */
  int32_t pull_levels;     /* levels run as pull, summed over launches */
  int32_t lane_width;
  int32_t batches;         /* launches: ceil(roots / lane width) */
  int32_t kernel_launches;
  int32_t pad;
  double init_ms;          /* device global timer, summed over launches: clearing the masks, seeding */
  double search_ms;        /* device global timer, summed over launches: the levels */
} g500_msbfs_stats;

typedef struct g500_msbfs_tune {
  int32_t lane_width;
  int32_t configs_tried;
  double alpha;
  double best_ms;
} g500_msbfs_tune;

int g500_msbfs_create(g500_graph* g, g500_msbfs** out);
/* lane_width 32/64/128; alpha: pull when the new frontier's degree sum exceeds
 * (degree sum of vertices with unvisited lanes) / alpha; use_cuda_graph != 0
 * replays a captured graph per launch. */
int g500_msbfs_set_params(g500_msbfs* m, int lane_width, double alpha, int use_cuda_graph);
/* 1..128 roots (original ids).  levels: num_roots x pred_size bytes, root-major,
 * original vertex ids, the BFS level or 255 if unreached; device or host
 * memory per levels_on_device, or NULL to keep them on the device only
 * (g500_msbfs_device_levels). */
int g500_msbfs_run(g500_msbfs* m, const int64_t* roots, int num_roots, uint8_t* levels, int levels_on_device,
                   g500_msbfs_stats* stats);
/* Per root of the last run (which must have fitted one launch): vertices
 * reached and input edges inside the reached component (validate.hpp's
 * edge_visit_count for a valid BFS). */
int g500_msbfs_root_stats(g500_msbfs* m, int64_t* reached, int64_t* nedge);
int g500_msbfs_device_levels(const g500_msbfs* m, const uint8_t** dev_levels);
/* One level of one launch of the last run: its direction, the (vertex, root)
 * pairs it discovered, and its device time from the kernel's global timer. */
typedef struct g500_msbfs_level {
  int32_t level;
  int32_t pull;            /* 1 = pull (unvisited lanes look at the frontier), 0 = push, 2 = both: the
                              lanes with a small frontier pushed, the others pulled */
  int64_t discovered;      /* new (vertex, lane) pairs */
  double device_ms;        /* the whole level */
  double expand_ms;        /* its pull or push phase (the rest is the apply pass) */
  int64_t rows_read;       /* counting runs: row (or hub chunk) offset reads of the level, else -1 */
  int64_t sectors;         /* counting runs: 32-byte adjacency sectors the level's examined entries span, else -1 */
} g500_msbfs_level;
/* Copies up to max_levels records of launch `batch` of the last run into out;
 * *num_levels receives the launch's level count. */
int g500_msbfs_level_info(const g500_msbfs* m, int batch, g500_msbfs_level* out, int max_levels, int* num_levels);
/* on != 0: later runs are counting runs (a kernel variant that also records
 * each level's rows_read and sectors for the bytes model, launched without
 * the CUDA graph); their levels are the same.  Meant for untimed runs. */
int g500_msbfs_set_count(g500_msbfs* m, int on);
/* Asynchronous form of g500_msbfs_run for callers that overlap several
 * handles (the serving loop): launch enqueues the whole call on the handle's
 * stream and returns; poll reports whether it finished; wait blocks until it
 * has, checks the device status and fills stats.  One launch in flight per
 * handle; levels stay on the device (g500_msbfs_device_levels). */
int g500_msbfs_launch(g500_msbfs* m, const int64_t* roots, int num_roots);
int g500_msbfs_poll(g500_msbfs* m, int* done);
int g500_msbfs_wait(g500_msbfs* m, g500_msbfs_stats* stats);
/* on != 0: every call that fits one launch also computes the per-root
 * statistics of g500_msbfs_root_stats on the device, in the same stream. */
int g500_msbfs_set_root_stats(g500_msbfs* m, int on);
/* Blocks per launch (0 = every co-resident block of the device).  Fewer
 * blocks leave SMs to launches of other handles running at the same time. */
int g500_msbfs_set_grid(g500_msbfs* m, int blocks);
int g500_msbfs_get_grid(const g500_msbfs* m, int lane_width, int* blocks, int* max_blocks);
/* Sparse levels: a push level whose last frontier has a degree sum of at most
 * `limit` (0 = nlv / 8) works on the marked vertices only (the frontier rows
 * and the vertices it touches) instead of every vertex; on = 0 makes every
 * level dense.  Default: on with nlv / 8 from 2^22 vertices with edges, off
 * below.  The levels are the same either way. */
int g500_msbfs_set_sparse(g500_msbfs* m, int on, int64_t limit);
/* Device memory one handle on this graph allocates (an upper bound). */
int g500_msbfs_workspace_bytes(const g500_graph* g, uint64_t* bytes);
/* Autotuner over lane width and alpha on sample roots (kept on the handle). */
int g500_msbfs_autotune(g500_msbfs* m, const int64_t* roots, int num_roots, int reps, g500_msbfs_tune* out);
int g500_msbfs_destroy(g500_msbfs* m);

/* ------------------------------------------------------------- serving */
/* A request loop over several resident graphs: BFS queries (graph, root) are
 * admitted as they arrive, batched into multi-source launches while earlier
 * launches run (continuous batching), and overlap on the device on separate
 * streams.  The launch slots (g500_msbfs workspaces, up to
 * max_workers_per_graph per graph) are created with the server, each only
 * while the device keeps hbm_reserve_bytes free; a graph with fewer slots
 * gets another later only if memory allows then.  No counterpart in the reference,
 * which runs one root at a time (main.cc:105-160).  Each query's levels equal
 * the plain BFS's (pred >> 48) for its root, alone or in any mix.  The graphs
 * stay owned by the caller and must outlive the server. */
typedef struct g500_server g500_server;
enum g500_serve_mode { G500_SERVE_BATCHED = 0, G500_SERVE_PLAIN = 1 };

typedef struct g500_server_config {
  int32_t max_batch;             /* queries per launch, 1..128 */
  int32_t max_workers_per_graph; /* concurrent launches per graph */
  int32_t mode;                  /* G500_SERVE_BATCHED, or G500_SERVE_PLAIN: one g500_bfs_run per query */
  int32_t vertices_per_block;    /* grid of a graph's launches: ceil(num_local_verts / this), >= 16 blocks */
  uint64_t hbm_reserve_bytes;    /* free device memory a new launch slot must leave */
  double alpha;                  /* multi-source direction threshold (g500_msbfs_set_params) */
  double max_grid_fraction;      /* a launch uses at most this share of the device's co-resident blocks
                                    (so that launches of other graphs run beside it); (0, 1] */
  int32_t plain_below;           /* a graph with at most this many waiting queries runs them one plain
                                    BFS each (0 never; negative: calibrated per graph at create) */
  int32_t batch_target;          /* while a launch of a graph is in flight, another starts only once this
                                    many of its queries wait (0, the default: whenever a worker is idle) */
} g500_server_config;

typedef struct g500_query_result {
  int64_t id;
  uint64_t tag;
  int32_t graph;
  int32_t status;                /* G500_OK or the error of its launch */
  int64_t root;
  int64_t reached;               /* vertices with a level */
  int64_t nedge;                 /* input edges inside the reached component */
  double arrival_us;             /* host steady clock, microseconds since the server was created */
  double start_us;               /* its launch */
  double done_us;                /* seen complete by the server */
  int32_t batch_size;            /* queries in its launch */
  int32_t lane_width;
} g500_query_result;

typedef struct g500_server_info_t {
  int64_t submitted, finished, launches, queries_launched;
  int32_t workers, max_in_flight, block_capacity, pad;
} g500_server_info_t;

typedef struct g500_serve_report {
  double rate_qps;               /* offered Poisson rate */
  int64_t queries;               /* measured (after warm-up) and completed */
  int64_t failed;
  double wall_s;                 /* first measured arrival to last completion */
  double achieved_qps;
  double p50_ms, p99_ms, mean_ms, max_ms;  /* completion - arrival */
  double gteps;                  /* sum of nedge / wall */
  int64_t nedge;
  double mean_batch;             /* queries per launch */
  int64_t launches;
  int32_t max_in_flight;         /* launches running at once */
  int32_t workers;               /* launch slots created so far */
  int32_t delivery;              /* G500_DELIVER_*: where each query's levels went before it completed */
  int32_t pad;
} g500_serve_report;

/* Result delivery of the load generator's queries (g500_server_set_delivery). */
#define G500_DELIVER_NONE 0   /* levels stay in the launch's workspace (completion only) */
#define G500_DELIVER_DEVICE 1 /* each query's levels copied to a device buffer of its own */
#define G500_DELIVER_HOST 2   /* each query's levels copied to a pinned host buffer of its own */

int g500_server_default_config(g500_server_config* cfg);
int g500_server_create(g500_graph* const* graphs, int num_graphs, const g500_server_config* cfg, g500_server** out);
/* levels_out: NULL, or pred_size bytes that receive the query's levels (uint8,
 * original ids, 255 unreached) before it completes; pinned host memory
 * (g500_host_alloc) or device memory keeps the copy asynchronous. */
int g500_server_submit(g500_server* s, int graph, int64_t root, uint64_t tag, uint8_t* levels_out, int64_t* id);
/* Up to max_results completed queries (waiting up to wait_us for the first). */
int g500_server_poll(g500_server* s, g500_query_result* out, int max_results, int* num, int wait_us);
/* Wait until every submitted query has completed. */
int g500_server_drain(g500_server* s, int timeout_ms);
int g500_server_info(g500_server* s, g500_server_info_t* info);
/* Open-loop load: num_queries Poisson arrivals at rate_qps, each on a graph
 * chosen uniformly and a root chosen uniformly among vertices with at least
 * one edge (splitmix64 stream from seed); latency statistics skip the first
 * `warmup` queries.  With a delivery mode set (g500_server_set_delivery) each
 * query's level array (pred_size bytes) is copied to a buffer of its own
 * before the query completes, so its latency includes delivering the result. */
int g500_server_run_poisson(g500_server* s, double rate_qps, int64_t num_queries, uint64_t seed, int64_t warmup,
                            g500_serve_report* rep);
int g500_server_destroy(g500_server* s);
/* Where run_poisson delivers each query's levels: G500_DELIVER_NONE (default),
 * _DEVICE or _HOST.  Waits for the queries in flight, then allocates per graph
 * max_batch x max_workers_per_graph + 1 level buffers (a query waits for a free
 * one); G500_E_NOMEM when they do not fit. */
int g500_server_set_delivery(g500_server* s, int mode);

/* ------------------------------------------- partitioned single-root BFS */
/* One rank's share of a 1-D vertex partition for a BFS over several GPUs (or
 * ranks emulated in one process).  The reference runs one root over a 2-D
 * partition of MPI ranks, exchanging top-down "fold" packets to the owners of
 * discovered vertices (mpi/bfs.hpp:521-572, :962-1137) and the bottom-up
 * visited bitmap (bottom_up_comm.hpp:172-280) every level.  Here rank r of n
 * owns the reordered vertex ids [32*S*r, 32*S*(r+1)) (S bitmap words each;
 * g500_part_info) and the rows of those vertices in its replica of the CSR.
 * The caller runs the level loop and the collectives (graph500_b200.partitioned
 * does, over torch.distributed): per level every rank runs either
 * g500_part_top_down (then an all-to-all of the (target << 32 | parent) pairs
 * of g500_part_send_buffer, split by send_counts, and g500_part_apply of what
 * it received) or g500_part_bottom_up, sums the level counters
 * out[0..3] = {found, their degree sum, next frontier length, scanned} over the
 * ranks, calls g500_part_compact before a top-down level that follows a
 * bottom-up one, and all-gathers every rank's own slice (S words) into the
 * full bitmap (nranks * S words) of every rank (g500_part_buffers; the
 * slices and the bitmap are device memory, ordered on the rank's stream,
 * which every call has finished when it returns).  g500_part_write_pred then
 * writes pred (nolv entries, device memory) with this rank's reached vertices
 * and -1 elsewhere; the element-wise max over the ranks is the run's pred
 * (bfs.hpp:2651-2940 semantics: parent | level << 48, root = root).
 * g500_part_begin out[0..2] = {root has edges, frontier length, frontier
 * degree sum}.  A root without edges reached only itself: no rank lists it,
 * the caller writes pred[root] = root. */
#define G500_PART_MAX_RANKS 64
typedef struct g500_part g500_part;
int g500_part_create(g500_graph* g, int rank, int nranks, g500_part** out);
int g500_part_info(const g500_part* p, int64_t* words_per_rank, int64_t* first_vertex, int64_t* end_vertex);
int g500_part_buffers(g500_part* p, uint32_t** vis_full, uint32_t** own_slice, void** stream);
int g500_part_begin(g500_part* p, int64_t root, int64_t* out);
int g500_part_top_down(g500_part* p, int64_t frontier_edges, int64_t* send_counts);
int g500_part_send_buffer(g500_part* p, uint64_t** pairs);
int g500_part_apply(g500_part* p, const uint64_t* recv_pairs, int64_t num_pairs, int64_t* out);
int g500_part_bottom_up(g500_part* p, int64_t* out);
int g500_part_compact(g500_part* p, int64_t* num_frontier);
int g500_part_write_pred(g500_part* p, int64_t* dev_pred);
int g500_part_destroy(g500_part* p);

/* Self-test of the failure path of the bounded grid barrier (no counterpart in
 * the reference): a cooperative launch in which one block never arrives must
 * end with the others giving up (*timed_out = 1) and leave the context usable
 * for a following launch (*recovered = 1).  Causes no fault. */
int g500_selftest_barrier_timeout(int device, int* timed_out, int* recovered);

/* Validation that allocates nothing, for callers that cannot call cudaMalloc
 * (a host framework owning all device memory through its own arena or caching
 * allocator, or a serving loop that forbids allocation after start-up).  No
 * counterpart in the reference.  Same checks and results as g500_validate,
 * with every buffer passed by the caller in device memory (edges, pred) and
 * nglobalverts / nlocalverts given explicitly (main.cc:129-133 passes
 * max_used_vertex + 1 and pred_size).  Scratch is a fixed device array of
 * G500_VALIDATE_STATIC_MAX_VERTS bytes plus a few counters, held by every GPU
 * that loads the library until the process exits; larger nlocalverts is
 * refused with G500_E_RANGE.  The first call on a device resolves that
 * device's scratch address (cudaGetSymbolAddress); make that first call before
 * any stream capture.  Every call shares the same scratch: calls that overlap
 * on the GPU (e.g. on two streams) race and must be serialised by the caller.
 * stream may be NULL (the default stream); the call returns after the stream
 * has finished the validation.  The call runs on the device that is current
 * when it is made: dev_pred and dev_edges must be that device's memory
 * (otherwise G500_E_INVAL).  The scratch addresses are resolved once per device
 * and kept for the life of the library: after a cudaDeviceReset the library
 * must be unloaded and loaded again before this call is used on that device. */
#define G500_VALIDATE_STATIC_MAX_VERTS (1 << 22)
int g500_validate_noalloc(const g500_packed_edge* dev_edges, int64_t num_edges, int64_t nglobalverts,
                          int64_t nlocalverts, int64_t root, const int64_t* dev_pred, void* stream,
                          int64_t* edge_visit_count, int* ok, g500_validate_report* report);

#ifdef __cplusplus
}
#endif
#endif
