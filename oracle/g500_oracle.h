/*
 * g500_oracle.h -- CPU restatement of the Graph500 BFS hot path of the
 * suzumura/graph500 reference.
 *
 * THIS IS TEST INFRASTRUCTURE.  It is the checker the parity tests, smoke()
 * and the CPU-baseline leg of bench.py compare the CUDA path against.  No
 * product code path links, loads or calls it.
 *
 * Every function cites the reference file:line it restates.  Parity of this
 * restatement is pinned two ways (see tests/test_oracle_golden.py):
 *   - the reference's own known-answer table pf_nedge[] (mpi/utils.hpp:3663-3707),
 *   - fixtures produced by the unmodified reference compiled here against a
 *     single-rank MPI stand-in (oracle/ref_driver.cc, tests/golden/make_golden.py).
 */
#ifndef G500_ORACLE_H
#define G500_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- splittable MRG (generator/splittable_mrg.[ch], mod_arith_64bit.h) ---- */
typedef struct orc_mrg_state { uint32_t z1, z2, z3, z4, z5; } orc_mrg_state;

void     orc_make_mrg_seed(uint64_t userseed1, uint64_t userseed2, orc_mrg_state* st);
void     orc_mrg_skip(orc_mrg_state* st, uint64_t exp_high, uint64_t exp_mid, uint64_t exp_low);
uint32_t orc_mrg_get_uint_orig(orc_mrg_state* st);
double   orc_mrg_get_double_orig(orc_mrg_state* st);
void     orc_make_random_numbers(int64_t nvalues, uint64_t userseed1, uint64_t userseed2,
                                 int64_t position, double* result);
/* 5x5 transition matrix A^(val * 256^byte_index), row-major, entries < 2^31-1. */
void     orc_mrg_skip_matrix(int byte_index, int val, uint32_t out[25]);

/* ---- Kronecker generator (generator/graph_generator.hpp:327-705) ---- */
typedef struct orc_packed_edge { uint32_t v0_low, v1_low, high; } orc_packed_edge;

int64_t  orc_edge_v0(const orc_packed_edge* e);
int64_t  orc_edge_v1(const orc_packed_edge* e);
void     orc_scramble_values(int scale, uint64_t userseed1, uint64_t userseed2,
                             uint64_t* val0, uint64_t* val1);
int64_t  orc_scramble(int64_t v, int scale, uint64_t val0, uint64_t val1);
/* Edges [start, end) of the spec-2010 R-MAT graph (A=.57, B=C=.19), written
 * to out[0 .. end-start).  OpenMP parallel over edge indices. */
void     orc_generate_edges(int scale, int edgefactor, uint64_t userseed1, uint64_t userseed2,
                            int64_t start, int64_t end, orc_packed_edge* out);
/* WeightedEdge, mpi/primitives.hpp:87-106 */
typedef struct orc_weighted_edge { uint32_t v0_low, v1_low, high; int32_t weight; } orc_weighted_edge;
void     orc_generate_edges_spec2012(int scale, int edgefactor, uint64_t userseed1, uint64_t userseed2,
                                     int64_t start, int64_t end, orc_weighted_edge* out);

/* ---- graph construction (mpi/graph_constructor.hpp, one rank) ---- */
typedef struct orc_graph orc_graph;

enum {
  ORC_INFO_LOG_ORIG_GLOBAL_VERTS = 0, /* estimated SCALE */
  ORC_INFO_NUM_ORIG_LOCAL_VERTS,      /* pred_size() */
  ORC_INFO_NUM_LOCAL_VERTS,           /* reordered vertex range (multiple of 65536) */
  ORC_INFO_NUM_GLOBAL_VERTS,          /* vertices with >= 1 non-self-loop edge */
  ORC_INFO_NUM_GLOBAL_EDGES,          /* directed CSR entries after dedup */
  ORC_INFO_MAX_USED_VERTEX,           /* find_max_used_vertex() */
  ORC_INFO_COUNT
};

orc_graph* orc_graph_build(const orc_packed_edge* edges, int64_t m, int reorder_mode);
void       orc_graph_free(orc_graph* g);
void       orc_graph_info(const orc_graph* g, int64_t info[ORC_INFO_COUNT]);
/* Views (owned by the graph):
 *   offsets[num_local_verts+1] (uint64), cols[num_global_edges] (uint32, reordered ids,
 *   each row ascending, no duplicates, no self loops), reorder_map/invert_map
 *   [num_orig_local_verts], degree[num_orig_local_verts] (non-self-loop endpoint
 *   occurrences incl. duplicates, by ORIGINAL id). */
const uint64_t* orc_graph_offsets(const orc_graph* g);
const uint32_t* orc_graph_cols(const orc_graph* g);
const uint32_t* orc_graph_reorder_map(const orc_graph* g);
const uint32_t* orc_graph_invert_map(const orc_graph* g);
const int64_t*  orc_graph_degree(const orc_graph* g);
int             orc_graph_has_edge(const orc_graph* g, int64_t v);

/* ---- roots (mpi/benchmark_helper.hpp:475-528) ---- */
int     orc_find_roots(const orc_graph* g, int num_roots, uint64_t userseed1, uint64_t userseed2,
                       int64_t* roots);
int64_t orc_find_max_used_vertex(const orc_graph* g);

/* ---- BFS ---- */
/* Distances from root, indexed by ORIGINAL id; 0xFFFF for unreached. */
void orc_bfs_levels(const orc_graph* g, int64_t root, uint16_t* levels);
/* A valid Graph500 predecessor map (parent | level << 48, -1 unreached). */
void orc_bfs_pred(const orc_graph* g, int64_t root, int64_t* pred);

/* Direction-optimizing schedule of mpi/bfs.hpp:2651-2940 replayed on the CSR,
 * with the per-level counts of the algorithmic-bytes model. */
typedef struct orc_level_stats {
  int32_t  direction;       /* 1 = top-down, 0 = bottom-up */
  int32_t  pad;
  int64_t  frontier;        /* |F| (TD) : vertices at level-1 */
  int64_t  discovered;      /* |D| : vertices found at this level */
  int64_t  scanned;         /* U (BU) : unvisited vertices with edges at level start */
  int64_t  edge_sectors;    /* TD: sum ceil(deg(u)/8); BU: sum ceil(k_v/8) */
  int64_t  edges_examined;  /* TD: sum deg(u); BU: sum k_v */
} orc_level_stats;
int orc_dobfs_schedule(const orc_graph* g, int64_t root, double alpha, double beta,
                       orc_level_stats* out, int max_levels);

/* ---- validation (mpi/validate.hpp:506-995, one rank) ---- */
typedef struct orc_validate_report {
  int64_t range_errors;
  int64_t root_errors;
  int64_t self_parent_errors;
  int64_t depth_errors;
  int64_t edge_errors;
  int64_t missing_parent_edge_errors;
} orc_validate_report;
int orc_validate(const orc_packed_edge* edges, int64_t m, int64_t nglobalverts,
                 int64_t nlocalverts, int64_t root, const int64_t* pred,
                 int64_t* edge_visit_count, orc_validate_report* report);

/* ---- result statistics (mpi/logfile.h:19-44) ---- */
enum { ORC_S_MIN, ORC_S_Q1, ORC_S_MEDIAN, ORC_S_Q3, ORC_S_MAX, ORC_S_MEAN, ORC_S_STD, ORC_S_LAST };
void orc_statistics(const double* x, int n, double r[ORC_S_LAST]);

#ifdef __cplusplus
}
#endif
#endif
