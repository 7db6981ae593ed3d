/*
 * ref_driver.cc -- a thin C entry layer over the UNMODIFIED suzumura/graph500
 * CPU path, compiled from the reference sources where they lie (the build
 * recipe is oracle/Makefile; outputs go to oracle/_ref/ only).
 *
 * TEST INFRASTRUCTURE: it generates golden fixtures (tests/golden/), pins the
 * C restatement in oracle/g500_oracle.c, and is the "reference" arm of
 * bench.py.  Nothing in the CUDA product links it.
 *
 * The call sequence mirrors mpi/main.cc:34-178 (generate -> construct ->
 * find_roots -> prepare_bfs -> run_bfs/validate per root -> end_bfs).
 * VERTEX_REORDERING and REAL_BENCHMARK are compile-time switches of the
 * reference, so one library is built per reordering mode.
 */
#include <mpi.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <inttypes.h>
#include <math.h>
#include <string>

#include "parameters.h"
#include "utils_core.h"
#include "primitives.hpp"
#include "utils.hpp"
#include "../generator/graph_generator.hpp"
#include "graph_constructor.hpp"
#include "validate.hpp"
#include "benchmark_helper.hpp"
#include "bfs.hpp"
#include "bfs_cpu.hpp"

typedef EdgeListStorage<UnweightedPackedEdge, 8 * 1024 * 1024> RefEdgeList;

static RefEdgeList* g_edges = NULL;
static BfsOnCPU* g_bfs = NULL;
static int g_scale = 0, g_ef = 0;
static bool g_setup = false;

#define REF_API extern "C" __attribute__((visibility("default")))

REF_API int ref_reordering_mode() { return VERTEX_REORDERING; }

/* setup_globals (utils.hpp:1566) + generate_graph_spec2010 (benchmark_helper.hpp:308).
 * Returns the generation wall time in seconds. */
REF_API double ref_generate(int scale, int edgefactor) {
  if (!g_setup) {
    static char arg0[] = "ref_driver";
    static char* argv[] = {arg0, NULL};
    setup_globals(1, argv, scale, edgefactor);
    g_setup = true;
  }
  g_scale = scale;
  g_ef = edgefactor;
  delete g_bfs; g_bfs = NULL;
  delete g_edges;
  g_edges = new RefEdgeList((int64_t(1) << scale) * edgefactor / mpi.size_2d, NULL);
  double t = MPI_Wtime();
  generate_graph_spec2010(g_edges, scale, edgefactor);
  return MPI_Wtime() - t;
}

/* Copies the generated packed edges [start, start+count) into out (12 bytes each). */
REF_API int64_t ref_copy_edges(void* out, int64_t start, int64_t count) {
  if (!g_edges) return -1;
  int loops = g_edges->beginRead(false);
  int64_t pos = 0, copied = 0;
  for (int l = 0; l < loops; ++l) {
    UnweightedPackedEdge* buf;
    int n = g_edges->read(&buf);
    int64_t lo = std::max<int64_t>(start, pos), hi = std::min<int64_t>(start + count, pos + n);
    if (hi > lo) {
      memcpy((char*)out + (lo - start) * sizeof(UnweightedPackedEdge), buf + (lo - pos),
             (size_t)(hi - lo) * sizeof(UnweightedPackedEdge));
      copied += hi - lo;
    }
    pos += n;
  }
  g_edges->endRead();
  return copied;
}

/* BfsBase::construct (bfs.hpp:102-113) + redistribute_edge_2d (identity on one rank). */
REF_API double ref_construct() {
  if (!g_edges) return -1;
  delete g_bfs;
  g_bfs = new BfsOnCPU();
  double t = MPI_Wtime();
  g_bfs->construct(g_edges);
  t = MPI_Wtime() - t;
  redistribute_edge_2d(g_edges);
  return t;
}

/* info: log_orig_global_verts, pred_size, num_local_verts, num_global_verts,
 * num_global_edges, max_used_vertex (same order as ORC_INFO_*). */
REF_API void ref_graph_info(int64_t* info) {
  Graph2DCSR& g = g_bfs->graph_;
  info[0] = g.log_orig_global_verts_;
  info[1] = g.pred_size();
  info[2] = g.num_local_verts_;
  info[3] = g.num_global_verts_;
  info[4] = g.num_global_edges_;
  info[5] = find_max_used_vertex(g);
}

REF_API int ref_has_edge(int64_t v) { return g_bfs->graph_.has_edge(v) ? 1 : 0; }

REF_API int ref_find_roots(int num_roots, int64_t* roots) {
  int n = num_roots;
  find_roots(g_bfs->graph_, roots, n);
  return n;
}

REF_API void ref_prepare_bfs() { g_bfs->prepare_bfs(); }

/* One timed run_bfs exactly as main.cc:111-117 times it. */
REF_API double ref_run_bfs(int64_t root, int64_t* pred) {
  MPI_Barrier(mpi.comm_2d);
  double t = MPI_Wtime();
  g_bfs->run_bfs(root, pred);
  t = MPI_Wtime() - t;
  g_bfs->get_pred(pred);
  return t;
}

/* validate_bfs_result (validate.hpp:1008-1019) with nglobalverts = max_used_vertex + 1
 * as main.cc:129-133 passes it.  Returns 1 when valid. */
REF_API int ref_validate(int64_t root, int64_t* pred, int64_t* edge_visit_count) {
  const int64_t max_used_vertex = find_max_used_vertex(g_bfs->graph_);
  const int64_t nlocalverts = g_bfs->graph_.pred_size();
  *edge_visit_count = 0;
  return validate_bfs_result(g_edges, max_used_vertex + 1, nlocalverts, root, pred, edge_visit_count) ? 1 : 0;
}

REF_API void ref_end_bfs() { g_bfs->end_bfs(); }

/* The reference's print_bfs_result (logfile.h:49-107) on given runs, to stdout. */
REF_API void ref_print_bfs_result(int n, double* bfs_times, double* validate_times, double* edge_counts, int ok) {
  print_bfs_result(n, bfs_times, validate_times, edge_counts, ok != 0);
  fflush(stdout);
}

/* generate_graph_spec2012 (benchmark_helper.hpp:316-322) into a weighted edge
 * list of its own (main.cc never calls it; the generator is compiled from the
 * reference as it stands).  max_weight is unused by the reference's constant
 * weight.  Returns the number of edges. */
typedef EdgeListStorage<WeightedEdge, 8 * 1024 * 1024> RefWeightedEdgeList;
static RefWeightedEdgeList* g_wedges = NULL;

REF_API int64_t ref_generate_spec2012(int scale, int edgefactor) {
  if (!g_setup) {
    static char arg0[] = "ref_driver";
    static char* argv[] = {arg0, NULL};
    setup_globals(1, argv, scale, edgefactor);
    g_setup = true;
  }
  delete g_wedges;
  const int64_t n = int64_t(1) << scale;
  g_wedges = new RefWeightedEdgeList(n * edgefactor + n, NULL);
  generate_graph_spec2012(g_wedges, scale, edgefactor, 255);
  int loops = g_wedges->beginRead(false);
  int64_t total = 0;
  for (int l = 0; l < loops; ++l) {
    WeightedEdge* buf;
    total += g_wedges->read(&buf);
  }
  g_wedges->endRead();
  return total;
}

/* Copies weighted edges [start, start+count) into out (16 bytes each). */
REF_API int64_t ref_copy_edges_spec2012(void* out, int64_t start, int64_t count) {
  if (!g_wedges) return -1;
  int loops = g_wedges->beginRead(false);
  int64_t pos = 0, copied = 0;
  for (int l = 0; l < loops; ++l) {
    WeightedEdge* buf;
    int n = g_wedges->read(&buf);
    int64_t lo = std::max<int64_t>(start, pos), hi = std::min<int64_t>(start + count, pos + n);
    if (hi > lo) {
      memcpy((char*)out + (lo - start) * sizeof(WeightedEdge), buf + (lo - pos),
             (size_t)(hi - lo) * sizeof(WeightedEdge));
      copied += hi - lo;
    }
    pos += n;
  }
  g_wedges->endRead();
  return copied;
}

REF_API void ref_release() {
  delete g_wedges; g_wedges = NULL;
  delete g_bfs; g_bfs = NULL;
  delete g_edges; g_edges = NULL;
}

#ifdef G500_REF_MAIN
/*
 * Stand-alone bounded benchmark of the reference path:
 *   ref_bench SCALE EDGEFACTOR NROOTS WARMUP STEPS ROOTS_PER_STEP [gate]
 * Generation, construction and validation are untimed; each step runs
 * ROOTS_PER_STEP consecutive roots (cycling over the NROOTS find_roots roots)
 * and reports per-root BFS wall times.  Output: one JSON object on stdout.
 * With "gate", the process prints "ready" on stdout once the graph is built
 * and validated, and starts the timed runs only when a line arrives on stdin
 * (so that a caller can overlap construction with other work and time the
 * runs alone); an empty stdin (EOF) ends it without timing.
 */
int main(int argc, char** argv) {
  if (argc < 7) {
    fprintf(stderr, "usage: %s SCALE EDGEFACTOR NROOTS WARMUP STEPS ROOTS_PER_STEP [gate]\n", argv[0]);
    return 2;
  }
  const bool gate = argc > 7 && strcmp(argv[7], "gate") == 0;
  int scale = atoi(argv[1]), ef = atoi(argv[2]), nroots = atoi(argv[3]);
  int warmup = atoi(argv[4]), steps = atoi(argv[5]), per_step = atoi(argv[6]);
  double gen = ref_generate(scale, ef);
  double cons = ref_construct();
  int64_t roots[64];
  if (nroots > 64) nroots = 64;
  nroots = ref_find_roots(nroots, roots);
  int64_t* pred = (int64_t*)cache_aligned_xmalloc(g_bfs->graph_.pred_size() * sizeof(int64_t));
  int64_t nedge[64];
  ref_prepare_bfs();
  double val_time = 0;
  for (int i = 0; i < nroots; ++i) {
    ref_run_bfs(roots[i], pred);
    double t = MPI_Wtime();
    if (!ref_validate(roots[i], pred, &nedge[i])) { fprintf(stderr, "reference validation failed\n"); return 1; }
    val_time += MPI_Wtime() - t;
  }
  if (gate) {
    printf("ready\n");
    fflush(stdout);
    char line[64];
    if (!fgets(line, sizeof(line), stdin)) return 0;
  }
  int k = 0;
  for (int w = 0; w < warmup; ++w)
    for (int j = 0; j < per_step; ++j, ++k) ref_run_bfs(roots[k % nroots], pred);
  printf("{\"scale\": %d, \"edgefactor\": %d, \"generation_s\": %.6f, \"construction_s\": %.6f, "
         "\"validate_total_s\": %.6f, \"threads\": %d, \"runs\": [",
         scale, ef, gen, cons, val_time, omp_get_max_threads());
  for (int s = 0; s < steps; ++s)
    for (int j = 0; j < per_step; ++j, ++k) {
      int r = k % nroots;
      double t = ref_run_bfs(roots[r], pred);
      printf("%s[%d, %" PRId64 ", %.9f, %" PRId64 "]", (s || j) ? ", " : "", s, roots[r], t, nedge[r]);
    }
  printf("]}\n");
  ref_end_bfs();
  free(pred);
  ref_release();
  return 0;
}
#endif
