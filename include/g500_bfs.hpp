// C++ drop-in for the reference's BFS object, over the C ABI of g500.h.
//
// main.cc (mpi/main.cc:34-178) drives the BFS object through
//   construct(&edge_list)            bfs.hpp:102-113
//   graph_.has_edge / pred_size /    graph_constructor.hpp:64, :101-110
//   log_orig_global_verts_
//   prepare_bfs()                    bfs.hpp:115-118
//   run_bfs(root, pred)              bfs.hpp:120, :2651-2940
//   get_pred(pred)                   bfs.hpp:122 (a no-op there too)
//   end_bfs()                        bfs.hpp:126-128
// and the helpers find_roots / find_max_used_vertex (benchmark_helper.hpp:
// 475-528) and validate_bfs_result (validate.hpp:1008-1019).  BfsOnGPU offers
// the same names with the same meaning; a failing call throws
// std::runtime_error carrying g500_last_error() (the reference aborts).
#ifndef G500_BFS_HPP
#define G500_BFS_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "g500.h"

namespace g500cpp {

inline void check(int rc) {
  if (rc != G500_OK) throw std::runtime_error(std::string("g500: ") + g500_last_error());
}

// Graph2DCSR's interface as main.cc and the helpers use it.
class Graph {
 public:
  Graph() = default;
  Graph(const Graph&) = delete;
  Graph& operator=(const Graph&) = delete;
  ~Graph() { reset(); }

  void reset() {
    if (h_) g500_graph_destroy(h_);
    h_ = nullptr;
  }
  void adopt(g500_graph* h) {
    reset();
    h_ = h;
    check(g500_graph_info_get(h_, &info_));
    log_orig_global_verts_ = (int)info_.log_orig_global_verts;
  }
  bool has_edge(int64_t v) const {
    int out = 0;
    check(g500_graph_has_edge(h_, v, &out));
    return out != 0;
  }
  int pred_size() const { return (int)info_.pred_size; }
  const g500_graph_info& info() const { return info_; }
  g500_graph* handle() const { return h_; }

  int log_orig_global_verts_ = 0;

 private:
  g500_graph* h_ = nullptr;
  g500_graph_info info_{};
};

class BfsOnGPU {
 public:
  explicit BfsOnGPU(int vertex_reordering = 2, int device = 0) : reorder_(vertex_reordering), device_(device) {}
  BfsOnGPU(const BfsOnGPU&) = delete;
  BfsOnGPU& operator=(const BfsOnGPU&) = delete;
  ~BfsOnGPU() { end_bfs(); }

  // construct(&edge_list): packed edges in host memory (the reference's
  // UnweightedPackedEdge layout); the edge list is kept on the device for
  // validate_bfs_result.
  void construct(const g500_packed_edge* edges, int64_t num_edges) {
    g500_graph* h = nullptr;
    check(g500_graph_build(edges, num_edges, 0, reorder_, 1, device_, &h));
    graph_.adopt(h);
  }
  // generate_graph_spec2010 + construct, both on the device.
  void generate_and_construct(int scale, int edgefactor, uint64_t seed1 = 2, uint64_t seed2 = 3) {
    g500_graph* h = nullptr;
    check(g500_graph_generate(scale, edgefactor, seed1, seed2, reorder_, device_, &h));
    graph_.adopt(h);
  }
  void prepare_bfs() {
    if (!b_) check(g500_bfs_create(graph_.handle(), &b_));
  }
  // Writes every pred entry (host memory): parent | level << 48, root = root, -1 unreached.
  void run_bfs(int64_t root, int64_t* pred, g500_bfs_stats* stats = nullptr) {
    check(g500_bfs_run(b_, root, pred, 0, stats));
  }
  void get_pred(int64_t*) {}
  void end_bfs() {
    if (b_) g500_bfs_destroy(b_);
    b_ = nullptr;
  }
  // Autotune the direction switch on sample roots (untimed; the reference
  // reads fixed denominators from parameters.h:87-88).
  g500_tune_result autotune(const int64_t* roots, int n, int reps = 2) {
    g500_tune_result r{};
    check(g500_bfs_autotune(b_, roots, n, reps, &r));
    return r;
  }
  g500_bfs* handle() const { return b_; }

  Graph graph_;

 private:
  int reorder_;
  int device_;
  g500_bfs* b_ = nullptr;
};

inline void find_roots(const Graph& g, int64_t* roots, int& num_roots, uint64_t seed1 = 2, uint64_t seed2 = 3) {
  int found = 0;
  check(g500_graph_find_roots(g.handle(), num_roots, seed1, seed2, roots, &found));
  num_roots = found;
}

inline int64_t find_max_used_vertex(const Graph& g) { return g.info().max_used_vertex; }

// validate_bfs_result against the graph's device-resident edge list.
inline bool validate_bfs_result(const Graph& g, int64_t root, const int64_t* pred, int64_t* edge_visit_count,
                                g500_validate_report* report = nullptr) {
  int ok = 0;
  check(g500_validate(g.handle(), nullptr, 0, 1, root, pred, 0, edge_visit_count, &ok, report));
  return ok != 0;
}

}  // namespace g500cpp

#endif  // G500_BFS_HPP
