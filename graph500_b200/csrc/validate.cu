// Graph500 result validation on the device: BfsValidation::validate
// (mpi/validate.hpp:506-802) for one rank.
//
//   vertex pass  -- check_value_ranges (:822-839), root is its own parent
//                   (:529-537), no other self parent (:542-571), and
//                   check_bfs_depth_map_using_predecessors (:920-995)
//   edge pass    -- every input edge: both ends in or both out of the tree,
//                   |depth difference| <= 1, count edge_visit_count, and mark
//                   vertices whose parent edge appears (:598-776)
//   parent pass  -- every reached non-root vertex has an input edge to its
//                   parent (:780-792)
//
// The reference stops after the first failing stage; this version computes
// every stage (guarding the reads an out-of-range parent would make) and
// reports per-stage error counts.  The result is valid iff all are zero.
#include "g500_internal.cuh"

#include <algorithm>
#include <mutex>

namespace g500 {

enum { VE_RANGE, VE_ROOT, VE_SELF, VE_DEPTH, VE_EDGE, VE_MISSING, VE_COUNT_EDGES, VE_N };

__device__ __forceinline__ int64_t pred_of(int64_t e) { return (int64_t)((uint64_t)e << 16) >> 16; }  // :809
__device__ __forceinline__ int depth_of(int64_t e) { return (int)((e >> 48) & 0xFFFF); }              // :813

__device__ __forceinline__ void warp_add(unsigned long long* dst, unsigned long long v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

__global__ void val_vertex_kernel(const int64_t* __restrict__ pred, int64_t nlocal, int64_t nglobal, int64_t root,
                                  unsigned long long* err) {
  unsigned long long range = 0, self = 0, depth = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nlocal; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = pred[i];
    const int64_t p = pred_of(e);
    const int d = depth_of(e);
    if (p < -1 || p >= nglobal) {
      ++range;
      continue;
    }
    if (i != root && p != -1 && p == i) ++self;
    if (p == -1 && d != 0xFFFF) ++depth;
    else if (p != -1 && d == 0xFFFF) ++depth;
    if (i != root && p != -1) {
      const int64_t pp = pred[p];  // p in [0, nglobal) and nglobal <= nlocal
      if (depth_of(pp) == 0xFFFF) ++depth;
      if (d != depth_of(pp) + 1) ++depth;
    }
  }
  warp_add(&err[VE_RANGE], range);
  warp_add(&err[VE_SELF], self);
  warp_add(&err[VE_DEPTH], depth);
}

// validate.hpp:513-515 only reports a root outside [0, nglobalverts); its
// pred entry then fails the range check.  A root outside pred[] is refused.
__global__ void val_root_kernel(const int64_t* __restrict__ pred, int64_t root, int64_t nlocal,
                                unsigned long long* err) {
  if (root < 0 || root >= nlocal) {
    atomicAdd(&err[VE_ROOT], 1ull);
    return;
  }
  const int64_t e = pred[root];
  if (pred_of(e) != root) atomicAdd(&err[VE_ROOT], 1ull);
  if (depth_of(e) != 0) atomicAdd(&err[VE_DEPTH], 1ull);
}

__device__ __forceinline__ int64_t ev0(const g500_packed_edge& e) {
  return (int64_t)e.v0_low | ((int64_t)(e.high & 0xFFFF) << 32);
}
__device__ __forceinline__ int64_t ev1(const g500_packed_edge& e) {
  return (int64_t)e.v1_low | ((int64_t)(e.high >> 16) << 32);
}

__global__ void val_edge_kernel(const g500_packed_edge* __restrict__ edges, int64_t m,
                                const int64_t* __restrict__ pred, int64_t nlocal, uint8_t* valid,
                                unsigned long long* err) {
  unsigned long long bad = 0, count = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const g500_packed_edge ed = edges[i];
    const int64_t src = ev0(ed), tgt = ev1(ed);
    if (src >= nlocal || tgt >= nlocal) {
      ++bad;
      continue;
    }
    const int64_t ps = pred[src], pt = pred[tgt];
    const int sd = depth_of(ps), td = depth_of(pt);
    if (sd != 0xFFFF && td == 0xFFFF) ++bad;
    else if (sd == 0xFFFF && td != 0xFFFF) ++bad;
    else if (sd - td < -1 || sd - td > 1) ++bad;
    else if (sd != 0xFFFF) ++count;
    if (pred_of(ps) == tgt) valid[src] = 1;
    if (pred_of(pt) == src) valid[tgt] = 1;
  }
  warp_add(&err[VE_EDGE], bad);
  warp_add(&err[VE_COUNT_EDGES], count);
}

__global__ void val_parent_kernel(const int64_t* __restrict__ pred, int64_t nlocal, int64_t root,
                                  const uint8_t* __restrict__ valid, unsigned long long* err) {
  unsigned long long missing = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nlocal; i += (int64_t)gridDim.x * blockDim.x) {
    if (i == root || pred_of(pred[i]) == -1) continue;
    if (!valid[i]) ++missing;
  }
  warp_add(&err[VE_MISSING], missing);
}

}  // namespace g500

using namespace g500;

extern "C" int g500_validate(g500_graph* g, const g500_packed_edge* edges, int64_t m, int edges_on_device,
                             int64_t root, const int64_t* pred, int pred_on_device, int64_t* edge_visit_count,
                             int* ok, g500_validate_report* report) {
  if (!g || !pred || !ok) return set_error(G500_E_INVAL, "null argument");
  if (!edges) {
    if (!g->d_edges) return set_error(G500_E_STATE, "graph keeps no edge list; pass one");
    edges = g->d_edges;
    m = g->num_edges;
    edges_on_device = 1;
  }
  G500_CUDA(cudaSetDevice(g->device));
  cudaStream_t s = g->stream;
  const int64_t nlocal = g->nolv;
  const int64_t nglobal = g->max_used_vertex + 1;  // main.cc:129-133
  std::vector<void*> owned;
  auto cleanup = [&]() {
    for (void* p : owned) dev_free(p);
  };
  const int64_t* d_pred = pred;
  const g500_packed_edge* d_edges = edges;
  int st = G500_OK;
  if (!pred_on_device) {
    int64_t* p = nullptr;
    st = dev_alloc_n(&p, nlocal, "validation pred copy");
    if (st != G500_OK) return st;
    owned.push_back(p);
    cudaError_t e = cudaMemcpyAsync(p, pred, sizeof(int64_t) * nlocal, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { cleanup(); return cuda_error(e, "cudaMemcpyAsync(pred)", __FILE__, __LINE__); }
    d_pred = p;
  }
  if (!edges_on_device && m > 0) {
    g500_packed_edge* p = nullptr;
    st = dev_alloc_n(&p, m, "validation edge copy");
    if (st != G500_OK) { cleanup(); return st; }
    owned.push_back(p);
    cudaError_t e = cudaMemcpyAsync(p, edges, sizeof(g500_packed_edge) * m, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { cleanup(); return cuda_error(e, "cudaMemcpyAsync(edges)", __FILE__, __LINE__); }
    d_edges = p;
  }
  unsigned long long* d_err = nullptr;
  uint8_t* d_valid = nullptr;
  st = dev_alloc_n(&d_err, VE_N, "validation counters");
  if (st == G500_OK) owned.push_back(d_err);
  if (st == G500_OK) st = dev_alloc_n(&d_valid, nlocal, "pred_valid");
  if (st == G500_OK) owned.push_back(d_valid);
  if (st != G500_OK) { cleanup(); return st; }
  cudaError_t e = cudaMemsetAsync(d_err, 0, sizeof(unsigned long long) * VE_N, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_valid, 0, (size_t)nlocal, s);
  if (e != cudaSuccess) { cleanup(); return cuda_error(e, "cudaMemsetAsync", __FILE__, __LINE__); }
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(std::max<int64_t>(nlocal, m), 256),
                                                    (int64_t)num_sms() * 16);
  val_root_kernel<<<1, 1, 0, s>>>(d_pred, root, nlocal, d_err);
  val_vertex_kernel<<<grid, 256, 0, s>>>(d_pred, nlocal, nglobal, root, d_err);
  if (m > 0) val_edge_kernel<<<grid, 256, 0, s>>>(d_edges, m, d_pred, nlocal, d_valid, d_err);
  val_parent_kernel<<<grid, 256, 0, s>>>(d_pred, nlocal, root, d_valid, d_err);
  e = cudaGetLastError();
  unsigned long long h[VE_N];
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_err, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cleanup();
  if (e != cudaSuccess) return cuda_error(e, "validation", __FILE__, __LINE__);
  g500_validate_report r;
  r.range_errors = (int64_t)h[VE_RANGE];
  r.root_errors = (int64_t)h[VE_ROOT];
  r.self_parent_errors = (int64_t)h[VE_SELF];
  r.depth_errors = (int64_t)h[VE_DEPTH];
  r.edge_errors = (int64_t)h[VE_EDGE];
  r.missing_parent_edge_errors = (int64_t)h[VE_MISSING];
  const bool valid = !(r.range_errors || r.root_errors || r.self_parent_errors || r.depth_errors ||
                       r.edge_errors || r.missing_parent_edge_errors);
  *ok = valid ? 1 : 0;
  if (edge_visit_count) *edge_visit_count = valid ? (int64_t)h[VE_COUNT_EDGES] : 0;
  if (report) *report = r;
  return G500_OK;
}

// ---------------------------------------------------------------------------
// Validation that allocates nothing.
//
// Some callers cannot call cudaMalloc: a host framework that owns all device
// memory through its own arena or caching allocator, or a serving loop that
// forbids allocation once it has started.  For them the scratch of the
// validator (one flag byte per vertex and the error counters) lives in
// file-scope device arrays of a fixed size, held by every GPU that loads the
// library until the process exits.  Host code cannot use the arrays' names as
// device addresses, so each device's addresses are fetched once with
// cudaGetSymbolAddress, with that device current.
// ---------------------------------------------------------------------------
namespace g500 {

static __device__ __align__(256) uint8_t g_static_valid[G500_VALIDATE_STATIC_MAX_VERTS];
static __device__ __align__(256) unsigned long long g_static_err[VE_N];

struct StaticScratch {
  uint8_t* valid = nullptr;
  unsigned long long* err = nullptr;
};
static StaticScratch g_static_scratch[64];
static std::mutex g_static_mu;

// G500_OK when p is device (or managed) memory of device dev.
static int on_device(const void* p, int dev, const char* what) {
  cudaPointerAttributes a;
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(G500_E_INVAL, "%s: not a CUDA pointer (%s)", what, cudaGetErrorString(e));
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
    return set_error(G500_E_INVAL, "%s is not in device memory", what);
  if (a.type == cudaMemoryTypeDevice && a.device != dev)
    return set_error(G500_E_INVAL, "%s is on device %d, but device %d is current; make the device that holds the "
                     "buffers current before the call", what, a.device, dev);
  return G500_OK;
}

// Resolve this device's scratch addresses (first call on a device only).
static int static_scratch(int dev, StaticScratch* out) {
  if (dev < 0 || dev >= 64) return set_error(G500_E_INVAL, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_static_mu);
  StaticScratch& s = g_static_scratch[dev];
  if (!s.valid) {
    void* v = nullptr;
    void* e = nullptr;
    G500_CUDA(cudaGetSymbolAddress(&v, g_static_valid));
    G500_CUDA(cudaGetSymbolAddress(&e, g_static_err));
    s.valid = static_cast<uint8_t*>(v);
    s.err = static_cast<unsigned long long*>(e);
  }
  *out = s;
  return G500_OK;
}

}  // namespace g500

extern "C" int g500_validate_noalloc(const g500_packed_edge* dev_edges, int64_t num_edges, int64_t nglobalverts,
                                     int64_t nlocalverts, int64_t root, const int64_t* dev_pred, void* stream,
                                     int64_t* edge_visit_count, int* ok, g500_validate_report* report) {
  if (!dev_pred || !ok || (num_edges > 0 && !dev_edges)) return set_error(G500_E_INVAL, "null argument");
  if (num_edges < 0 || nlocalverts <= 0 || nglobalverts < 0 || nglobalverts > nlocalverts)
    return set_error(G500_E_INVAL, "bad sizes (num_edges %lld, nglobalverts %lld, nlocalverts %lld)",
                     (long long)num_edges, (long long)nglobalverts, (long long)nlocalverts);
  if (nlocalverts > G500_VALIDATE_STATIC_MAX_VERTS)
    return set_error(G500_E_RANGE, "g500_validate_noalloc handles at most %d vertices (pred_size %lld); "
                     "use g500_validate", G500_VALIDATE_STATIC_MAX_VERTS, (long long)nlocalverts);
  int dev = 0;
  G500_CUDA(cudaGetDevice(&dev));
  // the scratch and the kernels belong to the current device: pred and the
  // edge list must live there too (a peer's or a host pointer is refused)
  G500_TRY(on_device(dev_pred, dev, "pred"));
  if (num_edges > 0) G500_TRY(on_device(dev_edges, dev, "edge list"));
  StaticScratch sc;
  G500_TRY(static_scratch(dev, &sc));
  cudaStream_t s = (cudaStream_t)stream;
  // the arrays keep the last call's contents: clear what must start at zero
  G500_CUDA(cudaMemsetAsync(sc.err, 0, sizeof(unsigned long long) * VE_N, s));
  G500_CUDA(cudaMemsetAsync(sc.valid, 0, (size_t)nlocalverts, s));
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(std::max<int64_t>(nlocalverts, num_edges), 256),
                                                    (int64_t)num_sms() * 16);
  val_root_kernel<<<1, 1, 0, s>>>(dev_pred, root, nlocalverts, sc.err);
  val_vertex_kernel<<<grid, 256, 0, s>>>(dev_pred, nlocalverts, nglobalverts, root, sc.err);
  if (num_edges > 0) val_edge_kernel<<<grid, 256, 0, s>>>(dev_edges, num_edges, dev_pred, nlocalverts, sc.valid, sc.err);
  val_parent_kernel<<<grid, 256, 0, s>>>(dev_pred, nlocalverts, root, sc.valid, sc.err);
  G500_CUDA(cudaGetLastError());
  unsigned long long h[VE_N];
  G500_CUDA(cudaMemcpyAsync(h, sc.err, sizeof(h), cudaMemcpyDeviceToHost, s));
  G500_CUDA(cudaStreamSynchronize(s));
  g500_validate_report r;
  r.range_errors = (int64_t)h[VE_RANGE];
  r.root_errors = (int64_t)h[VE_ROOT];
  r.self_parent_errors = (int64_t)h[VE_SELF];
  r.depth_errors = (int64_t)h[VE_DEPTH];
  r.edge_errors = (int64_t)h[VE_EDGE];
  r.missing_parent_edge_errors = (int64_t)h[VE_MISSING];
  const bool valid = !(r.range_errors || r.root_errors || r.self_parent_errors || r.depth_errors ||
                       r.edge_errors || r.missing_parent_edge_errors);
  *ok = valid ? 1 : 0;
  if (edge_visit_count) *edge_visit_count = valid ? (int64_t)h[VE_COUNT_EDGES] : 0;
  if (report) *report = r;
  return G500_OK;
}
