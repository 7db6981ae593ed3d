// Graph construction on the device: the one-rank restatement of
// GraphConstructor2DCSR::construct (mpi/graph_constructor.hpp:554-574).
//
//   searchMaxVertex (:735-763)        -> or_reduce_kernel
//   DegreeCalculation::calc_degree    -> degree_kernel + reorder by radix sort
//     (:296-352, VERTEX_REORDERING 0/1/2; ties ordered by original id)
//   scatterAndStore + sortEdges       -> one (src, tgt) key per direction,
//     (:1183-1280, :1363-1442)           radix sort, duplicate drop, compaction
//   constructFromWideCSR (:881-990)   -> offsets = prefix sum of row lengths
//   isolateFirstEdge (:845-879)       -> first[] = first neighbour of each row
//   computeNumVertices (:1444-1464)   -> has-edge bitmap, num_global_verts
//
// Layout in HBM (reordered ids r in [0, num_local_verts)):
//   offsets u64[nlv+1], cols u32[nge] (ascending per row), first u32[nlv],
//   reorder/invert u32[pred_size], vis_init u32[nlv/32] (= ~has_edge),
//   endp u32[pred_size] (input endpoint occurrences, by reordered id).
#include "g500_internal.cuh"

#include <algorithm>
#include <chrono>

namespace g500 {

__device__ __forceinline__ int64_t edge_v0(const g500_packed_edge& e) {
  return (int64_t)e.v0_low | ((int64_t)(e.high & 0xFFFF) << 32);
}
__device__ __forceinline__ int64_t edge_v1(const g500_packed_edge& e) {
  return (int64_t)e.v1_low | ((int64_t)(e.high >> 16) << 32);
}

__global__ void or_reduce_kernel(const g500_packed_edge* __restrict__ edges, int64_t m,
                                 unsigned long long* out) {
  unsigned long long acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    g500_packed_edge e = edges[i];
    acc |= (unsigned long long)(edge_v0(e) | edge_v1(e));
  }
  unsigned lo = __reduce_or_sync(FULL_MASK, (unsigned)acc);
  unsigned hi = __reduce_or_sync(FULL_MASK, (unsigned)(acc >> 32));
  if ((threadIdx.x & 31) == 0) atomicOr(out, ((unsigned long long)hi << 32) | lo);
}

// degree = non-self-loop endpoint occurrences, duplicates included
// (graph_constructor.hpp:249-278, :312-316); self loops counted apart.
__global__ void degree_kernel(const g500_packed_edge* __restrict__ edges, int64_t m, uint32_t* deg,
                              uint32_t* selfloops) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    g500_packed_edge e = edges[i];
    int64_t a = edge_v0(e), b = edge_v1(e);
    if (a == b) {
      atomicAdd(&selfloops[a], 1u);
    } else {
      atomicAdd(&deg[a], 1u);
      atomicAdd(&deg[b], 1u);
    }
  }
}

// max degree, count of vertices with edges, last vertex with edges
__global__ void degree_summary_kernel(const uint32_t* __restrict__ deg, int64_t n, unsigned* maxdeg,
                                      unsigned long long* nnz, unsigned long long* last_plus1) {
  unsigned mx = 0;
  unsigned long long cnt = 0, last = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    unsigned d = deg[i];
    mx = max(mx, d);
    if (d) {
      ++cnt;
      last = max(last, (unsigned long long)i + 1);
    }
  }
  mx = __reduce_max_sync(FULL_MASK, mx);
  for (int o = 16; o; o >>= 1) {
    cnt += __shfl_xor_sync(FULL_MASK, cnt, o);
    last = max(last, __shfl_xor_sync(FULL_MASK, last, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(maxdeg, mx);
    atomicAdd(nnz, cnt);
    atomicMax(last_plus1, last);
  }
}

// reorder keys: VR2 -> (maxdeg - deg) in the high word (degree descending),
// VR1 -> (deg == 0) in the high word; the low word is the original id, so a
// stable sort leaves ties in ascending original id.
__global__ void reorder_keys_kernel(const uint32_t* __restrict__ deg, int64_t n, int mode, unsigned maxdeg,
                                    uint64_t* keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t hi = (mode == 2) ? (uint64_t)(maxdeg - deg[i]) : (uint64_t)(deg[i] == 0);
    keys[i] = (hi << 32) | (uint64_t)i;
  }
}

__global__ void maps_from_keys_kernel(const uint64_t* __restrict__ keys, int64_t n, uint32_t* invert,
                                      uint32_t* reorder) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t v = keys ? (uint32_t)keys[i] : (uint32_t)i;
    invert[i] = v;
    reorder[v] = (uint32_t)i;
  }
}

// one key per direction of every non-self-loop edge: (r(src) << lb) | r(tgt);
// self loops become ~0, which sorts last and is dropped.
__global__ void edge_keys_kernel(const g500_packed_edge* __restrict__ edges, int64_t m,
                                 const uint32_t* __restrict__ reorder, int lb, uint64_t* keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    g500_packed_edge e = edges[i];
    int64_t a = edge_v0(e), b = edge_v1(e);
    uint64_t k0 = ~0ull, k1 = ~0ull;
    if (a != b) {
      uint64_t ra = reorder[a], rb = reorder[b];
      k0 = (ra << lb) | rb;
      k1 = (rb << lb) | ra;
    }
    keys[2 * i] = k0;
    keys[2 * i + 1] = k1;
  }
}

constexpr int CP_THREADS = 256;
constexpr int CP_ITEMS = 8;
constexpr int CP_TILE = CP_THREADS * CP_ITEMS;

__device__ __forceinline__ bool key_is_new(const uint64_t* __restrict__ k, int64_t i) {
  uint64_t v = k[i];
  return v != ~0ull && (i == 0 || k[i - 1] != v);
}

// pass 1 of the duplicate drop: unique keys per tile and per row
__global__ void __launch_bounds__(CP_THREADS) unique_count_kernel(const uint64_t* __restrict__ k, int64_t n, int lb,
                                                                  uint32_t* tile_counts, uint32_t* rowcnt) {
  __shared__ uint32_t sh;
  if (threadIdx.x == 0) sh = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * CP_TILE;
  const int lane = threadIdx.x & 31;
  uint32_t c = 0;
#pragma unroll
  for (int j = 0; j < CP_ITEMS; ++j) {
    int64_t i = base + j * CP_THREADS + threadIdx.x;
    bool u = i < n && key_is_new(k, i);
    c += u;
    // one atomic per run of equal rows inside the warp
    uint32_t row = u ? (uint32_t)(k[i] >> lb) : 0xFFFFFFFFu;
    unsigned peers = __match_any_sync(FULL_MASK, row);
    if (u && (__ffs(peers) - 1) == lane) atomicAdd(&rowcnt[row], (unsigned)__popc(peers));
  }
  c = __reduce_add_sync(FULL_MASK, c);
  if (lane == 0) atomicAdd(&sh, c);
  __syncthreads();
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = sh;
}

// pass 2: write the unique targets in order
__global__ void __launch_bounds__(CP_THREADS) unique_write_kernel(const uint64_t* __restrict__ k, int64_t n, int lb,
                                                                  const uint64_t* __restrict__ tile_offsets,
                                                                  uint32_t* cols) {
  __shared__ uint32_t warp_tot[CP_THREADS / 32];
  const int64_t base = (int64_t)blockIdx.x * CP_TILE;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // thread t owns the contiguous run [base + t*ITEMS, +ITEMS) so order is kept
  bool u[CP_ITEMS];
  uint32_t c = 0;
#pragma unroll
  for (int j = 0; j < CP_ITEMS; ++j) {
    int64_t i = base + (int64_t)threadIdx.x * CP_ITEMS + j;
    u[j] = i < n && key_is_new(k, i);
    c += u[j];
  }
  uint32_t x = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(FULL_MASK, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  uint32_t wp = 0;
  for (int w = 0; w < warp; ++w) wp += warp_tot[w];
  uint64_t pos = tile_offsets[blockIdx.x] + wp + x - c;
  const uint64_t mask = (lb >= 64) ? ~0ull : ((1ull << lb) - 1);
#pragma unroll
  for (int j = 0; j < CP_ITEMS; ++j) {
    if (u[j]) cols[pos++] = (uint32_t)(k[base + (int64_t)threadIdx.x * CP_ITEMS + j] & mask);
  }
}

__global__ void finish_rows_kernel(const uint64_t* __restrict__ offsets, const uint32_t* __restrict__ cols,
                                   int64_t nlv, int flags, uint32_t* first, uint32_t* vis_init) {
  const int lane = threadIdx.x & 31;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nlv; v += (int64_t)gridDim.x * blockDim.x) {
    uint64_t b = offsets[v], e = offsets[v + 1];
    first[v] = e > b ? (cols[b] | (flags && e - b > 1 ? FIRST_MORE : 0u)) : NO_VERTEX;
    unsigned none = __ballot_sync(FULL_MASK, e == b);  // nlv is a multiple of 32
    if (lane == 0) vis_init[v >> 5] = none;
  }
}

__global__ void endp_kernel(const uint32_t* __restrict__ deg, const uint32_t* __restrict__ sl,
                            const uint32_t* __restrict__ invert, int64_t n, uint32_t* endp) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    uint32_t v = invert[r];
    endp[r] = deg[v] + 2u * sl[v];
  }
}

__global__ void has_edge_orig_kernel(const uint32_t* __restrict__ deg, int64_t n, uint32_t* bits) {
  const int lane = threadIdx.x & 31;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    unsigned b = __ballot_sync(FULL_MASK, deg[v] != 0);  // n is a multiple of 32
    if (lane == 0) bits[v >> 5] = b;
  }
}

static inline unsigned grid_for(int64_t n, int threads = 256) {
  int64_t b = ceil_div(std::max<int64_t>(n, 1), threads);
  return (unsigned)std::min<int64_t>(b, (int64_t)num_sms() * 16);
}

// Scoped device buffers freed on every exit path.
struct Scratch {
  std::vector<void*> ptrs;
  ~Scratch() {
    for (void* p : ptrs) dev_free(p);
  }
  template <typename T>
  int alloc(T** p, int64_t n, const char* what) {
    G500_TRY(dev_alloc_n(p, n, what));
    ptrs.push_back(*p);
    return G500_OK;
  }
};

int graph_destroy_internal(g500_graph* g);

static int build_from_device_edges(g500_graph* g, const g500_packed_edge* d_edges, int64_t m) {
  cudaStream_t s = g->stream;
  Scratch tmp;
  unsigned long long* d_scalars = nullptr;  // [0] or, [1] nnz, [2] last+1, [3] maxdeg
  G500_TRY(tmp.alloc(&d_scalars, 4, "construction scalars"));
  G500_CUDA(cudaMemsetAsync(d_scalars, 0, 4 * sizeof(unsigned long long), s));

  // searchMaxVertex
  or_reduce_kernel<<<grid_for(m), 256, 0, s>>>(d_edges, m, d_scalars);
  G500_CUDA(cudaGetLastError());
  unsigned long long orv = 0;
  G500_CUDA(cudaMemcpyAsync(&orv, d_scalars, sizeof(orv), cudaMemcpyDeviceToHost, s));
  G500_CUDA(cudaStreamSynchronize(s));
  const int log_max = orv ? msb_index(orv) + 1 : 0;
  if (log_max > 32) return set_error(G500_E_RANGE, "vertex ids need %d bits; 32 supported", log_max);
  g->log_orig_global_verts = log_max;
  g->nolv = roundup(int64_t(1) << log_max, LOCAL_VERTS_UNIT);
  const int64_t nolv = g->nolv;

  // degrees
  uint32_t *deg = nullptr, *sl = nullptr;
  G500_TRY(tmp.alloc(&deg, nolv, "degree"));
  G500_TRY(tmp.alloc(&sl, nolv, "self loops"));
  G500_CUDA(cudaMemsetAsync(deg, 0, sizeof(uint32_t) * nolv, s));
  G500_CUDA(cudaMemsetAsync(sl, 0, sizeof(uint32_t) * nolv, s));
  degree_kernel<<<grid_for(m), 256, 0, s>>>(d_edges, m, deg, sl);
  G500_CUDA(cudaGetLastError());
  unsigned* d_maxdeg = reinterpret_cast<unsigned*>(d_scalars + 3);
  degree_summary_kernel<<<grid_for(nolv), 256, 0, s>>>(deg, nolv, d_maxdeg, d_scalars + 1, d_scalars + 2);
  G500_CUDA(cudaGetLastError());
  unsigned long long sc[4];
  G500_CUDA(cudaMemcpyAsync(sc, d_scalars, sizeof(sc), cudaMemcpyDeviceToHost, s));
  G500_CUDA(cudaStreamSynchronize(s));
  const int64_t nnz = (int64_t)sc[1];
  const unsigned maxdeg = (unsigned)(sc[3] & 0xFFFFFFFFu);
  g->ngv = nnz;

  // vertex reordering (calc_degree)
  G500_TRY(dev_alloc_n(&g->d_reorder, nolv, "reorder_map"));
  G500_TRY(dev_alloc_n(&g->d_invert, nolv, "invert_map"));
  const size_t sort_tmp = sort_tmp_bytes(std::max<int64_t>(nolv, 2 * m));
  void* d_sort_tmp = nullptr;
  G500_TRY(tmp.alloc(reinterpret_cast<char**>(&d_sort_tmp), (int64_t)sort_tmp, "sort scratch"));
  if (g->reorder_mode == 0) {
    maps_from_keys_kernel<<<grid_for(nolv), 256, 0, s>>>(nullptr, nolv, g->d_invert, g->d_reorder);
  } else {
    uint64_t *k = nullptr, *k2 = nullptr, *sorted = nullptr;
    G500_TRY(tmp.alloc(&k, nolv, "reorder keys"));
    G500_TRY(tmp.alloc(&k2, nolv, "reorder keys (alt)"));
    reorder_keys_kernel<<<grid_for(nolv), 256, 0, s>>>(deg, nolv, g->reorder_mode, maxdeg, k);
    G500_CUDA(cudaGetLastError());
    int hi = 32 + (g->reorder_mode == 2 ? std::max(1, bits_for((uint64_t)maxdeg + 1)) : 1);
    G500_TRY(radix_sort_u64(k, k2, nolv, 32, hi, d_sort_tmp, s, &sorted));
    maps_from_keys_kernel<<<grid_for(nolv), 256, 0, s>>>(sorted, nolv, g->d_invert, g->d_reorder);
  }
  G500_CUDA(cudaGetLastError());
  const int64_t last_plus1 = (g->reorder_mode == 0) ? (int64_t)sc[2] : nnz;
  g->nlv = roundup(last_plus1, LOCAL_VERTS_UNIT);
  const int64_t nlv = g->nlv;
  const int lb = std::max(1, bits_for((uint64_t)std::max<int64_t>(nlv, 1)));
  g->log_bits = lb;

  G500_TRY(dev_alloc_n(&g->d_endp, nolv, "endpoint counts"));
  endp_kernel<<<grid_for(nolv), 256, 0, s>>>(deg, sl, g->d_invert, nolv, g->d_endp);
  G500_CUDA(cudaGetLastError());

  // host bitmap of has_edge over original ids
  uint32_t* d_hbits = nullptr;
  G500_TRY(tmp.alloc(&d_hbits, nolv / 32, "has_edge bitmap"));
  has_edge_orig_kernel<<<grid_for(nolv), 256, 0, s>>>(deg, nolv, d_hbits);
  G500_CUDA(cudaGetLastError());
  g->h_has_edge_orig.assign((size_t)(nolv / 32), 0u);
  G500_CUDA(cudaMemcpyAsync(g->h_has_edge_orig.data(), d_hbits, sizeof(uint32_t) * (nolv / 32),
                            cudaMemcpyDeviceToHost, s));

  // CSR: keys for both directions, sort, drop duplicates
  G500_TRY(dev_alloc_n(&g->d_offsets, nlv + 1, "row offsets"));
  G500_TRY(dev_alloc_n(&g->d_first, nlv, "first neighbours"));
  G500_TRY(dev_alloc_n(&g->d_vis_init, std::max<int64_t>(nlv / 32, 1), "visited init bitmap"));
  const int64_t nk = 2 * m;
  uint64_t *keys = nullptr, *alt = nullptr, *sorted = nullptr;
  G500_TRY(tmp.alloc(&keys, nk, "edge keys"));
  G500_TRY(tmp.alloc(&alt, nk, "edge keys (alt)"));
  edge_keys_kernel<<<grid_for(m), 256, 0, s>>>(d_edges, m, g->d_reorder, lb, keys);
  G500_CUDA(cudaGetLastError());
  G500_TRY(radix_sort_u64(keys, alt, nk, 0, 2 * lb, d_sort_tmp, s, &sorted));
  uint32_t* rowcnt = nullptr;
  G500_TRY(tmp.alloc(&rowcnt, nlv + 1, "row lengths"));
  G500_CUDA(cudaMemsetAsync(rowcnt, 0, sizeof(uint32_t) * (nlv + 1), s));
  const int64_t ntiles = ceil_div(std::max<int64_t>(nk, 1), CP_TILE);
  uint32_t* tile_counts = nullptr;
  uint64_t* tile_offsets = nullptr;
  G500_TRY(tmp.alloc(&tile_counts, ntiles, "tile counts"));
  G500_TRY(tmp.alloc(&tile_offsets, ntiles + 1, "tile offsets"));
  void* scan_tmp = nullptr;
  G500_TRY(tmp.alloc(reinterpret_cast<char**>(&scan_tmp), (int64_t)scan_tmp_bytes(std::max(ntiles, nlv + 1)),
                     "scan scratch"));
  if (nk > 0) {
    unique_count_kernel<<<(unsigned)ntiles, CP_THREADS, 0, s>>>(sorted, nk, lb, tile_counts, rowcnt);
    G500_CUDA(cudaGetLastError());
  }
  G500_TRY(exclusive_scan_u32(tile_counts, tile_offsets, ntiles, scan_tmp, s));
  G500_TRY(exclusive_scan_u32(rowcnt, g->d_offsets, nlv, scan_tmp, s));
  uint64_t nge = 0;
  G500_CUDA(cudaMemcpyAsync(&nge, g->d_offsets + nlv, sizeof(nge), cudaMemcpyDeviceToHost, s));
  G500_CUDA(cudaStreamSynchronize(s));
  g->nge = (int64_t)nge;
  G500_TRY(dev_alloc_n(&g->d_cols, (int64_t)nge, "adjacency"));
  if (nk > 0) {
    unique_write_kernel<<<(unsigned)ntiles, CP_THREADS, 0, s>>>(sorted, nk, lb, tile_offsets, g->d_cols);
    G500_CUDA(cudaGetLastError());
  }
  if (nlv > 0) {
    g->first_flags = nlv <= (int64_t)FIRST_ID;
    finish_rows_kernel<<<grid_for(nlv), 256, 0, s>>>(g->d_offsets, g->d_cols, nlv, g->first_flags ? 1 : 0,
                                                     g->d_first, g->d_vis_init);
    G500_CUDA(cudaGetLastError());
  }
  G500_CUDA(cudaStreamSynchronize(s));

  // find_max_used_vertex (benchmark_helper.hpp:510-528) on the host bitmap
  g->max_used_vertex = 0;
  for (int64_t w = nolv / 32 - 1; w >= 0; --w) {
    uint32_t b = g->h_has_edge_orig[(size_t)w];
    if (b) {
      int64_t v = w * 32 + (31 - __builtin_clz(b));
      g->max_used_vertex = v > 0 ? v : 0;
      break;
    }
  }
  g->device_bytes = (int64_t)(sizeof(uint64_t) * (nlv + 1) + sizeof(uint32_t) * nge + sizeof(uint32_t) * nlv +
                              sizeof(uint32_t) * 3 * nolv + nlv / 8) +
                    (g->owns_edges ? (int64_t)sizeof(g500_packed_edge) * g->num_edges : 0);
  return G500_OK;
}

int new_graph(int device, int reorder_mode, g500_graph** out) {
  if (!out) return set_error(G500_E_INVAL, "null output handle");
  if (reorder_mode < 0 || reorder_mode > 2) return set_error(G500_E_INVAL, "reorder_mode %d not in 0..2", reorder_mode);
  G500_CUDA(cudaSetDevice(device));
  g500_graph* g = new g500_graph();
  g->device = device;
  g->reorder_mode = reorder_mode;
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete g;
    return cuda_error(e, "cudaStreamCreate", __FILE__, __LINE__);
  }
  *out = g;
  return G500_OK;
}

int graph_destroy_internal(g500_graph* g) {
  if (!g) return G500_OK;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  dev_free(g->d_offsets);
  dev_free(g->d_cols);
  dev_free(g->d_first);
  dev_free(g->d_reorder);
  dev_free(g->d_invert);
  dev_free(g->d_vis_init);
  dev_free(g->d_endp);
  if (g->owns_edges) dev_free(g->d_edges);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
  return G500_OK;
}

static double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace g500

using namespace g500;

extern "C" int g500_graph_build(const g500_packed_edge* edges, int64_t m, int edges_on_device, int reorder_mode,
                                int keep_edges, int device, g500_graph** out) {
  if (!edges && m > 0) return set_error(G500_E_INVAL, "null edge list");
  if (m < 0) return set_error(G500_E_INVAL, "negative edge count");
  g500_graph* g = nullptr;
  G500_TRY(new_graph(device, reorder_mode, &g));
  auto t0 = std::chrono::steady_clock::now();
  const g500_packed_edge* d_edges = edges;
  g500_packed_edge* d_copy = nullptr;
  int st = G500_OK;
  if (!edges_on_device && m > 0) {
    st = dev_alloc_n(&d_copy, m, "edge list");
    if (st == G500_OK) {
      cudaError_t e = cudaMemcpyAsync(d_copy, edges, sizeof(g500_packed_edge) * m, cudaMemcpyHostToDevice, g->stream);
      if (e != cudaSuccess) st = cuda_error(e, "cudaMemcpyAsync(edges)", __FILE__, __LINE__);
    }
    d_edges = d_copy;
  }
  if (st == G500_OK) st = build_from_device_edges(g, d_edges, m);
  if (st == G500_OK && keep_edges) {
    if (d_copy) {
      g->d_edges = d_copy;
      g->owns_edges = true;
      d_copy = nullptr;
    } else {
      g->d_edges = const_cast<g500_packed_edge*>(edges);  // caller-owned device list
      g->owns_edges = false;
    }
    g->num_edges = m;
  }
  dev_free(d_copy);
  if (st != G500_OK) {
    graph_destroy_internal(g);
    return st;
  }
  g->build_seconds = seconds_since(t0);
  *out = g;
  return G500_OK;
}

extern "C" int g500_graph_generate(int scale, int edgefactor, uint64_t s1, uint64_t s2, int reorder_mode, int device,
                                   g500_graph** out) {
  if (scale < 1 || scale > 32) return set_error(G500_E_INVAL, "scale %d not in 1..32", scale);
  if (edgefactor < 1) return set_error(G500_E_INVAL, "edgefactor %d < 1", edgefactor);
  g500_graph* g = nullptr;
  G500_TRY(new_graph(device, reorder_mode, &g));
  const int64_t m = (int64_t(1) << scale) * edgefactor;
  auto t0 = std::chrono::steady_clock::now();
  int st = dev_alloc_n(&g->d_edges, m, "edge list");
  if (st == G500_OK) {
    g->owns_edges = true;
    g->num_edges = m;
    st = gen_edges_device(scale, s1, s2, 0, m, g->d_edges, g->stream);
  }
  if (st == G500_OK) {
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) st = cuda_error(e, "generation", __FILE__, __LINE__);
  }
  g->gen_seconds = seconds_since(t0);
  auto t1 = std::chrono::steady_clock::now();
  if (st == G500_OK) st = build_from_device_edges(g, g->d_edges, m);
  if (st != G500_OK) {
    graph_destroy_internal(g);
    return st;
  }
  g->build_seconds = seconds_since(t1);
  *out = g;
  return G500_OK;
}

extern "C" int g500_graph_info_get(const g500_graph* g, g500_graph_info* info) {
  if (!g || !info) return set_error(G500_E_INVAL, "null argument");
  info->log_orig_global_verts = g->log_orig_global_verts;
  info->pred_size = g->nolv;
  info->num_local_verts = g->nlv;
  info->num_global_verts = g->ngv;
  info->num_global_edges = g->nge;
  info->max_used_vertex = g->max_used_vertex;
  info->num_input_edges = g->num_edges;
  info->device_bytes = g->device_bytes;
  info->reorder_mode = g->reorder_mode;
  info->device = g->device;
  return G500_OK;
}

static inline bool host_has_edge(const g500_graph* g, int64_t v) {
  if (v < 0 || v >= g->nolv) return false;
  return (g->h_has_edge_orig[(size_t)(v >> 5)] >> (v & 31)) & 1u;
}

extern "C" int g500_graph_has_edge(const g500_graph* g, int64_t v, int* out) {
  if (!g || !out) return set_error(G500_E_INVAL, "null argument");
  *out = host_has_edge(g, v) ? 1 : 0;
  return G500_OK;
}

// find_roots, benchmark_helper.hpp:475-508 (make_random_numbers: two MRG
// outputs per double at exponent 2 * 2^128 + 2 * counter, graph_generator.hpp:338-354)
extern "C" int g500_graph_find_roots(const g500_graph* g, int num_roots, uint64_t s1, uint64_t s2, int64_t* roots,
                                     int* found) {
  if (!g || !roots || num_roots < 0) return set_error(G500_E_INVAL, "bad argument");
  int64_t counter = 0;
  const int64_t nglobalverts = int64_t(1) << g->log_orig_global_verts;
  int k;
  for (k = 0; k < num_roots; ++k) {
    int64_t root;
    for (;;) {
      uint32_t z[5];
      mrg_seed_host(s1, s2, z);
      mrg_skip_host(z, 2, 0, (uint64_t)(2 * counter));
      double d[2];
      for (int j = 0; j < 2; ++j) {
        double a = (double)mrg_next_host(z) * .000000000465661287524579692;
        double b = (double)mrg_next_host(z) * .0000000000000000002168404346990492787;
        d[j] = a + b;
      }
      root = (int64_t)((d[0] + d[1]) * (double)nglobalverts) % nglobalverts;
      counter += 2;
      if (counter > 2 * nglobalverts) break;
      bool dup = false;
      for (int i = 0; i < k; ++i)
        if (roots[i] == root) { dup = true; break; }
      if (dup) continue;
      if (host_has_edge(g, root)) break;
    }
    roots[k] = root;
  }
  if (found) *found = k;
  return G500_OK;
}

extern "C" int g500_graph_edges(const g500_graph* g, const g500_packed_edge** dev_edges, int64_t* m) {
  if (!g) return set_error(G500_E_INVAL, "null graph");
  if (dev_edges) *dev_edges = g->d_edges;
  if (m) *m = g->d_edges ? g->num_edges : 0;
  return G500_OK;
}

extern "C" int g500_graph_copy_csr(const g500_graph* g, uint64_t* offsets, uint32_t* cols, uint32_t* reorder_map) {
  if (!g) return set_error(G500_E_INVAL, "null graph");
  G500_CUDA(cudaSetDevice(g->device));
  if (offsets) G500_CUDA(cudaMemcpy(offsets, g->d_offsets, sizeof(uint64_t) * (g->nlv + 1), cudaMemcpyDeviceToHost));
  if (cols && g->nge) G500_CUDA(cudaMemcpy(cols, g->d_cols, sizeof(uint32_t) * g->nge, cudaMemcpyDeviceToHost));
  if (reorder_map) G500_CUDA(cudaMemcpy(reorder_map, g->d_reorder, sizeof(uint32_t) * g->nolv, cudaMemcpyDeviceToHost));
  return G500_OK;
}

extern "C" int g500_graph_timings(const g500_graph* g, double* gen_s, double* build_s) {
  if (!g) return set_error(G500_E_INVAL, "null graph");
  if (gen_s) *gen_s = g->gen_seconds;
  if (build_s) *build_s = g->build_seconds;
  return G500_OK;
}

extern "C" int g500_graph_destroy(g500_graph* g) { return graph_destroy_internal(g); }
