// Partitioned single-root BFS: one rank's share of a 1-D vertex partition.
//
// The reference partitions the graph in 2-D over MPI ranks and exchanges the
// frontier every level: top-down "fold" packets to the owners of discovered
// vertices (mpi/bfs.hpp:521-572, :962-1137) and, bottom-up, the visited bitmap
// around the ranks (bottom_up_comm.hpp:172-280); the 2-D layout is
// graph_constructor.hpp:18-22.  Here each rank owns a contiguous range of
// reordered vertex ids (S 32-bit bitmap words each, the last range padded) and
// the CSR rows of those vertices; the graph itself is the rank's replica of
// the whole CSR (rows outside the range are never read).  Per level:
//
//   top-down   the rank expands its own frontier rows; a target it owns is
//              claimed in its own bitmap slice (atomicOr; the winner writes its
//              pred entry and lists it as next frontier), a target owned by
//              another rank and not visited before the level becomes a
//              (target, parent) pair for that rank; the pairs cross over in
//              one all-to-all and the owner claims them the same way;
//   bottom-up  every unvisited vertex of the range scans its row for a
//              neighbour visited before the level (the full bitmap, which every
//              rank holds) and takes the first one as parent;
//
// then the ranks sum their counters (the direction switch, bfs.hpp:2799-2829,
// is taken by every rank from the same sums) and all-gather their bitmap
// slices into the full bitmap.  The collectives belong to the caller (NCCL
// through torch.distributed, or copies between ranks emulated in one process);
// this file holds only the device work of one rank, stream-ordered on the
// rank's stream.  No TMA and no peer memory: every buffer is this GPU's own.
#include "g500_internal.cuh"
#include "device_common.cuh"

#include <algorithm>

namespace g500 {

struct PartCtr {
  unsigned long long disc;    // vertices of the range found this level
  unsigned long long mf;      // their degree sum
  unsigned long long nnext;   // next frontier list length
  unsigned long long scanned; // bottom-up: unvisited vertices of the range examined
  unsigned long long cnt[G500_PART_MAX_RANKS];  // top-down: pairs per destination rank
};

struct PartView {
  const uint64_t* __restrict__ off;
  const uint32_t* __restrict__ col;
  const uint32_t* __restrict__ invert;
  const uint32_t* __restrict__ reorder;
  const uint32_t* __restrict__ vis_init;
  const uint32_t* __restrict__ vis_full;  // [nranks * S] visited before the level (all ranks)
  uint32_t* own;                          // [S] this rank's slice, updated during the level
  int64_t* pred_r;                        // [32 * S] entries of the range's vertices
  int64_t lo_w, S, nwords, nlv, nolv;
  int rank, nranks;
};

__device__ __forceinline__ bool full_bit(const PartView& v, uint32_t t) {
  return (__ldcg(v.vis_full + (t >> 5)) >> (t & 31)) & 1u;
}

// claim target t of the own range for parent (original id); the winner writes
// its entry and lists it as next frontier
__device__ __forceinline__ void claim_own(const PartView& v, uint32_t t, uint32_t parent, int64_t lvl,
                                          uint32_t* next, PartCtr* c) {
  const int64_t lw = (int64_t)(t >> 5) - v.lo_w;
  const uint32_t bit = 1u << (t & 31);
  if (__ldcg(v.own + lw) & bit) return;
  if (atomicOr(v.own + lw, bit) & bit) return;
  const int64_t li = (int64_t)t - v.lo_w * 32;
  v.pred_r[li] = (int64_t)parent | lvl;
  next[atomicAdd(&c->nnext, 1ull)] = t;
  atomicAdd(&c->disc, 1ull);
  atomicAdd(&c->mf, (unsigned long long)(__ldg(v.off + t + 1) - __ldg(v.off + t)));
}

// begin: the own slice from vis_init (vertices without edges start visited),
// padding words past the graph visited, the root if it is in the range
__global__ void part_begin_kernel(PartView v, uint32_t root_r, int has_edges, int64_t root, uint32_t* front,
                                  PartCtr* c) {
  const int64_t rw = has_edges ? (int64_t)(root_r >> 5) : -1;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < v.S; w += (int64_t)gridDim.x * blockDim.x) {
    const int64_t gw = v.lo_w + w;
    uint32_t x = gw < v.nwords ? __ldg(v.vis_init + gw) : ~0u;
    if (rw == gw) x |= 1u << (root_r & 31);
    v.own[w] = x;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c->nnext = 0;
    if (rw >= v.lo_w && rw < v.lo_w + v.S) {
      v.pred_r[(int64_t)root_r - v.lo_w * 32] = root;
      front[0] = root_r;
      c->nnext = 1;
      c->mf = __ldg(v.off + root_r + 1) - __ldg(v.off + root_r);
    }
  }
}

// top-down: one warp per frontier vertex of the range, its lanes along the row
__global__ void __launch_bounds__(256) part_td_kernel(PartView v, const uint32_t* __restrict__ front, int64_t nfront,
                                                       int64_t lvl, uint32_t* next, uint64_t* pairs, int64_t cap,
                                                       PartCtr* c) {
  const int lane = threadIdx.x & 31;
  for (int64_t i = gwarp_id(); i < nfront; i += gwarp_count()) {
    const uint32_t u = __ldg(front + i);
    const uint32_t parent = __ldg(v.invert + u);
    const uint64_t b = __ldg(v.off + u), e = __ldg(v.off + u + 1);
    for (uint64_t k = b + lane; k < e; k += 32) {
      const uint32_t t = __ldg(v.col + k);
      const int64_t tw = (int64_t)(t >> 5);
      if (tw >= v.lo_w && tw < v.lo_w + v.S) {
        claim_own(v, t, parent, lvl, next, c);
      } else if (!full_bit(v, t)) {
        const int d = (int)(tw / v.S);
        const unsigned long long j = atomicAdd(&c->cnt[d], 1ull);
        if ((int64_t)j < cap) pairs[(int64_t)d * cap + (int64_t)j] = ((uint64_t)t << 32) | parent;
      }
    }
  }
}

// the pairs other ranks sent: claim them like own top-down targets
__global__ void part_apply_kernel(PartView v, const uint64_t* __restrict__ recv, int64_t n, int64_t lvl,
                                  uint32_t* next, PartCtr* c) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t x = __ldg(recv + i);
    claim_own(v, (uint32_t)(x >> 32), (uint32_t)x, lvl, next, c);
  }
}

// bottom-up: lane l of a warp owns vertex l of a word of the range; an
// unvisited vertex scans its row (ascending reordered ids: under
// VERTEX_REORDERING 2 its highest-degree neighbours first) for a neighbour
// visited before the level
__global__ void __launch_bounds__(256) part_bu_kernel(PartView v, int64_t lvl, PartCtr* c) {
  const int lane = threadIdx.x & 31;
  unsigned long long disc = 0, mf = 0, scanned = 0;
  for (int64_t w = gwarp_id(); w < v.S; w += gwarp_count()) {
    const int64_t gw = v.lo_w + w;
    if (gw >= v.nwords) break;
    const uint32_t vw = __ldcg(v.vis_full + gw);
    if (vw == ~0u) continue;
    const uint32_t r = (uint32_t)(gw * 32 + lane);
    uint32_t parent = NO_VERTEX, deg = 0;
    if (!((vw >> lane) & 1u)) {
      const uint64_t b = __ldg(v.off + r), e = __ldg(v.off + r + 1);
      deg = (uint32_t)(e - b);
      ++scanned;
      for (uint64_t k = b; k < e; ++k) {
        const uint32_t n = __ldg(v.col + k);
        if (full_bit(v, n)) {
          parent = n;
          break;
        }
      }
    }
    const unsigned found = __ballot_sync(FULL_MASK, parent != NO_VERTEX);
    if (lane == 0 && found) atomicOr(v.own + w, found);
    if (parent != NO_VERTEX) {
      v.pred_r[(int64_t)r - v.lo_w * 32] = (int64_t)__ldg(v.invert + parent) | lvl;
      ++disc;
      mf += deg;
    }
  }
  disc = warp_sum(disc);
  mf = warp_sum(mf);
  scanned = warp_sum(scanned);
  if (lane == 0) {
    if (disc) atomicAdd(&c->disc, disc);
    if (mf) atomicAdd(&c->mf, mf);
    if (scanned) atomicAdd(&c->scanned, scanned);
  }
}

// bottom-up -> top-down: the vertices of the range found by the last level
// (own & ~vis_full, before the all-gather) become the frontier list
__global__ void part_compact_kernel(PartView v, uint32_t* next, PartCtr* c) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < v.S; w += (int64_t)gridDim.x * blockDim.x) {
    const int64_t gw = v.lo_w + w;
    if (gw >= v.nwords) continue;
    uint32_t f = v.own[w] & ~__ldcg(v.vis_full + gw);
    while (f) {
      const int b = __ffs(f) - 1;
      f &= f - 1;
      next[atomicAdd(&c->nnext, 1ull)] = (uint32_t)(gw * 32 + b);
    }
  }
}

// pred in original-id order: the range's reached vertices get their entries,
// every other entry -1 (the ranks' arrays combine by an element-wise max)
__global__ void part_pred_kernel(PartView v, int64_t* __restrict__ pred) {
  for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < v.nolv; u += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t r = __ldg(v.reorder + u);
    int64_t val = -1;
    const int64_t rw = (int64_t)(r >> 5);
    if ((int64_t)r < v.nlv && rw >= v.lo_w && rw < v.lo_w + v.S) {
      const bool reached = ((__ldcg(v.vis_full + rw) & ~__ldg(v.vis_init + rw)) >> (r & 31)) & 1u;
      if (reached) val = v.pred_r[(int64_t)r - v.lo_w * 32];
    }
    pred[u] = val;
  }
}

}  // namespace g500

using namespace g500;

struct g500_part {
  g500_graph* g = nullptr;
  cudaStream_t stream = nullptr;
  int rank = 0, nranks = 1;
  int64_t S = 0, lo_w = 0;
  uint32_t* vis_full = nullptr;  // [nranks * S]
  uint32_t* own = nullptr;       // [S]
  int64_t* pred_r = nullptr;     // [32 * S]
  uint32_t* front[2] = {nullptr, nullptr};  // [32 * S] each
  int cur = 0;
  int64_t nfront = 0;
  uint64_t* pairs = nullptr;     // [nranks * cap] by destination
  uint64_t* packed = nullptr;    // [nranks * cap] contiguous in destination order
  int64_t cap = 0;
  PartCtr* d_ctr = nullptr;
  PartCtr* h_ctr = nullptr;      // pinned
  int64_t level = 0;
};

static PartView part_view(const g500_part* p) {
  const g500_graph* g = p->g;
  PartView v;
  v.off = g->d_offsets;
  v.col = g->d_cols;
  v.invert = g->d_invert;
  v.reorder = g->d_reorder;
  v.vis_init = g->d_vis_init;
  v.vis_full = p->vis_full;
  v.own = p->own;
  v.pred_r = p->pred_r;
  v.lo_w = p->lo_w;
  v.S = p->S;
  v.nwords = g->nlv / 32;
  v.nlv = g->nlv;
  v.nolv = g->nolv;
  v.rank = p->rank;
  v.nranks = p->nranks;
  return v;
}

static unsigned grid_for(int64_t n, int threads) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(std::max<int64_t>(n, 1), threads),
                                                          (int64_t)num_sms() * 8));
}

static int part_read_ctr(g500_part* p) {
  G500_CUDA(cudaMemcpyAsync(p->h_ctr, p->d_ctr, sizeof(PartCtr), cudaMemcpyDeviceToHost, p->stream));
  G500_CUDA(cudaStreamSynchronize(p->stream));
  return G500_OK;
}

extern "C" int g500_part_create(g500_graph* g, int rank, int nranks, g500_part** out) {
  if (!g || !out) return set_error(G500_E_INVAL, "null argument");
  if (nranks < 1 || nranks > G500_PART_MAX_RANKS || rank < 0 || rank >= nranks)
    return set_error(G500_E_INVAL, "rank %d of %d (1..%d ranks)", rank, nranks, G500_PART_MAX_RANKS);
  if (g->nlv < 32 || g->nolv > (int64_t)0xFFFFFFFF)
    return set_error(G500_E_INVAL, "graph too small or ids beyond 32 bits for a partitioned BFS");
  G500_CUDA(cudaSetDevice(g->device));
  g500_part* p = new g500_part();
  p->g = g;
  p->rank = rank;
  p->nranks = nranks;
  const int64_t nwords = g->nlv / 32;
  p->S = ceil_div(nwords, nranks);
  p->lo_w = (int64_t)rank * p->S;
  int st = G500_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) st = cuda_error(e, "cudaStreamCreate", __FILE__, __LINE__);
  if (st == G500_OK) st = dev_alloc_n(&p->vis_full, p->S * nranks, "partition full bitmap");
  if (st == G500_OK) st = dev_alloc_n(&p->own, p->S, "partition own bitmap");
  if (st == G500_OK) st = dev_alloc_n(&p->pred_r, 32 * p->S, "partition pred entries");
  if (st == G500_OK) st = dev_alloc_n(&p->front[0], 32 * p->S, "partition frontier");
  if (st == G500_OK) st = dev_alloc_n(&p->front[1], 32 * p->S, "partition frontier");
  if (st == G500_OK) st = dev_alloc_n(&p->d_ctr, 1, "partition counters");
  if (st == G500_OK) {
    e = cudaHostAlloc(&p->h_ctr, sizeof(PartCtr), cudaHostAllocDefault);
    if (e != cudaSuccess) st = cuda_error(e, "cudaHostAlloc", __FILE__, __LINE__);
  }
  if (st != G500_OK) {
    g500_part_destroy(p);
    return st;
  }
  *out = p;
  return G500_OK;
}

extern "C" int g500_part_info(const g500_part* p, int64_t* words_per_rank, int64_t* first_vertex,
                              int64_t* end_vertex) {
  if (!p) return set_error(G500_E_INVAL, "null handle");
  if (words_per_rank) *words_per_rank = p->S;
  if (first_vertex) *first_vertex = std::min<int64_t>(p->lo_w * 32, p->g->nlv);
  if (end_vertex) *end_vertex = std::min<int64_t>((p->lo_w + p->S) * 32, p->g->nlv);
  return G500_OK;
}

extern "C" int g500_part_buffers(g500_part* p, uint32_t** vis_full, uint32_t** own_slice, void** stream) {
  if (!p) return set_error(G500_E_INVAL, "null handle");
  if (vis_full) *vis_full = p->vis_full;
  if (own_slice) *own_slice = p->own;
  if (stream) *stream = p->stream;
  return G500_OK;
}

extern "C" int g500_part_begin(g500_part* p, int64_t root, int64_t* out) {
  if (!p || !out) return set_error(G500_E_INVAL, "null argument");
  g500_graph* g = p->g;
  if (root < 0 || root >= g->nolv)
    return set_error(G500_E_INVAL, "root %lld outside [0, %lld)", (long long)root, (long long)g->nolv);
  G500_CUDA(cudaSetDevice(g->device));
  uint32_t root_r = 0;
  G500_CUDA(cudaMemcpyAsync(&root_r, g->d_reorder + root, sizeof(uint32_t), cudaMemcpyDeviceToHost, p->stream));
  G500_CUDA(cudaStreamSynchronize(p->stream));
  uint32_t first = NO_VERTEX;
  if ((int64_t)root_r < g->nlv) {
    G500_CUDA(cudaMemcpyAsync(&first, g->d_first + root_r, sizeof(uint32_t), cudaMemcpyDeviceToHost, p->stream));
    G500_CUDA(cudaStreamSynchronize(p->stream));
  }
  const bool has_edges = (int64_t)root_r < g->nlv && first != NO_VERTEX;
  G500_CUDA(cudaMemsetAsync(p->d_ctr, 0, sizeof(PartCtr), p->stream));
  PartView v = part_view(p);
  p->cur = 0;
  p->level = 0;
  // a root without edges reached only itself: no vertex of any range is listed
  part_begin_kernel<<<grid_for(p->S, 256), 256, 0, p->stream>>>(v, root_r, has_edges ? 1 : 0, root, p->front[0],
                                                                 p->d_ctr);
  G500_CUDA(cudaGetLastError());
  G500_TRY(part_read_ctr(p));
  p->nfront = (int64_t)p->h_ctr->nnext;
  out[0] = has_edges ? 1 : 0;
  out[1] = p->nfront;
  out[2] = (int64_t)p->h_ctr->mf;  // frontier degree sum of the range
  return G500_OK;
}

// counters of the level just run: disc, mf, nnext, scanned
static void part_out(const g500_part* p, int64_t* out) {
  out[0] = (int64_t)p->h_ctr->disc;
  out[1] = (int64_t)p->h_ctr->mf;
  out[2] = (int64_t)p->h_ctr->nnext;
  out[3] = (int64_t)p->h_ctr->scanned;
}

extern "C" int g500_part_top_down(g500_part* p, int64_t frontier_edges, int64_t* send_counts) {
  if (!p || !send_counts) return set_error(G500_E_INVAL, "null argument");
  G500_CUDA(cudaSetDevice(p->g->device));
  ++p->level;
  // each frontier edge yields at most one pair: capacity for all of them per destination
  const int64_t need = std::max<int64_t>(frontier_edges, 1);
  if (need > p->cap) {
    dev_free(p->pairs);
    dev_free(p->packed);
    p->pairs = p->packed = nullptr;
    p->cap = 0;
    G500_TRY(dev_alloc_n(&p->pairs, need * p->nranks, "partition pairs"));
    G500_TRY(dev_alloc_n(&p->packed, need * p->nranks, "partition send buffer"));
    p->cap = need;
  }
  G500_CUDA(cudaMemsetAsync(p->d_ctr, 0, sizeof(PartCtr), p->stream));
  PartView v = part_view(p);
  const int64_t lvl = p->level << 48;
  if (p->nfront > 0) {
    const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(p->nfront, 8), (int64_t)num_sms() * 8);
    part_td_kernel<<<grid, 256, 0, p->stream>>>(v, p->front[p->cur], p->nfront, lvl, p->front[p->cur ^ 1], p->pairs,
                                                 p->cap, p->d_ctr);
    G500_CUDA(cudaGetLastError());
  }
  G500_TRY(part_read_ctr(p));
  // the pairs in destination order, one contiguous run per rank (none to itself)
  int64_t at = 0;
  for (int d = 0; d < p->nranks; ++d) {
    const int64_t n = std::min<int64_t>((int64_t)p->h_ctr->cnt[d], p->cap);
    send_counts[d] = n;
    if (n) G500_CUDA(cudaMemcpyAsync(p->packed + at, p->pairs + (int64_t)d * p->cap, sizeof(uint64_t) * n,
                                     cudaMemcpyDeviceToDevice, p->stream));
    at += n;
  }
  G500_CUDA(cudaStreamSynchronize(p->stream));
  return G500_OK;
}

extern "C" int g500_part_send_buffer(g500_part* p, uint64_t** pairs) {
  if (!p || !pairs) return set_error(G500_E_INVAL, "null argument");
  *pairs = p->packed;
  return G500_OK;
}

extern "C" int g500_part_apply(g500_part* p, const uint64_t* recv, int64_t n, int64_t* out) {
  if (!p || !out || (n > 0 && !recv)) return set_error(G500_E_INVAL, "null argument");
  G500_CUDA(cudaSetDevice(p->g->device));
  PartView v = part_view(p);
  const int64_t lvl = p->level << 48;
  if (n > 0) {
    part_apply_kernel<<<grid_for(n, 256), 256, 0, p->stream>>>(v, recv, n, lvl, p->front[p->cur ^ 1], p->d_ctr);
    G500_CUDA(cudaGetLastError());
  }
  G500_TRY(part_read_ctr(p));
  part_out(p, out);
  p->cur ^= 1;
  p->nfront = (int64_t)p->h_ctr->nnext;
  return G500_OK;
}

extern "C" int g500_part_bottom_up(g500_part* p, int64_t* out) {
  if (!p || !out) return set_error(G500_E_INVAL, "null argument");
  G500_CUDA(cudaSetDevice(p->g->device));
  ++p->level;
  G500_CUDA(cudaMemsetAsync(p->d_ctr, 0, sizeof(PartCtr), p->stream));
  PartView v = part_view(p);
  part_bu_kernel<<<grid_for(p->S * 32, 256), 256, 0, p->stream>>>(v, p->level << 48, p->d_ctr);
  G500_CUDA(cudaGetLastError());
  G500_TRY(part_read_ctr(p));
  part_out(p, out);
  p->nfront = 0;  // a following top-down level needs g500_part_compact
  return G500_OK;
}

extern "C" int g500_part_compact(g500_part* p, int64_t* nfront) {
  if (!p || !nfront) return set_error(G500_E_INVAL, "null argument");
  G500_CUDA(cudaSetDevice(p->g->device));
  G500_CUDA(cudaMemsetAsync(&p->d_ctr->nnext, 0, sizeof(unsigned long long), p->stream));
  PartView v = part_view(p);
  part_compact_kernel<<<grid_for(p->S, 256), 256, 0, p->stream>>>(v, p->front[p->cur], p->d_ctr);
  G500_CUDA(cudaGetLastError());
  G500_TRY(part_read_ctr(p));
  p->nfront = (int64_t)p->h_ctr->nnext;
  *nfront = p->nfront;
  return G500_OK;
}

extern "C" int g500_part_write_pred(g500_part* p, int64_t* dev_pred) {
  if (!p || !dev_pred) return set_error(G500_E_INVAL, "null argument");
  G500_CUDA(cudaSetDevice(p->g->device));
  PartView v = part_view(p);
  part_pred_kernel<<<grid_for(p->g->nolv, 256), 256, 0, p->stream>>>(v, dev_pred);
  G500_CUDA(cudaGetLastError());
  G500_CUDA(cudaStreamSynchronize(p->stream));
  return G500_OK;
}

extern "C" int g500_part_destroy(g500_part* p) {
  if (!p) return G500_OK;
  cudaSetDevice(p->g->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  dev_free(p->vis_full);
  dev_free(p->own);
  dev_free(p->pred_r);
  dev_free(p->front[0]);
  dev_free(p->front[1]);
  dev_free(p->pairs);
  dev_free(p->packed);
  dev_free(p->d_ctr);
  if (p->h_ctr) cudaFreeHost(p->h_ctr);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
  return G500_OK;
}
