// Direction-optimizing BFS on the device: BfsBase::run_bfs
// (mpi/bfs.hpp:2651-2940) for one GPU.
//
// State in HBM (reordered ids, nlv vertices, bitmaps of 32-bit words):
//   vis[2]    visited bitmaps (ping-pong for bottom-up snapshots); vertices
//             without edges start visited (bfs.hpp:262-265)
//   queue[2]  top-down work items (vertex, chunk): a row is cut into chunks of
//             TD_CHUNK edges so one hub does not serialise a warp
//   pred      int64 per ORIGINAL id, written once per discovered vertex with
//             parent | level << 48 (bfs.hpp:1203, :2470); -1 elsewhere
//
// Top-down (top_down_search, bfs.hpp:1139-1166, :1249-1364): each warp takes
// 32 work items, prefix-sums their lengths and walks the concatenated edge
// list 32 edges at a time (coalesced adjacency reads); a target whose visited
// bit is clear is claimed with atomicOr and the winner writes pred and appends
// the target's chunks to the next queue.
//
// Bottom-up (bottom_up_search_bitmap, bfs.hpp:1839-2038): each lane owns one
// unvisited vertex of a 32-vertex word; it tests the first (smallest-id,
// highest-degree under VERTEX_REORDERING=2) neighbour first -- the reference's
// isolated first edge -- then scans the row until a neighbour visited before
// this level is found.  New bits of a word are formed by one ballot, so the
// next visited bitmap is written without atomics.
//
// Direction switch (bfs.hpp:2799-2829): TD -> BU when growing and
// nq > num_global_verts / alpha; BU -> TD (and stop growing) when
// unvisited < num_global_verts / beta.
#include "g500_internal.cuh"

#include <algorithm>
#include <chrono>

namespace g500 {

struct BfsArgs {
  const uint64_t* __restrict__ off;
  const uint32_t* __restrict__ col;
  const uint32_t* __restrict__ first;
  const uint32_t* __restrict__ invert;
  int64_t* __restrict__ pred;
  int64_t nlv;
  int64_t nwords;
};

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(FULL_MASK, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(FULL_MASK, x, o);
  return x;
}

__device__ __forceinline__ uint32_t chunks_of(uint64_t deg) {
  return (uint32_t)((deg + TD_CHUNK - 1) / TD_CHUNK);
}

// Append the top-down work items of the discovered vertices of this warp.
// nch = number of chunks of the lane's vertex (0 = nothing to expand).
__device__ __forceinline__ void append_items(uint32_t w, uint32_t nch, uint2* __restrict__ q_out, int64_t cap,
                                             BfsCounters* cnt, unsigned* err) {
  const int lane = threadIdx.x & 31;
  uint32_t incl = warp_incl_scan(nch);
  uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
  if (total == 0) return;
  unsigned long long base = 0;
  if (lane == 31) base = atomicAdd(&cnt->q_items, (unsigned long long)total);
  base = __shfl_sync(FULL_MASK, base, 31);
  if (base + total > (unsigned long long)cap) {
    if (lane == 0) atomicOr(err, 1u);
    return;
  }
  uint64_t p = base + incl - nch;
  for (uint32_t c = 0; c < nch; ++c) q_out[p + c] = make_uint2(w, c);
}

__global__ void __launch_bounds__(256) bfs_seed_kernel(BfsArgs a, uint32_t root_r, int64_t root_orig, uint32_t* vis,
                                                       uint2* q, BfsCounters* cnt) {
  uint64_t b = a.off[root_r], e = a.off[root_r + 1];
  uint32_t nch = chunks_of(e - b);
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nch; c += gridDim.x * blockDim.x)
    q[c] = make_uint2(root_r, c);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    vis[root_r >> 5] |= 1u << (root_r & 31);
    a.pred[root_orig] = root_orig;  // first_expand, bfs.hpp:498
    cnt->q_items = nch;
  }
}

__global__ void __launch_bounds__(256) td_kernel(BfsArgs a, const uint2* __restrict__ q_in, int64_t qn,
                                                 uint32_t* vis, uint2* __restrict__ q_out, int64_t cap,
                                                 BfsCounters* cnt, unsigned* err, int level, int count_edges) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t lvl = (int64_t)level << 48;
  unsigned long long found = 0, skipped = 0, frontier = 0, edges = 0, sectors = 0;
  for (int64_t base = warp * 32; base < qn; base += nwarps * 32) {
    const int64_t qi = base + lane;
    uint64_t b = 0;
    uint32_t len = 0, orig_u = 0;
    if (qi < qn) {
      uint2 it = q_in[qi];
      uint64_t rb = a.off[it.x], re = a.off[it.x + 1];
      b = rb + (uint64_t)it.y * TD_CHUNK;
      len = (uint32_t)((re - b) < (uint64_t)TD_CHUNK ? (re - b) : (uint64_t)TD_CHUNK);
      orig_u = a.invert[it.x];
      if (count_edges) {
        frontier += (it.y == 0);
        edges += len;
        sectors += (len + 7) / 8;
      }
    }
    const uint32_t incl = warp_incl_scan(len);
    const uint32_t excl = incl - len;
    const uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
    for (uint32_t kb = 0; kb < total; kb += 32) {
      const uint32_t k = kb + lane;
      // owner item of virtual edge k: the last lane whose prefix is <= k
      int o = 0;
#pragma unroll
      for (int step = 16; step; step >>= 1) {
        uint32_t ex = __shfl_sync(FULL_MASK, excl, o + step);
        if (ex <= k) o += step;
      }
      const uint64_t bo = __shfl_sync(FULL_MASK, b, o);
      const uint32_t exo = __shfl_sync(FULL_MASK, excl, o);
      const uint32_t uo = __shfl_sync(FULL_MASK, orig_u, o);
      bool won = false;
      uint32_t w = 0, nch = 0;
      if (k < total) {
        w = a.col[bo + (k - exo)];
        const uint32_t bit = 1u << (w & 31);
        uint32_t* wp = vis + (w >> 5);
        if (!(__ldcg(wp) & bit)) won = !(atomicOr(wp, bit) & bit);
      }
      if (won) {
        a.pred[a.invert[w]] = (int64_t)uo | lvl;
        uint64_t d = a.off[w + 1] - a.off[w];
        nch = d >= 2 ? chunks_of(d) : 0;  // a degree-1 vertex only leads back to its parent
      }
      found += __popc(__ballot_sync(FULL_MASK, won));
      skipped += __popc(__ballot_sync(FULL_MASK, won && nch == 0));
      append_items(w, nch, q_out, cap, cnt, err);
    }
  }
  if (lane == 0 && found) atomicAdd(&cnt->discovered, found);
  if (lane == 0 && skipped) atomicAdd(&cnt->pad[1], skipped);
  if (count_edges) {
    frontier = warp_sum_u64(frontier);
    edges = warp_sum_u64(edges);
    sectors = warp_sum_u64(sectors);
    if (lane == 0) {
      atomicAdd(&cnt->frontier, frontier);
      atomicAdd(&cnt->edges, edges);
      atomicAdd(&cnt->sectors, sectors);
    }
  }
}

constexpr int BU_SERIAL = 6;  // row entries a lane checks on its own before the warp helps

__global__ void __launch_bounds__(256) bu_kernel(BfsArgs a, const uint32_t* __restrict__ vis_cur,
                                                 uint32_t* __restrict__ vis_next, BfsCounters* cnt, int level,
                                                 int count_edges) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t lvl = (int64_t)level << 48;
  unsigned long long found = 0, scanned = 0, edges = 0, sectors = 0;
  for (int64_t wbase = warp * 32; wbase < a.nwords; wbase += nwarps * 32) {
    const int64_t wi = wbase + lane;
    const uint32_t vw = wi < a.nwords ? __ldg(vis_cur + wi) : ~0u;
    if (wi < a.nwords && vw == ~0u) vis_next[wi] = vw;
    unsigned todo = __ballot_sync(FULL_MASK, vw != ~0u);
    while (todo) {
      const int j = __ffs(todo) - 1;
      todo &= todo - 1;
      const int64_t word = wbase + j;
      const uint32_t wv = __shfl_sync(FULL_MASK, vw, j);
      const int64_t v = word * 32 + lane;
      const bool active = !((wv >> lane) & 1u);
      uint32_t parent = NO_VERTEX;
      uint64_t pos = 0, end = 0;
      uint32_t k = 0;
      const uint32_t p = active ? __ldg(a.first + v) : NO_VERTEX;
      if (p != NO_VERTEX) {  // every unvisited vertex has an edge (vertices without one start visited)
        k = 1;
        if ((__ldg(vis_cur + (p >> 5)) >> (p & 31)) & 1u) {
          parent = p;
        } else {
          pos = __ldg(a.off + v) + 1;
          end = __ldg(a.off + v + 1);
          for (int s = 0; s < BU_SERIAL && pos < end; ++s, ++pos) {
            const uint32_t c = __ldg(a.col + pos);
            ++k;
            if ((__ldg(vis_cur + (c >> 5)) >> (c & 31)) & 1u) {
              parent = c;
              break;
            }
          }
        }
      }
      // rows still unresolved: the whole warp scans them one at a time
      unsigned rest = __ballot_sync(FULL_MASK, active && parent == NO_VERTEX && pos < end);
      while (rest) {
        const int r = __ffs(rest) - 1;
        rest &= rest - 1;
        const uint64_t rb = __shfl_sync(FULL_MASK, pos, r);
        const uint64_t re = __shfl_sync(FULL_MASK, end, r);
        uint32_t hitc = NO_VERTEX;
        uint64_t hitpos = re;
        for (uint64_t p0 = rb; p0 < re; p0 += 32) {
          const uint64_t pp = p0 + lane;
          bool h = false;
          uint32_t c = 0;
          if (pp < re) {
            c = __ldg(a.col + pp);
            h = (__ldg(vis_cur + (c >> 5)) >> (c & 31)) & 1u;
          }
          const unsigned hm = __ballot_sync(FULL_MASK, h);
          if (hm) {
            const int hl = __ffs(hm) - 1;
            hitc = __shfl_sync(FULL_MASK, c, hl);
            hitpos = p0 + hl;
            break;
          }
        }
        if (lane == r) {
          parent = hitc;
          k += (uint32_t)(min(hitpos + 1, re) - rb);
        }
      }
      const bool hit = parent != NO_VERTEX;
      const unsigned hits = __ballot_sync(FULL_MASK, hit);
      if (lane == 0) {
        vis_next[word] = wv | hits;
        found += __popc(hits);
        scanned += __popc(~wv);
      }
      if (hit) a.pred[a.invert[v]] = (int64_t)a.invert[parent] | lvl;
      if (count_edges) {
        edges += k;
        sectors += (k + 7) / 8;
      }
    }
  }
  found = warp_sum_u64(found);
  scanned = warp_sum_u64(scanned);
  if (lane == 0) {
    if (found) atomicAdd(&cnt->discovered, found);
    if (scanned) atomicAdd(&cnt->scanned, scanned);
  }
  if (count_edges) {
    edges = warp_sum_u64(edges);
    sectors = warp_sum_u64(sectors);
    if (lane == 0) {
      atomicAdd(&cnt->edges, edges);
      atomicAdd(&cnt->sectors, sectors);
    }
  }
}

// Bottom-up -> top-down: the vertices found by the last bottom-up level
// (vis_new & ~vis_old) become top-down work items.
__global__ void __launch_bounds__(256) front_to_queue_kernel(BfsArgs a, const uint32_t* __restrict__ vis_new,
                                                             const uint32_t* __restrict__ vis_old, uint2* q_out,
                                                             int64_t cap, BfsCounters* cnt, unsigned* err) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long skipped = 0;
  for (int64_t wbase = warp * 32; wbase < a.nwords; wbase += nwarps * 32) {
    const int64_t wi = wbase + lane;
    const uint32_t f = wi < a.nwords ? (vis_new[wi] & ~vis_old[wi]) : 0u;
    unsigned todo = __ballot_sync(FULL_MASK, f != 0);
    while (todo) {
      const int j = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t fj = __shfl_sync(FULL_MASK, f, j);
      const uint32_t w = (uint32_t)((wbase + j) * 32 + lane);
      uint32_t nch = 0;
      const bool in = (fj >> lane) & 1u;
      if (in) {
        uint64_t d = a.off[w + 1] - a.off[w];
        nch = d >= 2 ? chunks_of(d) : 0;
      }
      skipped += __popc(__ballot_sync(FULL_MASK, in && nch == 0));
      append_items(w, nch, q_out, cap, cnt, err);
    }
  }
  if (lane == 0 && skipped) atomicAdd(&cnt->pad[1], skipped);
}

// reached vertices and the input edges inside the reached component
// (sum of endpoint occurrences / 2 = validate.hpp's edge_visit_count for a valid tree)
__global__ void __launch_bounds__(256) reach_kernel(const uint32_t* __restrict__ vis,
                                                    const uint32_t* __restrict__ vis_init,
                                                    const uint32_t* __restrict__ endp, int64_t nwords,
                                                    unsigned long long* out) {
  unsigned long long reached = 0, e2 = 0;
  for (int64_t wi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; wi < nwords;
       wi += (int64_t)gridDim.x * blockDim.x) {
    uint32_t bits = vis[wi] & ~vis_init[wi];
    reached += __popc(bits);
    while (bits) {
      int b = __ffs(bits) - 1;
      bits &= bits - 1;
      e2 += endp[wi * 32 + b];
    }
  }
  reached = warp_sum_u64(reached);
  e2 = warp_sum_u64(e2);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[0], reached);
    atomicAdd(&out[1], e2);
  }
}

static int level_event(g500_bfs* b, size_t i) {
  while (b->level_events.size() <= i) {
    cudaEvent_t e;
    G500_CUDA(cudaEventCreate(&e));
    b->level_events.push_back(e);
  }
  return G500_OK;
}

static unsigned persistent_grid(const void* kernel, int threads) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
  if (per_sm <= 0) per_sm = 1;
  return (unsigned)(num_sms() * per_sm);
}

}  // namespace g500

using namespace g500;

static int bfs_free(g500_bfs* b) {
  if (!b) return G500_OK;
  cudaSetDevice(b->g->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  dev_free(b->d_pred);
  dev_free(b->d_vis[0]);
  dev_free(b->d_vis[1]);
  dev_free(b->d_queue[0]);
  dev_free(b->d_queue[1]);
  dev_free(b->d_counters);
  dev_free(b->d_reach);
  if (b->h_counters) cudaFreeHost(b->h_counters);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  for (cudaEvent_t e : b->level_events) cudaEventDestroy(e);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  delete b;
  return G500_OK;
}

extern "C" int g500_bfs_create(g500_graph* g, g500_bfs** out) {
  if (!g || !out) return set_error(G500_E_INVAL, "null argument");
  G500_CUDA(cudaSetDevice(g->device));
  g500_bfs* b = new g500_bfs();
  b->g = g;
  int st = G500_OK;
  auto chk = [&](cudaError_t e, const char* what) {
    if (st == G500_OK && e != cudaSuccess) st = cuda_error(e, what, __FILE__, __LINE__);
  };
  chk(cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  b->stream = b->own_stream;
  const int64_t nwords = std::max<int64_t>(g->nlv / 32, 1);
  b->queue_cap = g->nlv + g->nge / TD_CHUNK + 1024;
  if (st == G500_OK) st = dev_alloc_n(&b->d_pred, g->nolv, "pred");
  if (st == G500_OK) st = dev_alloc_n(&b->d_vis[0], nwords, "visited bitmap");
  if (st == G500_OK) st = dev_alloc_n(&b->d_vis[1], nwords, "visited bitmap");
  if (st == G500_OK) st = dev_alloc_n(&b->d_queue[0], b->queue_cap, "top-down queue");
  if (st == G500_OK) st = dev_alloc_n(&b->d_queue[1], b->queue_cap, "top-down queue");
  if (st == G500_OK) st = dev_alloc_n(&b->d_counters, 2, "level counters");
  if (st == G500_OK) st = dev_alloc_n(&b->d_reach, 4, "reach counters");
  if (st == G500_OK) chk(cudaHostAlloc(&b->h_counters, 2 * sizeof(BfsCounters), cudaHostAllocDefault), "cudaHostAlloc");
  chk(cudaEventCreate(&b->ev0), "cudaEventCreate");
  chk(cudaEventCreate(&b->ev1), "cudaEventCreate");
  if (st != G500_OK) {
    bfs_free(b);
    return st;
  }
  *out = b;
  return G500_OK;
}

extern "C" int g500_bfs_set_params(g500_bfs* b, double alpha, double beta, int count_edges) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  if (!(alpha > 0) || !(beta > 0)) return set_error(G500_E_INVAL, "alpha and beta must be > 0");
  b->alpha = alpha;
  b->beta = beta;
  b->count_edges = count_edges ? 1 : 0;
  return G500_OK;
}

extern "C" int g500_bfs_set_stream(g500_bfs* b, void* stream) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  b->stream = stream ? (cudaStream_t)stream : b->own_stream;
  return G500_OK;
}

extern "C" int g500_bfs_run(g500_bfs* b, int64_t root, int64_t* pred, int pred_on_device, g500_bfs_stats* stats) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  g500_graph* g = b->g;
  if (root < 0 || root >= g->nolv) return set_error(G500_E_INVAL, "root %lld outside [0, %lld)", (long long)root,
                                                    (long long)g->nolv);
  if (!pred) return set_error(G500_E_INVAL, "null pred");
  G500_CUDA(cudaSetDevice(g->device));
  auto t0 = std::chrono::steady_clock::now();
  cudaStream_t s = b->stream;
  int64_t* d_pred = pred_on_device ? pred : b->d_pred;
  const int64_t nwords = g->nlv / 32;
  uint32_t root_r = 0;
  G500_CUDA(cudaMemcpyAsync(&root_r, g->d_reorder + root, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  G500_CUDA(cudaStreamSynchronize(s));
  BfsArgs a{g->d_offsets, g->d_cols, g->d_first, g->d_invert, d_pred, g->nlv, nwords};
  const bool root_has_edges = (int64_t)root_r < g->nlv && ((g->h_has_edge_orig[(size_t)(root >> 5)] >> (root & 31)) & 1u);
  const unsigned grid_td = persistent_grid((const void*)td_kernel, 256);
  const unsigned grid_bu = persistent_grid((const void*)bu_kernel, 256);
  int launches = 0;
  b->levels.clear();

  G500_CUDA(cudaEventRecord(b->ev0, s));
  // initialize_memory (bfs.hpp:241-276): pred = -1, visited = ~has_edge
  G500_CUDA(cudaMemsetAsync(d_pred, 0xFF, sizeof(int64_t) * g->nolv, s));
  int64_t root_val = root;
  if (!root_has_edges) {
    G500_CUDA(cudaMemcpyAsync(d_pred + root, &root_val, sizeof(int64_t), cudaMemcpyHostToDevice, s));
  } else {
    G500_CUDA(cudaMemcpyAsync(b->d_vis[0], g->d_vis_init, sizeof(uint32_t) * nwords, cudaMemcpyDeviceToDevice, s));
    G500_CUDA(cudaMemsetAsync(b->d_counters, 0, 2 * sizeof(BfsCounters), s));
    bfs_seed_kernel<<<4, 256, 0, s>>>(a, root_r, root, b->d_vis[0], b->d_queue[0], b->d_counters);
    G500_CUDA(cudaGetLastError());
    ++launches;
    G500_CUDA(cudaMemcpyAsync(b->h_counters, b->d_counters, sizeof(BfsCounters), cudaMemcpyDeviceToHost, s));
    G500_CUDA(cudaStreamSynchronize(s));
    int64_t qn = (int64_t)b->h_counters[0].q_items;
    int cur_vis = 0, cur_q = 0;
    bool forward = true, growing = true;
    int64_t prev_nq = 0, visited = 1;
    int64_t carried = 0;  // degree-1 frontier vertices the queue skips: 1 edge, 1 sector each
    unsigned* d_err = reinterpret_cast<unsigned*>(&b->d_counters[1].pad[0]);
    for (int level = 1;; ++level) {
      if (level > 0xFFFE) return set_error(G500_E_RANGE, "BFS depth exceeds the 16-bit level field");
      G500_TRY(level_event(b, 2 * (level - 1)));
      G500_CUDA(cudaEventRecord(b->level_events[2 * (level - 1)], s));
      G500_CUDA(cudaMemsetAsync(b->d_counters, 0, sizeof(BfsCounters), s));
      g500_level_stats ls;
      memset(&ls, 0, sizeof(ls));
      ls.level = level;
      ls.direction = forward ? 1 : 0;
      if (forward) {
        if (qn > 0) {
          td_kernel<<<grid_td, 256, 0, s>>>(a, b->d_queue[cur_q], qn, b->d_vis[cur_vis], b->d_queue[cur_q ^ 1],
                                            b->queue_cap, b->d_counters, d_err, level, b->count_edges);
          G500_CUDA(cudaGetLastError());
          ++launches;
        }
      } else {
        bu_kernel<<<grid_bu, 256, 0, s>>>(a, b->d_vis[cur_vis], b->d_vis[cur_vis ^ 1], b->d_counters, level,
                                          b->count_edges);
        G500_CUDA(cudaGetLastError());
        ++launches;
      }
      G500_TRY(level_event(b, 2 * (level - 1) + 1));
      G500_CUDA(cudaEventRecord(b->level_events[2 * (level - 1) + 1], s));
      G500_CUDA(cudaMemcpyAsync(b->h_counters, b->d_counters, 2 * sizeof(BfsCounters), cudaMemcpyDeviceToHost, s));
      G500_CUDA(cudaStreamSynchronize(s));
      const BfsCounters c = b->h_counters[0];
      float lms = 0;
      G500_CUDA(cudaEventElapsedTime(&lms, b->level_events[2 * (level - 1)], b->level_events[2 * (level - 1) + 1]));
      ls.device_ms = lms;
      if (b->h_counters[1].pad[0]) return set_error(G500_E_RANGE, "top-down queue overflow");
      const int64_t nq = (int64_t)c.discovered;
      ls.discovered = nq;
      ls.frontier = forward ? (int64_t)c.frontier + carried : 0;
      ls.scanned = (int64_t)c.scanned;
      ls.edges_examined = (int64_t)c.edges + (forward ? carried : 0);
      ls.edge_sectors = (int64_t)c.sectors + (forward ? carried : 0);
      carried = (int64_t)c.pad[1];
      b->levels.push_back(ls);
      visited += nq;
      const bool was_forward = forward;
      if (!forward) cur_vis ^= 1;  // the BU output becomes the current visited map
      if (nq == 0) break;
      const int64_t unvisited = g->ngv - visited;
      if (growing && nq > prev_nq) {
        if (forward && (double)nq > (double)g->ngv / b->alpha) forward = false;
      } else {
        if (!forward && unvisited < (int64_t)((double)g->ngv / b->beta)) {
          forward = true;
          growing = false;
        }
      }
      prev_nq = nq;
      if (forward) {
        if (was_forward) {
          cur_q ^= 1;
          qn = (int64_t)c.q_items;
        } else {
          // BU -> TD: the last BU level's discoveries become work items
          G500_CUDA(cudaMemsetAsync(b->d_counters, 0, sizeof(BfsCounters), s));
          front_to_queue_kernel<<<grid_td, 256, 0, s>>>(a, b->d_vis[cur_vis], b->d_vis[cur_vis ^ 1],
                                                        b->d_queue[cur_q], b->queue_cap, b->d_counters, d_err);
          G500_CUDA(cudaGetLastError());
          ++launches;
          G500_CUDA(cudaMemcpyAsync(b->h_counters, b->d_counters, 2 * sizeof(BfsCounters), cudaMemcpyDeviceToHost, s));
          G500_CUDA(cudaStreamSynchronize(s));
          if (b->h_counters[1].pad[0]) return set_error(G500_E_RANGE, "top-down queue overflow");
          qn = (int64_t)b->h_counters[0].q_items;
          carried = (int64_t)b->h_counters[0].pad[1];
        }
      }
    }
    // the current visited map for the reach statistics
    if (stats) {
      G500_CUDA(cudaEventRecord(b->ev1, s));
      G500_CUDA(cudaMemsetAsync(b->d_reach, 0, 4 * sizeof(unsigned long long), s));
      reach_kernel<<<grid_bu, 256, 0, s>>>(b->d_vis[cur_vis], g->d_vis_init, g->d_endp, nwords, b->d_reach);
      G500_CUDA(cudaGetLastError());
    }
  }
  if (!stats || !root_has_edges) G500_CUDA(cudaEventRecord(b->ev1, s));
  if (!pred_on_device) {
    G500_CUDA(cudaMemcpyAsync(pred, d_pred, sizeof(int64_t) * g->nolv, cudaMemcpyDeviceToHost, s));
  }
  unsigned long long reach[2] = {1, 0};
  if (stats && root_has_edges)
    G500_CUDA(cudaMemcpyAsync(reach, b->d_reach, sizeof(reach), cudaMemcpyDeviceToHost, s));
  G500_CUDA(cudaStreamSynchronize(s));
  if (stats) {
    float ms = 0;
    G500_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    memset(stats, 0, sizeof(*stats));
    stats->device_ms = ms;
    stats->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (root_has_edges) {
      stats->reached = (int64_t)reach[0];
      stats->nedge = (int64_t)(reach[1] / 2);
    } else {
      uint32_t e = 0;
      G500_CUDA(cudaMemcpy(&e, g->d_endp + root_r, sizeof(uint32_t), cudaMemcpyDeviceToHost));
      stats->reached = 1;
      stats->nedge = e / 2;
    }
    stats->num_levels = (int32_t)b->levels.size();
    for (const auto& l : b->levels) (l.direction ? stats->td_levels : stats->bu_levels)++;
    stats->kernel_launches = launches;
  }
  return G500_OK;
}

extern "C" int g500_bfs_level_stats(const g500_bfs* b, g500_level_stats* out, int max_levels, int* n) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  int k = (int)std::min<size_t>(b->levels.size(), (size_t)std::max(max_levels, 0));
  if (out)
    for (int i = 0; i < k; ++i) out[i] = b->levels[(size_t)i];
  if (n) *n = (int)b->levels.size();
  return G500_OK;
}

extern "C" int g500_bfs_device_pred(const g500_bfs* b, const int64_t** dev_pred) {
  if (!b || !dev_pred) return set_error(G500_E_INVAL, "null argument");
  *dev_pred = b->d_pred;
  return G500_OK;
}

extern "C" int g500_bfs_destroy(g500_bfs* b) { return bfs_free(b); }
