// Direction-optimizing BFS on the device: BfsBase::run_bfs
// (mpi/bfs.hpp:2651-2940) for one GPU, as ONE persistent cooperative kernel
// per BFS.  Levels are separated by a grid barrier (bounded spin: on timeout
// the kernel sets an error flag and every block returns); each block takes
// the same direction decision from the same level counters, so no host round
// trip happens between levels.
//
// State in HBM (reordered ids, nlv vertices, bitmaps of 32-bit words):
//   vis[2]    visited bitmaps (ping-pong for bottom-up snapshots); vertices
//             without edges start visited (initialize_memory, bfs.hpp:262-265)
//   queue[2]  top-down work items (vertex, chunk): a row is cut into chunks of
//             TD_CHUNK edges so a hub spreads over many warps
//   pred      int64 per ORIGINAL id: parent | level << 48 (bfs.hpp:1203,
//             :2470), root = root (:498), -1 unreached.  Written as vertices
//             are found, or (deferred mode, for pred arrays beyond L2) by
//             reordered id into pred_r during the search (packed in 32 bits
//             where the ids allow) and in original-id order by one sequential
//             pass after it (deferred_pred_kernel)
//
// Top-down (top_down_search, bfs.hpp:1139-1166, :1249-1364): a warp takes B
// work items (B adapts to the queue length so every warp has work), prefix-
// sums their lengths and walks the concatenated edges TD_UNROLL*32 at a time;
// a target whose visited bit is clear is claimed with atomicOr, and the
// winner writes pred and appends the target's chunks to the next queue.
//
// Bottom-up (bottom_up_search_bitmap, bfs.hpp:1839-2038): lane l owns vertex
// l of a 32-vertex word, BU_WORDS words in flight per warp.  It tests the
// first (smallest reordered id; under VERTEX_REORDERING=2 the highest-degree)
// neighbour -- the reference's isolated first edge -- then scans the row until
// a neighbour visited before this level is found; long rows are scanned by
// the whole warp.  New bits of a word come from one ballot, so the next
// visited bitmap is written without atomics.
//
// Direction switch (bfs.hpp:2799-2829): TD -> BU when growing and
// nq > num_global_verts / alpha; BU -> TD (and stop growing) when
// unvisited < num_global_verts / beta.
#include "g500_internal.cuh"
#include "device_common.cuh"

#include <algorithm>
#include <chrono>

namespace g500 {

constexpr int BFS_THREADS = 512;
// pred arrays larger than this (beyond what L2 keeps) are written in deferred
// mode: the search records pred entries by reordered id, contiguous and
// coalesced, and one final pass writes pred in original-id order; writing
// pred at random during the search costs a DRAM read-modify-write per
// discovered vertex once pred no longer fits in L2.
constexpr uint64_t BFS_DEFERRED_PRED_BYTES = 100ull << 20;
// Packed deferred entries: parent original id in the low PACK_SHIFT bits, the
// level above it, in 32 bits instead of 64.  At SCALE 26 that halves the
// array the final pass gathers from (131 MB against 262 MB), so most of the
// gathers hit L2.  Graphs with more than 2^PACK_SHIFT vertex ids use 64-bit
// entries; a search that reaches level PACK_LEVELS - 1 stops, and the host
// runs it again with 64-bit entries (and keeps them for that handle), so that
// the all-ones word never is an entry: it marks an unreached vertex
// (PACK_NONE; -1 in 64-bit entries).
constexpr int PACK_SHIFT = 27;
constexpr int PACK_LEVELS = 1 << (32 - PACK_SHIFT);
constexpr uint32_t PACK_NONE = 0xFFFFFFFFu;
constexpr int BFS_MIN_BLOCKS = 2;        // co-resident blocks per SM (64 registers, no spills)
constexpr int TD_UNROLL = TD_CHUNK / 32;  // virtual edges per lane per pass
constexpr int BU_WORDS = 4;               // 32-vertex words a warp keeps in flight (bottom-up pass A)
constexpr int BU_SERIAL = 8;              // row entries a lane checks alone per step (one sector)
constexpr int BU_LANE_MAX = 64;           // a row with at most this many entries left is scanned by its own lane
// A frontier row of more than BIG_CHUNKS work items is listed whole (up to
// BIG_ROWS rows per level) instead of cut into items by one warp; the next
// top-down level spreads its chunks over every warp.
constexpr uint32_t BIG_CHUNKS = 64;
constexpr int BIG_ROWS = 1024;

struct RunParams {
  const uint64_t* __restrict__ off;
  const uint32_t* __restrict__ col;
  const uint32_t* __restrict__ first;
  const uint32_t* __restrict__ invert;
  const uint32_t* __restrict__ reorder;
  const uint32_t* __restrict__ vis_init;
  int64_t* __restrict__ pred;
  int64_t* __restrict__ pred_r;  // deferred mode: pred entries by reordered id, [nlv]
  uint32_t* pred_p;              // the same buffer holding packed entries (deferred == 2)
  TdItem* big;                   // [BIG_ROWS] long rows for the next top-down level (begin, deg, orig)
  int deferred;                  // 0: pred as found; 1: pred_r during the search, pred in one pass
                                 // at the end; 2: the same with packed entries
  uint32_t first_id;             // mask of the vertex id in first[] (FIRST_ID, or all bits without flags)
  uint32_t first_more;           // FIRST_MORE, or 0 when first[] has no flags (every miss is scanned)
  uint32_t* vis[2];
  TdItem* queue[2];
  BfsCtl* ctl;
  LevelRecord* rec;
  int64_t nolv, nlv, nwords, ngv, cap;
  int64_t root;
  double alpha, beta;
  int count_edges;
  int policy;
};

constexpr uint32_t FIRST_CHUNK = 0x80000000u;

// pred = -1 except pred[root] = root (initialize_memory, bfs.hpp:241-276)
__device__ __forceinline__ void fill_pred(const RunParams& p, int64_t tid, int64_t nthreads) {
  if (!(reinterpret_cast<uintptr_t>(p.pred) & 15)) {  // 16-byte stores (nolv is even)
    longlong2* pv = reinterpret_cast<longlong2*>(p.pred);
    for (int64_t i = tid; i < p.nolv / 2; i += nthreads)
      pv[i] = make_longlong2(2 * i == p.root ? p.root : -1, 2 * i + 1 == p.root ? p.root : -1);
  } else {
    for (int64_t i = tid; i < p.nolv; i += nthreads) p.pred[i] = i == p.root ? p.root : -1;
  }
}

// deferred modes (DEF = RunParams::deferred, a template argument of the
// kernel so that each mode compiles to its own code): the entry of reordered
// vertex r (parent's original id, level << 48)
template <int DEF>
__device__ __forceinline__ void put_deferred(const RunParams& p, int64_t r, uint32_t parent, int64_t lvl) {
  if constexpr (DEF == 2) p.pred_p[r] = parent | ((uint32_t)(lvl >> 48) << PACK_SHIFT);
  else p.pred_r[r] = (int64_t)parent | lvl;
}

__device__ __forceinline__ uint32_t chunks_of(uint64_t deg) { return (uint32_t)((deg + TD_CHUNK - 1) / TD_CHUNK); }

__device__ __forceinline__ void flush_counter(unsigned long long* c, unsigned long long v) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(c, v);
}

// Append the chunks of one row per lane (rows of degree < 2 and lanes with no
// row pass deg 0).  The whole warp writes the items, so a hub's thousands of
// chunks are not left to one lane; a row of more than BIG_CHUNKS chunks is
// listed whole instead (while the list has room), for the next top-down
// level to spread over every warp.
// The warp's items and the listed rows are added to *items / *bigs (lane 0
// counts the items, each listing lane its row) for the phase's totals.
__device__ __forceinline__ void append_row(uint64_t rb, uint64_t deg, uint32_t orig, TdItem* __restrict__ q_out,
                                           int64_t cap, unsigned long long* qcount, BfsCtl* ctl, TdItem* big,
                                           unsigned long long* bigcount, unsigned long long* items,
                                           unsigned long long* bigs) {
  const int lane = threadIdx.x & 31;
  uint32_t nch = chunks_of(deg);
  if (nch > BIG_CHUNKS && deg < (1ull << 31)) {
    const unsigned long long bi = atomicAdd(bigcount, 1ull);
    ++*bigs;
    if (bi < (unsigned long long)BIG_ROWS) {
      TdItem it;
      it.begin = rb;
      it.orig = orig;
      it.len = (uint32_t)deg;  // < 2^31: a row is shorter than the graph's 2^31 entries per vertex
      big[bi] = it;
      nch = 0;
    }
  }
  const uint32_t incl = warp_incl_scan(nch);
  const uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
  if (total == 0) return;
  if (lane == 0) *items += total;
  const uint32_t excl = incl - nch;
  unsigned long long base = 0;
  if (lane == 31) base = atomicAdd(qcount, (unsigned long long)total);
  base = __shfl_sync(FULL_MASK, base, 31);
  if (base + total > (unsigned long long)cap) {
    if (lane == 0) atomicOr(&ctl->bar.err, (unsigned)BFS_ERR_QUEUE);
    return;
  }
  for (uint32_t i0 = 0; i0 < total; i0 += 32) {
    const uint32_t i = i0 + lane;
    const int o = owner_lane(excl, i);
    const uint64_t rbo = __shfl_sync(FULL_MASK, rb, o);
    const uint64_t dego = __shfl_sync(FULL_MASK, deg, o);
    const uint32_t origo = __shfl_sync(FULL_MASK, orig, o);
    const uint32_t exo = __shfl_sync(FULL_MASK, excl, o);
    if (i < total) {
      const uint64_t c = i - exo;
      const uint64_t b = rbo + c * TD_CHUNK;
      const uint64_t left = rbo + dego - b;
      TdItem it;
      it.begin = b;
      it.orig = origo;
      it.len = (uint32_t)(left < (uint64_t)TD_CHUNK ? left : (uint64_t)TD_CHUNK) | (c == 0 ? FIRST_CHUNK : 0u);
      q_out[base + i] = it;
    }
  }
}

// Top-down level: expand the work items, claim unvisited targets, and list the
// discovered (vertex, original id) pairs.  Rows are cut into work items only
// if the next level is top-down as well (chunk_phase).  The nbig rows listed
// whole (p.big) are expanded as virtual items qn, qn + 1, ... after the
// queue's: item qn + c is chunk c of their concatenated chunks, found from
// a prefix of their chunk counts that each block keeps in shared memory.
template <int DEF>
__device__ void td_phase(const RunParams& p, const TdItem* __restrict__ q_in, int64_t qn, int64_t nbig, uint32_t* vis,
                         uint2* __restrict__ found_list, unsigned long long* pos, unsigned long long* sh_acc,
                         int64_t lvl) {
  __shared__ uint32_t sh_bigpre[BIG_ROWS + 1];  // sh_bigpre[i] = chunks of big rows 0 .. i-1
  const int lane = threadIdx.x & 31;
  int64_t nall = qn;
  if (nbig > 0) {
    if (threadIdx.x < 32) {
      uint32_t run = 0;
      if (lane == 0) sh_bigpre[0] = 0;
      for (int64_t i0 = 0; i0 < nbig; i0 += 32) {
        const int64_t i = i0 + lane;
        const uint32_t c = i < nbig ? chunks_of(__ldcg(&p.big[i].len)) : 0u;
        const uint32_t incl = warp_incl_scan(c);
        if (i < nbig) sh_bigpre[i + 1] = run + incl;
        run += __shfl_sync(FULL_MASK, incl, 31);
      }
    }
    __syncthreads();
    nall = qn + (int64_t)sh_bigpre[nbig];
  }
  const int64_t nwarps = gwarp_count();
  const int64_t per_warp = (nall + nwarps - 1) / nwarps;
  const int B = per_warp >= 32 ? 32 : (per_warp < 1 ? 1 : (int)per_warp);  // items per batch
  unsigned long long found = 0, frontier = 0, edges = 0, sectors = 0, mf = 0;
  for (int64_t base = gwarp_id() * B; base < nall; base += nwarps * B) {
    const int64_t qi = base + lane;
    uint64_t b = 0;
    uint32_t len = 0, orig_u = 0, first = 0;
    if (lane < B && qi < qn) {
      const TdItem it = q_in[qi];
      b = it.begin;
      len = it.len & ~FIRST_CHUNK;
      orig_u = it.orig;
      first = it.len >> 31;
    } else if (lane < B && qi < nall) {  // chunk c of the big rows: binary search of the prefix
      const uint32_t c = (uint32_t)(qi - qn);
      int lo = 0, hi = (int)nbig - 1;  // the row i with sh_bigpre[i] <= c < sh_bigpre[i + 1]
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sh_bigpre[mid] <= c) lo = mid;
        else hi = mid - 1;
      }
      const uint64_t rbeg = __ldcg(&p.big[lo].begin);
      const uint32_t rdeg = __ldcg(&p.big[lo].len);
      const uint32_t j = c - sh_bigpre[lo];
      const uint64_t left = (uint64_t)rdeg - (uint64_t)j * TD_CHUNK;
      b = rbeg + (uint64_t)j * TD_CHUNK;
      len = (uint32_t)(left < (uint64_t)TD_CHUNK ? left : (uint64_t)TD_CHUNK);
      orig_u = __ldcg(&p.big[lo].orig);
      first = j == 0;
    }
    if (p.count_edges && len) {
      frontier += first;
      edges += len;
      sectors += (len + 7) / 8;
    }
    const uint32_t incl = warp_incl_scan(len);
    const uint32_t excl = incl - len;
    const uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
    for (uint32_t kb = 0; kb < total; kb += 32 * TD_UNROLL) {
      uint32_t w[TD_UNROLL], uo[TD_UNROLL], ow[TD_UNROLL];
      bool won[TD_UNROLL];
#pragma unroll
      for (int j = 0; j < TD_UNROLL; ++j) {
        const uint32_t k = kb + j * 32 + lane;
        const int o = owner_lane(excl, k);
        const uint64_t bo = __shfl_sync(FULL_MASK, b, o);
        const uint32_t exo = __shfl_sync(FULL_MASK, excl, o);
        uo[j] = __shfl_sync(FULL_MASK, orig_u, o);
        w[j] = (k < total) ? __ldg(p.col + bo + (k - exo)) : NO_VERTEX;
      }
      uint32_t nwon = 0;
#pragma unroll
      for (int j = 0; j < TD_UNROLL; ++j) {
        won[j] = false;
        if (w[j] != NO_VERTEX) {
          const uint32_t bit = 1u << (w[j] & 31);
          uint32_t* wp = vis + (w[j] >> 5);
          if (!(__ldcg(wp) & bit)) won[j] = !(atomicOr(wp, bit) & bit);
        }
        nwon += won[j];
      }
#pragma unroll
      for (int j = 0; j < TD_UNROLL; ++j) {
        ow[j] = 0;
        if (won[j]) {
          ow[j] = __ldg(p.invert + w[j]);
          if constexpr (DEF != 0) put_deferred<DEF>(p, w[j], uo[j], lvl);
          else p.pred[ow[j]] = (int64_t)uo[j] | lvl;
          if (p.policy == G500_DIR_EDGES) mf += __ldg(p.off + w[j] + 1) - __ldg(p.off + w[j]);
        }
      }
      const uint32_t wincl = warp_incl_scan(nwon);
      const uint32_t wtotal = __shfl_sync(FULL_MASK, wincl, 31);
      if (wtotal) {
        unsigned long long fb = 0;
        if (lane == 31) fb = atomicAdd(&pos[P_ITEMS], (unsigned long long)wtotal);
        fb = __shfl_sync(FULL_MASK, fb, 31) + wincl - nwon;
#pragma unroll
        for (int j = 0; j < TD_UNROLL; ++j)
          if (won[j]) found_list[fb++] = make_uint2(w[j], ow[j]);
      }
      found += nwon;
    }
  }
  block_add(sh_acc, C_DISC, found);
  block_add(sh_acc, C_QITEMS, found);  // every find is listed
  block_add(sh_acc, C_MF, mf);
  if (p.count_edges) {
    block_add(sh_acc, C_FRONT, frontier);
    block_add(sh_acc, C_EDGES, edges);
    block_add(sh_acc, C_SECT, sectors);
  }
}

// Top-down -> top-down: the listed vertices' rows become work items.
__device__ void chunk_phase(const RunParams& p, const uint2* __restrict__ found_list, int64_t n, TdItem* q_out,
                            unsigned long long* pos, unsigned long long* sh_acc) {
  const int lane = threadIdx.x & 31;
  unsigned long long skipped = 0, items = 0, bigs = 0;
  for (int64_t base = gwarp_id() * 32; base < n; base += gwarp_count() * 32) {
    const int64_t i = base + lane;
    uint64_t rb = 0, deg = 0;
    uint32_t ow = 0;
    if (i < n) {
      const uint2 e = __ldcg(found_list + i);
      rb = __ldg(p.off + e.x);
      deg = __ldg(p.off + e.x + 1) - rb;
      ow = e.y;
      skipped += (deg < 2);
      if (deg < 2) deg = 0;  // a degree-1 vertex only leads back to its parent
    }
    append_row(rb, deg, ow, q_out, p.cap, &pos[P_ITEMS], p.ctl, p.big, &pos[P_BIG], &items, &bigs);
  }
  block_add(sh_acc, C_SKIP, skipped);
  block_add(sh_acc, C_QITEMS, items);
  block_add(sh_acc, C_BIG, bigs);
}

__device__ __forceinline__ bool vis_test(const uint32_t* __restrict__ vis, uint32_t v) {
  return (__ldg(vis + (v >> 5)) >> (v & 31)) & 1u;
}

// One lane's next BU_SERIAL entries of its row from pos (loads first, then the
// visited tests): the first entry visited before this level becomes the
// parent and ends the row; k counts the entries examined.
__device__ __forceinline__ void scan_serial(const RunParams& p, const uint32_t* __restrict__ vis_cur, uint64_t& pos,
                                            uint64_t end, uint32_t& parent, uint32_t& k) {
  uint32_t cv[BU_SERIAL];
#pragma unroll
  for (int t = 0; t < BU_SERIAL; ++t) cv[t] = pos + t < end ? __ldg(p.col + pos + t) : NO_VERTEX;
  int hit_t = -1;
  uint32_t hv = NO_VERTEX;  // cv[hit_t], kept as found: a dynamic index would put cv in local memory
#pragma unroll
  for (int t = BU_SERIAL - 1; t >= 0; --t)
    if (cv[t] != NO_VERTEX && vis_test(vis_cur, cv[t])) {
      hit_t = t;
      hv = cv[t];
    }
  if (hit_t >= 0) {
    parent = hv;
    k += (uint32_t)hit_t + 1;
    pos = end;
  } else {
    const uint64_t adv = end - pos < (uint64_t)BU_SERIAL ? end - pos : (uint64_t)BU_SERIAL;
    k += (uint32_t)adv;
    pos += adv;
  }
}

// Bottom-up level (bottom_up_search_bitmap, bfs.hpp:1839-2038), one warp per
// 32 words of the visited bitmap at a time, both steps on the same words so
// that no grid barrier separates them:
//  A. lane l owns vertex l of a word, BU_WORDS words in flight; each unvisited
//     vertex tests its first neighbour (the reference's isolated first edge;
//     under VERTEX_REORDERING=2 its highest-degree neighbour) against the
//     visited map of the previous levels.  Hits come from one ballot per word
//     and are written without atomics; the word's misses stay in a register of
//     the lane that owns the word.
//  B. the warp gathers 32 misses of its words into its lanes (select_bit); a
//     lane checks BU_SERIAL more row entries alone, and rows still unresolved
//     are scanned by the whole warp.
template <int DEF>
__device__ void bu_level(const RunParams& p, const uint32_t* __restrict__ vis_cur, uint32_t* __restrict__ vis_next,
                         unsigned long long* sh_acc, int64_t lvl) {
  const int lane = threadIdx.x & 31;
  unsigned long long found_a = 0, found_b = 0, scanned = 0, edges = 0, sectors = 0, single_misses = 0;
  // lane l of warp w owns word w + (32 k + l) * nwarps: a warp's words are
  // spread over the whole id range, so that the rows left for step B (under
  // VERTEX_REORDERING=2 concentrated in some id ranges) spread over the warps
  const int64_t nwarps = gwarp_count();
  for (int64_t k32 = 0; gwarp_id() + k32 * nwarps < p.nwords; k32 += 32) {
    const int64_t wi = gwarp_id() + (k32 + lane) * nwarps;
    const uint32_t vw = wi < p.nwords ? __ldg(vis_cur + wi) : ~0u;
    if (wi < p.nwords && vw == ~0u) vis_next[wi] = vw;
    uint32_t my_miss = 0;  // misses of word wi
    unsigned todo = __ballot_sync(FULL_MASK, vw != ~0u);
    while (todo) {
      int js[BU_WORDS];
      uint32_t wj[BU_WORDS];  // word index (nwords < 2^27)
      uint32_t wv[BU_WORDS], pf[BU_WORDS];
#pragma unroll
      for (int u = 0; u < BU_WORDS; ++u) {
        js[u] = todo ? __ffs(todo) - 1 : -1;
        todo &= todo ? todo - 1 : 0u;
        wv[u] = __shfl_sync(FULL_MASK, vw, js[u] < 0 ? 0 : js[u]);
        wj[u] = __shfl_sync(FULL_MASK, (uint32_t)wi, js[u] < 0 ? 0 : js[u]);
        if (js[u] < 0) wv[u] = ~0u;
        pf[u] = ((wv[u] >> lane) & 1u) ? NO_VERTEX : __ldg(p.first + (int64_t)wj[u] * 32 + lane);
      }
#pragma unroll
      for (int u = 0; u < BU_WORDS; ++u) {
        const bool active = !((wv[u] >> lane) & 1u);  // every unvisited vertex has an edge
        const uint32_t fv = pf[u] & p.first_id;
        const bool hit = active && pf[u] != NO_VERTEX && vis_test(vis_cur, fv);
        // a row of one edge has nothing more to scan: its miss is final for this level
        const bool more = p.first_more == 0 || (pf[u] & p.first_more);
        const unsigned hits = __ballot_sync(FULL_MASK, hit);
        const unsigned misses = __ballot_sync(FULL_MASK, active && !hit && more);
        if (p.count_edges && active && !hit && !more) ++single_misses;
        if (js[u] >= 0) {
          if (lane == 0) vis_next[wj[u]] = wv[u] | hits;
          if (lane == js[u]) my_miss = misses;
          if (lane == 0) {
            found_a += __popc(hits);
            scanned += __popc(~wv[u]);
          }
        }
        if (hit) {
          const int64_t vr = (int64_t)wj[u] * 32 + lane;
          const uint32_t par = __ldg(p.invert + fv);
          if constexpr (DEF != 0) put_deferred<DEF>(p, vr, par, lvl);
          else p.pred[__ldg(p.invert + vr)] = (int64_t)par | lvl;
        }
      }
    }
    // B: the vis_next words written above by lane 0 get the remaining finds by atomicOr
    __syncwarp();
    const uint32_t mw = my_miss;
    const uint32_t c = __popc(mw);
    const uint32_t incl = warp_incl_scan(c);
    const uint32_t excl = incl - c;
    const uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
    for (uint32_t b0 = 0; b0 < total; b0 += 32) {
      const uint32_t idx = b0 + lane;
      const int o = owner_lane(excl, idx);
      const uint32_t mwo = __shfl_sync(FULL_MASK, mw, o);
      const uint32_t exo = __shfl_sync(FULL_MASK, excl, o);
      const uint32_t wo = __shfl_sync(FULL_MASK, (uint32_t)wi, o);
      uint32_t v = NO_VERTEX, parent = NO_VERTEX, k = 0;
      uint64_t pos = 0, end = 0;
      if (idx < total) {
        v = wo * 32 + select_bit(mwo, idx - exo);
        pos = __ldg(p.off + v) + 1;
        end = __ldg(p.off + v + 1);
        k = 1;
        scan_serial(p, vis_cur, pos, end, parent, k);
      }
      // rows with at most BU_LANE_MAX entries left: every lane goes on along
      // its own row, all rows at once (one warp-wide scan per row serialised
      // the rows); longer rows are scanned by the whole warp below
      for (;;) {
        const bool mine = pos < end && end - pos <= (uint64_t)BU_LANE_MAX;
        if (!__any_sync(FULL_MASK, mine)) break;
        if (mine) scan_serial(p, vis_cur, pos, end, parent, k);
      }
      unsigned rest = __ballot_sync(FULL_MASK, pos < end);
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
          uint32_t cv = 0;
          if (pp < re) {
            cv = __ldg(p.col + pp);
            h = vis_test(vis_cur, cv);
          }
          const unsigned hm = __ballot_sync(FULL_MASK, h);
          if (hm) {
            const int hl = __ffs(hm) - 1;
            hitc = __shfl_sync(FULL_MASK, cv, hl);
            hitpos = p0 + hl;
            break;
          }
        }
        if (lane == r) {
          parent = hitc;
          k += (uint32_t)((hitpos + 1 < re ? hitpos + 1 : re) - rb);
        }
      }
      if (parent != NO_VERTEX) {
        atomicOr(vis_next + (v >> 5), 1u << (v & 31));
        const uint32_t par = __ldg(p.invert + parent);
        if constexpr (DEF != 0) put_deferred<DEF>(p, v, par, lvl);
        else p.pred[__ldg(p.invert + v)] = (int64_t)par | lvl;
        ++found_b;
      }
      if (p.count_edges && v != NO_VERTEX) {
        edges += k;
        sectors += (k + 7) / 8;
      }
    }
  }
  block_add(sh_acc, C_DISC, found_a + found_b);
  block_add(sh_acc, C_SCAN, scanned);
  if (p.count_edges) {  // a first-neighbour hit or a one-edge miss examined one edge (one sector)
    block_add(sh_acc, C_EDGES, found_a + single_misses + edges);
    block_add(sh_acc, C_SECT, found_a + single_misses + sectors);
  }
}

// Bottom-up -> top-down: vertices found by the last bottom-up level
// (vis_new & ~vis_old) become work items.
__device__ void compact_phase(const RunParams& p, const uint32_t* __restrict__ vis_new,
                              const uint32_t* __restrict__ vis_old, TdItem* q_out, unsigned long long* pos,
                              unsigned long long* sh_acc) {
  const int lane = threadIdx.x & 31;
  unsigned long long skipped = 0, items = 0, bigs = 0;
  for (int64_t wbase = gwarp_id() * 32; wbase < p.nwords; wbase += gwarp_count() * 32) {
    const int64_t wi = wbase + lane;
    const uint32_t f = wi < p.nwords ? (__ldcg(vis_new + wi) & ~__ldcg(vis_old + wi)) : 0u;
    unsigned todo = __ballot_sync(FULL_MASK, f != 0);
    while (todo) {
      const int jw = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t fj = __shfl_sync(FULL_MASK, f, jw);
      const uint32_t w = (uint32_t)((wbase + jw) * 32 + lane);
      uint64_t rb = 0, deg = 0;
      uint32_t ow = 0;
      if ((fj >> lane) & 1u) {
        rb = __ldg(p.off + w);
        deg = __ldg(p.off + w + 1) - rb;
        ow = __ldg(p.invert + w);
        skipped += (deg < 2);
        if (deg < 2) deg = 0;
      }
      append_row(rb, deg, ow, q_out, p.cap, &pos[P_ITEMS], p.ctl, p.big, &pos[P_BIG], &items, &bigs);
    }
  }
  block_add(sh_acc, C_SKIP, skipped);
  block_add(sh_acc, C_QITEMS, items);
  block_add(sh_acc, C_BIG, bigs);
}

__device__ __forceinline__ void write_record(LevelRecord* rec, int level, bool td, unsigned long long frontier,
                                             unsigned long long disc, unsigned long long scan,
                                             unsigned long long edges, unsigned long long sect,
                                             unsigned long long t_mid) {
  LevelRecord r;
  r.direction = td ? 1 : 0;
  r.level = level;
  r.frontier = td ? frontier : 0;
  r.discovered = disc;
  r.scanned = scan;
  r.edges = edges;
  r.sectors = sect;
  r.t_mid_ns = t_mid;
  r.t_ns = globaltimer();
  rec[level - 1] = r;
}

template <int DEF>
__global__ void __launch_bounds__(BFS_THREADS, BFS_MIN_BLOCKS) bfs_persistent_kernel(RunParams p) {
  __shared__ unsigned long long sh_cnt[C_NUM];
  __shared__ unsigned long long sh_acc[C_NUM];
  __shared__ unsigned sh_flag;
  BfsCtl* ctl = p.ctl;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  TdItem* items = p.queue[0];
  uint2* found_list = reinterpret_cast<uint2*>(p.queue[1]);
  if (threadIdx.x < C_NUM) sh_acc[threadIdx.x] = 0;

  // initialize_memory (bfs.hpp:241-276): pred = -1, visited = ~has_edge.  In
  // deferred mode pred is written whole by the final pass instead.
  if (tid == 0) ctl->t0_ns = globaltimer();
  // The root's own entries are written by the same fills, so one barrier
  // separates initialisation from the first level.
  // The root's id comes first; the fills below do not wait for the loads
  // that tell whether it has edges (pred is filled whether it has or not, and
  // its bit in the visited map is set either way: without edges it is set
  // already).
  const uint32_t root_r = p.reorder[p.root];
  if (DEF == 0) fill_pred(p, tid, nthreads);
  for (int64_t i = tid; i < p.nwords; i += nthreads)
    p.vis[0][i] = p.vis_init[i] | ((int64_t)root_r < p.nlv && i == (int64_t)(root_r >> 5) ? 1u << (root_r & 31) : 0u);
  const bool has_edges = (int64_t)root_r < p.nlv && p.first[root_r] != NO_VERTEX;
  const uint64_t root_b = has_edges ? p.off[root_r] : 0;
  const uint64_t root_deg = has_edges ? p.off[root_r + 1] - root_b : 0;
  const int64_t root_items = (int64_t)chunks_of(root_deg);
  if (DEF != 0 && !has_edges) fill_pred(p, tid, nthreads);  // deferred mode writes pred whole at the end
  if constexpr (DEF != 0)
    if (has_edges && tid == 0) put_deferred<DEF>(p, root_r, (uint32_t)p.root, 0);
  if (blockIdx.x == 0 && threadIdx.x < 3 * C_NUM) (&ctl->cnt[0][0])[threadIdx.x] = 0;
  if (blockIdx.x == 0 && threadIdx.x < 3 * P_NUM) (&ctl->pos[0][0])[threadIdx.x] = 0;

  // first_expand (bfs.hpp:477-518): the root's row becomes the first queue
  for (int64_t c = tid; c < root_items; c += nthreads) {
    TdItem it;
    it.begin = root_b + (uint64_t)c * TD_CHUNK;
    it.orig = (uint32_t)p.root;
    const uint64_t left = root_deg - (uint64_t)c * TD_CHUNK;
    it.len = (uint32_t)(left < (uint64_t)TD_CHUNK ? left : (uint64_t)TD_CHUNK) | (c == 0 ? FIRST_CHUNK : 0u);
    items[c] = it;
  }
  if (tid == 0) ctl->root_has_edges = has_edges ? 1 : 0;
  if (!has_edges) {  // the search is over before it starts: only the root has a parent
    if (tid == 0) {
      ctl->num_levels = 0;
      ctl->final_vis = 0;
      ctl->t_init_ns = ctl->t_end_ns = globaltimer();
    }
    return;
  }
  if (!grid_sync<C_NUM>(&ctl->bar, nullptr, sh_acc, nullptr, sh_cnt, &sh_flag)) return;
  if (tid == 0) ctl->t_init_ns = globaltimer();

  int cur_vis = 0;
  bool forward = true, growing = true;
  int64_t qn = root_items, prev_nq = 0, visited = 1, carried = 0, nbig = 0;
  int64_t mu = (int64_t)(p.off[p.nlv] - root_deg);  // degree sum of unvisited vertices (edge policy)
  unsigned phase = 0;
  int level = 1;
  // Each phase uses counter and position slot phase%3 and clears slot
  // (phase+1)%3 for the next one; a slot is read right after its phase's
  // barrier, so it is never cleared while a block may still read it, and it
  // is cleared before any block can arrive at the barrier that sums into it.
#define NEXT_PHASE_SLOT()                                                              \
  (blockIdx.x == 0 && threadIdx.x < C_NUM ? (void)(ctl->cnt[(phase + 1) % 3][threadIdx.x] = 0) : (void)0), \
  (blockIdx.x == 0 && threadIdx.x < P_NUM ? (void)(ctl->pos[(phase + 1) % 3][threadIdx.x] = 0) : (void)0), \
      ctl->cnt[phase % 3]
  for (;; ++level) {
    if (DEF == 2 && level >= PACK_LEVELS - 1) {  // the packed level field is full: the host reruns unpacked
      if (tid == 0) atomicOr(&ctl->bar.err, (unsigned)BFS_ERR_PACK);
      return;
    }
    unsigned long long* cnt = (NEXT_PHASE_SLOT());
    const int64_t lvl = (int64_t)level << 48;
    unsigned long long disc, scan = 0, edges, sect, front = 0, listed = 0, t_mid = 0, mf = 0;
    if (forward) {
      td_phase<DEF>(p, items, qn, nbig, p.vis[cur_vis], found_list, ctl->pos[phase % 3], sh_acc, lvl);
      if (!grid_sync_sum<C_NUM>(cnt, &ctl->bar, sh_acc, sh_cnt)) return;
      if (tid == 0) t_mid = globaltimer();
      ++phase;
      disc = sh_cnt[C_DISC];
      edges = sh_cnt[C_EDGES];
      sect = sh_cnt[C_SECT];
      front = sh_cnt[C_FRONT];
      listed = sh_cnt[C_QITEMS];
      mf = sh_cnt[C_MF];
    } else {
      bu_level<DEF>(p, p.vis[cur_vis], p.vis[cur_vis ^ 1], sh_acc, lvl);
      if (!grid_sync_sum<C_NUM>(cnt, &ctl->bar, sh_acc, sh_cnt)) return;
      if (tid == 0) t_mid = globaltimer();
      ++phase;
      disc = sh_cnt[C_DISC];
      scan = sh_cnt[C_SCAN];
      edges = sh_cnt[C_EDGES];
      sect = sh_cnt[C_SECT];
    }
    const int64_t nq = (int64_t)disc;
    const int64_t carried_in = carried;
    visited += nq;
    const bool was_forward = forward;
    if (!forward) cur_vis ^= 1;  // the bottom-up output is the current visited map
    if (nq == 0) {
      if (tid == 0) write_record(p.rec, level, was_forward, front + carried_in, disc, scan,
                                 edges + (was_forward ? carried_in : 0), sect + (was_forward ? carried_in : 0), t_mid);
      break;
    }
    if (level >= MAX_LEVELS) {
      if (tid == 0) atomicOr(&ctl->bar.err, (unsigned)BFS_ERR_DEPTH);
      break;
    }
    const int64_t unvisited = p.ngv - visited;
    if (was_forward) mu -= (int64_t)mf;
    if (p.policy == G500_DIR_EDGES) {
      if (forward && growing) {
        if ((double)mf > (double)mu / p.alpha) forward = false;
      } else if (!forward && nq < prev_nq && (double)nq < (double)p.ngv / p.beta) {
        forward = true;
        growing = false;
      }
    } else if (growing && nq > prev_nq) {  // the reference's rule, bfs.hpp:2799-2829
      if (forward && (double)nq > (double)p.ngv / p.alpha) forward = false;
    } else if (!forward && unvisited < (int64_t)((double)p.ngv / p.beta)) {
      forward = true;
      growing = false;
    }
    prev_nq = nq;
    if (forward) {
      unsigned long long* ccnt = (NEXT_PHASE_SLOT());
      if (was_forward) chunk_phase(p, found_list, (int64_t)listed, items, ctl->pos[phase % 3], sh_acc);
      else compact_phase(p, p.vis[cur_vis], p.vis[cur_vis ^ 1], items, ctl->pos[phase % 3], sh_acc);
      if (!grid_sync_sum<C_NUM>(ccnt, &ctl->bar, sh_acc, sh_cnt)) return;
      ++phase;
      qn = (int64_t)sh_cnt[C_QITEMS];
      nbig = (int64_t)(sh_cnt[C_BIG] < (unsigned long long)BIG_ROWS ? sh_cnt[C_BIG] : (unsigned long long)BIG_ROWS);
      carried = (int64_t)sh_cnt[C_SKIP];
      if (qn > p.cap) {  // append_row already flagged it; never read past the queue
        if (tid == 0) atomicOr(&ctl->bar.err, (unsigned)BFS_ERR_QUEUE);
        return;
      }
    }
    if (tid == 0)
      write_record(p.rec, level, was_forward, front + carried_in, disc, scan,
                   edges + (was_forward ? carried_in : 0), sect + (was_forward ? carried_in : 0), t_mid);
  }
#undef NEXT_PHASE_SLOT
  // deferred modes: the entries of the vertices the search did not reach (and
  // of those without edges) become "unreached", so that the final pass reads
  // one entry per vertex and no bitmap.  The last level's barrier has passed:
  // the visited map is final.  Under VERTEX_REORDERING 2 few such vertices lie
  // below nlv (those without edges sort last).
  if constexpr (DEF != 0) {
    const uint32_t* vf = p.vis[cur_vis];
    for (int64_t wi = tid; wi < p.nwords; wi += nthreads) {
      uint32_t miss = ~(__ldcg(vf + wi) & ~__ldg(p.vis_init + wi));
      while (miss) {
        const int b = __ffs(miss) - 1;
        miss &= miss - 1;
        if constexpr (DEF == 2) p.pred_p[wi * 32 + b] = PACK_NONE;
        else p.pred_r[wi * 32 + b] = -1;
      }
    }
  }
  if (tid == 0) {
    ctl->num_levels = (unsigned)level;
    ctl->final_vis = cur_vis;
    ctl->t_end_ns = globaltimer();
  }
}

// Deferred modes, after the search: pred in original-id order with
// sequential writes.  The entry of reordered vertex r (r < nlv) is its pred
// value, or "unreached" (PACK_NONE / -1, written by the search's last phase);
// a vertex beyond nlv has no edges and no entry.  Its own launch, so that 2048
// threads per SM (the persistent kernel has 1024) keep the gathers in flight;
// 4 consecutive vertices per thread, their loads issued together.  The
// streamed map and pred are evict-first, so that the gathered entries stay in
// L2.  nolv is a multiple of 65536.
constexpr int FINAL_THREADS = 256;
template <int DEF>
__device__ __forceinline__ long long final_entry(const RunParams& p, uint32_t r) {
  if ((int64_t)r >= p.nlv) return -1ll;
  if constexpr (DEF == 2) {
    const uint32_t e = __ldcg(p.pred_p + r);
    return e == PACK_NONE ? -1ll
                          : (long long)((int64_t)(e & ((1u << PACK_SHIFT) - 1u)) | ((int64_t)(e >> PACK_SHIFT) << 48));
  }
  return (long long)__ldcg(p.pred_r + r);
}

template <int DEF>
__global__ void __launch_bounds__(FINAL_THREADS, 8) deferred_pred_kernel(RunParams p) {
  const BfsCtl* ctl = p.ctl;
  if (!ctl->root_has_edges || ctl->bar.err) return;  // pred already written, or the search failed
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  if (reinterpret_cast<uintptr_t>(p.pred) & 15) {  // a caller's pred not 16-byte aligned: one entry at a time
    for (int64_t u = tid; u < p.nolv; u += nthreads) p.pred[u] = final_entry<DEF>(p, __ldg(p.reorder + u));
    return;
  }
  for (int64_t u0 = tid * 4; u0 < p.nolv; u0 += nthreads * 4) {
    const uint4 ra = __ldcs(reinterpret_cast<const uint4*>(p.reorder + u0));
    long long val[4];
    val[0] = final_entry<DEF>(p, ra.x);
    val[1] = final_entry<DEF>(p, ra.y);
    val[2] = final_entry<DEF>(p, ra.z);
    val[3] = final_entry<DEF>(p, ra.w);
    longlong2* dst = reinterpret_cast<longlong2*>(p.pred + u0);
    __stcs(dst, make_longlong2(val[0], val[1]));
    __stcs(dst + 1, make_longlong2(val[2], val[3]));
  }
}

// reached vertices and 2 x the input edges inside the reached component
// (sum of endpoint occurrences = 2 x validate.hpp's edge_visit_count for a valid tree)
__global__ void __launch_bounds__(256) reach_kernel(const uint32_t* vis0, const uint32_t* vis1,
                                                    const uint32_t* __restrict__ vis_init,
                                                    const uint32_t* __restrict__ endp, int64_t nwords,
                                                    BfsCtl* ctl) {
  if (!ctl->root_has_edges) return;
  const uint32_t* vis = ctl->final_vis ? vis1 : vis0;
  unsigned long long reached = 0, e2 = 0;
  for (int64_t wi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; wi < nwords;
       wi += (int64_t)gridDim.x * blockDim.x) {
    uint32_t bits = vis[wi] & ~vis_init[wi];
    reached += __popc(bits);
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1;
      e2 += endp[wi * 32 + b];
    }
  }
  flush_counter(&ctl->reach[0], reached);
  flush_counter(&ctl->reach[1], e2);
}

}  // namespace g500

using namespace g500;

static int bfs_free(g500_bfs* b) {
  if (!b) return G500_OK;
  cudaSetDevice(b->g->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  pred_expander_free(b);
  dev_free(b->d_pred);
  dev_free(b->d_pred_r);
  dev_free(b->d_levels);
  dev_free(b->d_overflow);
  if (b->ev_done) cudaEventDestroy(b->ev_done);
  dev_free(b->d_vis[0]);
  dev_free(b->d_vis[1]);
  dev_free(b->d_queue[0]);
  dev_free(b->d_queue[1]);
  dev_free(b->d_ctl);
  dev_free(b->d_rec);
  dev_free(b->d_big);
  if (b->h_ctl) cudaFreeHost(b->h_ctl);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  delete b;
  return G500_OK;
}

// the deferred modes' final pass, enqueued right after the search
static int launch_deferred_pred(const RunParams& p, cudaStream_t s) {
  if (!p.deferred) return G500_OK;
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(p.nolv / 4, FINAL_THREADS), (int64_t)num_sms() * 64);
  if (p.deferred == 2) deferred_pred_kernel<2><<<grid, FINAL_THREADS, 0, s>>>(p);
  else deferred_pred_kernel<1><<<grid, FINAL_THREADS, 0, s>>>(p);
  G500_CUDA(cudaGetLastError());
  return G500_OK;
}

static const void* bfs_kernel_for(int deferred) {
  if (deferred == 2) return (const void*)bfs_persistent_kernel<2>;
  if (deferred == 1) return (const void*)bfs_persistent_kernel<1>;
  return (const void*)bfs_persistent_kernel<0>;
}

// The kernel's parameters for one run from `root` writing pred to `pred`.
static int make_params(g500_bfs* b, int64_t root, int64_t* pred, RunParams* out) {
  g500_graph* g = b->g;
  RunParams& p = *out;
  p.off = g->d_offsets;
  p.col = g->d_cols;
  p.first = g->d_first;
  p.first_id = g->first_flags ? FIRST_ID : 0xFFFFFFFFu;
  p.first_more = g->first_flags ? FIRST_MORE : 0u;
  p.invert = g->d_invert;
  p.reorder = g->d_reorder;
  p.vis_init = g->d_vis_init;
  p.pred = pred;
  int mode = b->pred_mode;
  if (mode == 0) mode = (uint64_t)g->nolv * 8 > BFS_DEFERRED_PRED_BYTES ? 3 : 1;
  if (mode == 3 && (b->pack_off || g->nolv > (1ll << PACK_SHIFT))) mode = 2;
  p.deferred = mode == 1 ? 0 : (mode == 2 ? 1 : 2);
  if (p.deferred && !b->d_pred_r) G500_TRY(dev_alloc_n(&b->d_pred_r, std::max<int64_t>(g->nlv, 1), "deferred pred"));
  p.pred_r = b->d_pred_r;
  p.pred_p = reinterpret_cast<uint32_t*>(b->d_pred_r);
  p.big = b->d_big;
  p.vis[0] = b->d_vis[0];
  p.vis[1] = b->d_vis[1];
  p.queue[0] = b->d_queue[0];
  p.queue[1] = b->d_queue[1];
  p.ctl = b->d_ctl;
  p.rec = b->d_rec;
  p.nolv = g->nolv;
  p.nlv = g->nlv;
  p.nwords = g->nlv / 32;
  p.ngv = g->ngv;
  p.cap = b->queue_cap;
  p.root = root;
  p.alpha = b->alpha;
  p.policy = b->policy;
  p.beta = b->beta;
  p.count_edges = b->count_edges;
  return G500_OK;
}

// pred -> uint8 levels (255 unreached); a level over 254 raises *overflow
__global__ void levels_from_pred_kernel(const int64_t* __restrict__ pred, int64_t n, uint8_t* __restrict__ out,
                                        unsigned* overflow) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = pred[i];
    uint8_t l = 255;
    if (v != -1) {
      const int64_t lv = (v >> 48) & 0xFFFF;
      if (lv > 254) atomicOr(overflow, 1u);
      l = (uint8_t)(lv > 254 ? 254 : lv);
    }
    out[i] = l;
  }
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
  if (st == G500_OK) st = dev_alloc_n(&b->d_queue[0], b->queue_cap, "top-down work items");
  if (st == G500_OK) st = dev_alloc_n(&b->d_queue[1], b->queue_cap, "top-down discovered list");
  if (st == G500_OK) st = dev_alloc_n(&b->d_ctl, 1, "bfs control block");
  if (st == G500_OK) st = dev_alloc_n(&b->d_rec, MAX_LEVELS, "level records");
  if (st == G500_OK) st = dev_alloc_n(&b->d_big, BIG_ROWS, "long frontier rows");
  if (st == G500_OK) chk(cudaHostAlloc(&b->h_ctl, sizeof(BfsCtl), cudaHostAllocDefault), "cudaHostAlloc");
  if (st == G500_OK) chk(cudaMemset(b->d_ctl, 0, sizeof(BfsCtl)), "cudaMemset");
  if (st == G500_OK) memset(b->h_ctl, 0, sizeof(BfsCtl));
  chk(cudaEventCreate(&b->ev0), "cudaEventCreate");
  chk(cudaEventCreate(&b->ev1), "cudaEventCreate");
  if (st == G500_OK) {
    int per_sm = 0;
    chk(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfs_persistent_kernel<2>, BFS_THREADS, 0),
        "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    int coop = 0;
    chk(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, g->device), "cudaDeviceGetAttribute");
    if (st == G500_OK && (!coop || per_sm <= 0))
      st = set_error(G500_E_DEVICE, "device cannot co-schedule the persistent BFS kernel");
    b->grid = b->grid_full = (unsigned)(num_sms() * std::max(per_sm, 1));
  }
  if (st != G500_OK) {
    bfs_free(b);
    return st;
  }
  *out = b;
  return G500_OK;
}

extern "C" int g500_bfs_set_grid(g500_bfs* b, int blocks) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  if (blocks < 0) return set_error(G500_E_INVAL, "negative block count");
  if (b->in_flight) return set_error(G500_E_STATE, "a run is in flight");
  b->grid = blocks == 0 ? b->grid_full : std::min<unsigned>((unsigned)blocks, b->grid_full);
  return G500_OK;
}

namespace g500 {

int bfs_launch_levels(g500_bfs* b, int64_t root, uint8_t* levels_dst) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  if (b->in_flight) return set_error(G500_E_STATE, "the previous run has not completed");
  g500_graph* g = b->g;
  if (root < 0 || root >= g->nolv)
    return set_error(G500_E_INVAL, "root %lld outside [0, %lld)", (long long)root, (long long)g->nolv);
  G500_CUDA(cudaSetDevice(g->device));
  if (!b->d_levels) G500_TRY(dev_alloc_n(&b->d_levels, std::max<int64_t>(g->nolv, 1), "levels"));
  if (!b->d_overflow) G500_TRY(dev_alloc_n(&b->d_overflow, 1, "level overflow flag"));
  if (!b->ev_done) G500_CUDA(cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming));
  cudaStream_t s = b->stream;
  RunParams p;
  G500_TRY(make_params(b, root, b->d_pred, &p));
  void* args[] = {&p};
  G500_CUDA(cudaMemsetAsync(b->d_ctl, 0, sizeof(BfsCtl), s));
  G500_CUDA(cudaMemsetAsync(b->d_overflow, 0, sizeof(unsigned), s));
  G500_CUDA(cudaLaunchCooperativeKernel(bfs_kernel_for(p.deferred), dim3(b->grid), dim3(BFS_THREADS), args,
                                        0, s));
  G500_TRY(launch_deferred_pred(p, s));
  const unsigned rg = (unsigned)std::min<int64_t>(ceil_div(std::max<int64_t>(p.nwords, 1), 256), num_sms() * 8);
  reach_kernel<<<rg, 256, 0, s>>>(b->d_vis[0], b->d_vis[1], g->d_vis_init, g->d_endp, p.nwords, b->d_ctl);
  const unsigned lg = (unsigned)std::min<int64_t>(ceil_div(g->nolv, 256), num_sms() * 8);
  levels_from_pred_kernel<<<lg, 256, 0, s>>>(b->d_pred, g->nolv, b->d_levels, b->d_overflow);
  G500_CUDA(cudaGetLastError());
  if (levels_dst) G500_CUDA(cudaMemcpyAsync(levels_dst, b->d_levels, (size_t)g->nolv, cudaMemcpyDefault, s));
  G500_CUDA(cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(BfsCtl), cudaMemcpyDeviceToHost, s));
  G500_CUDA(cudaMemcpyAsync(&b->h_ctl->pad_overflow, b->d_overflow, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  G500_CUDA(cudaEventRecord(b->ev_done, s));
  b->last_root = root;
  b->last_levels_dst = levels_dst;
  b->in_flight = 1;
  return G500_OK;
}

int bfs_poll(g500_bfs* b, int* done) {
  if (!b || !done) return set_error(G500_E_INVAL, "null argument");
  if (!b->in_flight) return set_error(G500_E_STATE, "no run in flight");
  const cudaError_t e = cudaEventQuery(b->ev_done);
  if (e == cudaSuccess) {
    *done = 1;
    return G500_OK;
  }
  if (e == cudaErrorNotReady) {
    *done = 0;
    return G500_OK;
  }
  return cuda_error(e, "cudaEventQuery", __FILE__, __LINE__);
}

int bfs_complete(g500_bfs* b, int64_t* reached, int64_t* nedge) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  if (!b->in_flight) return set_error(G500_E_STATE, "no run in flight");
  b->in_flight = 0;
  G500_CUDA(cudaSetDevice(b->g->device));
  const cudaError_t e = cudaEventSynchronize(b->ev_done);
  if (e != cudaSuccess) return cuda_error(e, "cudaEventSynchronize", __FILE__, __LINE__);
  const BfsCtl& c = *b->h_ctl;
  if (c.bar.err & BFS_ERR_TIMEOUT) return set_error(G500_E_TIMEOUT, "grid barrier wait gave up (bounded spin)");
  if (c.bar.err & BFS_ERR_PACK) {  // deeper than the packed entries hold: the same run with 64-bit entries
    b->pack_off = 1;
    G500_TRY(bfs_launch_levels(b, b->last_root, b->last_levels_dst));
    return bfs_complete(b, reached, nedge);
  }
  if (c.bar.err & BFS_ERR_QUEUE) return set_error(G500_E_RANGE, "top-down queue overflow");
  if (c.bar.err & BFS_ERR_DEPTH) return set_error(G500_E_RANGE, "BFS depth exceeds the 16-bit level field");
  if (c.pad_overflow) return set_error(G500_E_RANGE, "a level over 254 does not fit the uint8 levels");
  if (c.root_has_edges) {
    if (reached) *reached = (int64_t)c.reach[0];
    if (nedge) *nedge = (int64_t)(c.reach[1] / 2);
  } else {  // a root without edges reached only itself; its self-loops are its edges
    uint32_t root_r = 0, ep = 0;
    G500_CUDA(cudaMemcpy(&root_r, b->g->d_reorder + b->last_root, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    G500_CUDA(cudaMemcpy(&ep, b->g->d_endp + root_r, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (reached) *reached = 1;
    if (nedge) *nedge = ep / 2;
  }
  return G500_OK;
}

}  // namespace g500

extern "C" int g500_bfs_set_params(g500_bfs* b, double alpha, double beta, int count_edges) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  if (!(alpha > 0) || !(beta > 0)) return set_error(G500_E_INVAL, "alpha and beta must be > 0");
  b->alpha = alpha;
  b->beta = beta;
  b->count_edges = count_edges ? 1 : 0;
  return G500_OK;
}

extern "C" int g500_bfs_set_pred_mode(g500_bfs* b, int mode) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  if (mode < 0 || mode > 3) return set_error(G500_E_INVAL, "unknown pred mode %d", mode);
  b->pred_mode = mode;
  return G500_OK;
}

extern "C" int g500_bfs_set_host_pack(g500_bfs* b, int on) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  b->pack_host_off = on ? 0 : 1;
  return G500_OK;
}

extern "C" int g500_bfs_set_policy(g500_bfs* b, int policy) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  if (policy != G500_DIR_REFERENCE && policy != G500_DIR_EDGES)
    return set_error(G500_E_INVAL, "unknown direction policy %d", policy);
  b->policy = policy;
  return G500_OK;
}

extern "C" int g500_bfs_autotune(g500_bfs* b, const int64_t* roots, int nroots, int reps, g500_tune_result* out) {
  if (!b || !roots || nroots <= 0) return set_error(G500_E_INVAL, "bad argument");
  if (reps < 1) reps = 1;
  struct Cfg { int policy; double alpha, beta; };
  static const Cfg grid[] = {
      {G500_DIR_REFERENCE, 2000.0, 8.0},  {G500_DIR_REFERENCE, 100.0, 8.0},  {G500_DIR_REFERENCE, 500.0, 1e9},
      {G500_DIR_REFERENCE, 100.0, 1e9},   {G500_DIR_REFERENCE, 2000.0, 1e9}, {G500_DIR_REFERENCE, 20000.0, 1e9},
      {G500_DIR_EDGES, 2.0, 24.0},        {G500_DIR_EDGES, 6.0, 24.0},       {G500_DIR_EDGES, 15.0, 24.0},
      {G500_DIR_EDGES, 2.0, 1e9},         {G500_DIR_EDGES, 6.0, 1e9},        {G500_DIR_EDGES, 15.0, 1e9},
      {G500_DIR_EDGES, 50.0, 1e9},        {G500_DIR_EDGES, 150.0, 1e9},
  };
  const int ncfg = (int)(sizeof(grid) / sizeof(grid[0]));
  const int saved_count = b->count_edges;
  b->count_edges = 0;
  double best = 1e300, ref_ms = 0;
  int best_i = 0;
  for (int c = 0; c < ncfg; ++c) {
    b->policy = grid[c].policy;
    b->alpha = grid[c].alpha;
    b->beta = grid[c].beta;
    double sum = 0;
    for (int r = 0; r < nroots; ++r) {
      double m = 1e300;
      for (int k = 0; k < reps; ++k) {
        g500_bfs_stats st;
        int rc = g500_bfs_run(b, roots[r], b->d_pred, 1, &st);
        if (rc != G500_OK) {
          b->count_edges = saved_count;
          return rc;
        }
        m = std::min(m, st.device_ms);
      }
      sum += m;
    }
    const double mean = sum / nroots;
    if (c == 0) ref_ms = mean;
    if (mean < best) {
      best = mean;
      best_i = c;
    }
  }
  b->policy = grid[best_i].policy;
  b->alpha = grid[best_i].alpha;
  b->beta = grid[best_i].beta;
  b->count_edges = saved_count;
  if (out) {
    out->policy = b->policy;
    out->configs_tried = ncfg;
    out->alpha = b->alpha;
    out->beta = b->beta;
    out->best_ms = best;
    out->reference_ms = ref_ms;
  }
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
  if (root < 0 || root >= g->nolv)
    return set_error(G500_E_INVAL, "root %lld outside [0, %lld)", (long long)root, (long long)g->nolv);
  if (!pred) return set_error(G500_E_INVAL, "null pred");
  G500_CUDA(cudaSetDevice(g->device));
  auto t0 = std::chrono::steady_clock::now();
  cudaStream_t s = b->stream;
  RunParams p;
  G500_TRY(make_params(b, root, pred_on_device ? pred : b->d_pred, &p));
  void* args[] = {&p};
  G500_CUDA(cudaMemsetAsync(b->d_ctl, 0, sizeof(BfsCtl), s));
  G500_CUDA(cudaEventRecord(b->ev0, s));
  G500_CUDA(cudaLaunchCooperativeKernel(bfs_kernel_for(p.deferred), dim3(b->grid), dim3(BFS_THREADS), args,
                                        0, s));
  G500_TRY(launch_deferred_pred(p, s));
  G500_CUDA(cudaEventRecord(b->ev1, s));
  if (stats) {
    const unsigned rg = (unsigned)std::min<int64_t>(ceil_div(std::max<int64_t>(p.nwords, 1), 256), num_sms() * 8);
    reach_kernel<<<rg, 256, 0, s>>>(b->d_vis[0], b->d_vis[1], g->d_vis_init, g->d_endp, p.nwords, b->d_ctl);
    G500_CUDA(cudaGetLastError());
  }
  G500_CUDA(cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(BfsCtl), cudaMemcpyDeviceToHost, s));
  if (!pred_on_device) {
    bool packed = false;
    G500_TRY(pred_to_host_packed(b, pred, s, &packed));
    if (!packed) G500_CUDA(cudaMemcpyAsync(pred, b->d_pred, sizeof(int64_t) * g->nolv, cudaMemcpyDeviceToHost, s));
  }
  G500_CUDA(cudaStreamSynchronize(s));
  b->last_root = root;
  const BfsCtl& c = *b->h_ctl;
  if (c.bar.err & BFS_ERR_TIMEOUT) return set_error(G500_E_TIMEOUT, "grid barrier wait gave up (bounded spin)");
  if (c.bar.err & BFS_ERR_PACK) {  // deeper than the packed entries hold: the same run with 64-bit entries
    b->pack_off = 1;
    return g500_bfs_run(b, root, pred, pred_on_device, stats);
  }
  if (c.bar.err & BFS_ERR_QUEUE) return set_error(G500_E_RANGE, "top-down queue overflow");
  if (c.bar.err & BFS_ERR_DEPTH) return set_error(G500_E_RANGE, "BFS depth exceeds the 16-bit level field");
  if (stats) {
    float ms = 0;
    G500_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    memset(stats, 0, sizeof(*stats));
    stats->device_ms = ms;
    stats->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (c.root_has_edges) {
      stats->reached = (int64_t)c.reach[0];
      stats->nedge = (int64_t)(c.reach[1] / 2);
    } else {
      uint32_t root_r = 0, e = 0;
      G500_CUDA(cudaMemcpy(&root_r, g->d_reorder + root, sizeof(uint32_t), cudaMemcpyDeviceToHost));
      G500_CUDA(cudaMemcpy(&e, g->d_endp + root_r, sizeof(uint32_t), cudaMemcpyDeviceToHost));
      stats->reached = 1;
      stats->nedge = e / 2;
    }
    stats->num_levels = (int32_t)c.num_levels;
    stats->kernel_launches = p.deferred ? 2 : 1;
    if (c.t_init_ns >= c.t0_ns) stats->init_ms = (double)(c.t_init_ns - c.t0_ns) * 1e-6;
    if (c.t_end_ns >= c.t_init_ns) stats->search_ms = (double)(c.t_end_ns - c.t_init_ns) * 1e-6;
    if (c.num_levels) {
      std::vector<LevelRecord> rec(c.num_levels);
      G500_CUDA(cudaMemcpy(rec.data(), b->d_rec, sizeof(LevelRecord) * c.num_levels, cudaMemcpyDeviceToHost));
      for (const auto& r : rec) (r.direction ? stats->td_levels : stats->bu_levels)++;
    }
  }
  return G500_OK;
}

extern "C" int g500_bfs_level_stats(const g500_bfs* b, g500_level_stats* out, int max_levels, int* n) {
  if (!b) return set_error(G500_E_INVAL, "null bfs");
  const int total = (int)b->h_ctl->num_levels;
  if (n) *n = total;
  const int k = std::min(total, std::max(max_levels, 0));
  if (!out || k == 0) return G500_OK;
  G500_CUDA(cudaSetDevice(b->g->device));
  std::vector<LevelRecord> rec((size_t)k);
  G500_CUDA(cudaMemcpy(rec.data(), b->d_rec, sizeof(LevelRecord) * k, cudaMemcpyDeviceToHost));
  unsigned long long prev = b->h_ctl->t_init_ns;
  for (int i = 0; i < k; ++i) {
    const LevelRecord& r = rec[(size_t)i];
    g500_level_stats& o = out[i];
    o.direction = r.direction;
    o.level = r.level;
    o.frontier = (int64_t)r.frontier;
    o.discovered = (int64_t)r.discovered;
    o.scanned = (int64_t)r.scanned;
    o.edges_examined = (int64_t)r.edges;
    o.edge_sectors = (int64_t)r.sectors;
    o.device_ms = (double)(r.t_ns - prev) * 1e-6;  // %globaltimer between level barriers
    o.device_ms_tail = r.t_mid_ns ? (double)(r.t_ns - r.t_mid_ns) * 1e-6 : 0.0;
    prev = r.t_ns;
  }
  return G500_OK;
}

extern "C" int g500_bfs_device_pred(const g500_bfs* b, const int64_t** dev_pred) {
  if (!b || !dev_pred) return set_error(G500_E_INVAL, "null argument");
  *dev_pred = b->d_pred;
  return G500_OK;
}

extern "C" int g500_bfs_destroy(g500_bfs* b) { return bfs_free(b); }
