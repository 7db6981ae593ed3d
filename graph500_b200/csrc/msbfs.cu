// Batched multi-source BFS: up to 128 roots per call, W = 32/64/128 roots per
// launch as one bit-lane each in W-bit masks per vertex (visited V, frontier
// F, next N), with a uint8 level per (vertex, lane).  Each launch is one
// persistent cooperative kernel; every level is
//
//   pull   every vertex with unvisited lanes ORs its neighbours' frontier
//          masks until all its unvisited lanes are found (bottom-up with
//          early exit; VERTEX_REORDERING=2 puts hubs first in each row), or
//   push   every frontier vertex ORs its mask into its neighbours' next masks
//          (atomicOr into N, only the bits a neighbour still lacks),
//
// followed by settling the new lanes (V |= new; next F = new; levels): a
// pulling row settles itself, the hub rows (split across warps) and every
// row after a push settle in a pass of their own.  The frontier masks are
// double-buffered by level parity.  Pull or push is chosen per level from
// edge counts: pull when the new frontier's degree sum exceeds (degree sum of
// vertices with unvisited lanes) / alpha.  On large graphs a push level with
// a small frontier is sparse: it works on the vertices marked in frontier and
// touched bitmaps instead of on every vertex (kernel argument SP).
// Levels come out per root in original-id order through a shared-memory
// transpose; the whole launch sequence is captured once as a CUDA graph and
// replayed for every batch.
//
// The levels of each lane are exactly the BFS distances from its root, the
// same as (pred >> 48) of the plain BFS (bfs.hpp:1203, :2470).
#include "g500_internal.cuh"
#include "device_common.cuh"

#include <algorithm>
#include <chrono>

namespace g500 {

constexpr int MS_THREADS = 256;
constexpr int MS_MIN_BLOCKS = 4;
constexpr int MS_MAX_LANES = 128;
constexpr int MS_MAX_LEVEL = 254;  // level bytes: 255 marks unreached
// M_ROWS / M_SECT (counting launches only): row and chunk offset reads, and
// the 32-byte adjacency sectors the level's entries span
enum MsCounter { M_NEW = 0, M_NF, M_MF, M_MU, M_EDGES, M_ROWS, M_SECT, M_NUM = 8 };
enum MsErr { MS_ERR_DEPTH = 4 };

struct MsCtl {
  unsigned long long cnt[3][M_NUM];
  GridBarrier bar;
  unsigned num_levels;
  unsigned pull_levels;
  unsigned long long t0_ns, t_init_ns, t_end_ns;
  unsigned alive[3][4];      // lanes that found vertices in the phase (rotating like cnt)
  unsigned long long level_new[MS_MAX_LEVEL + 2];
  unsigned long long lane_deg[MS_MAX_LANES];  // sampled frontier degree sum per lane (lane survey)
  unsigned long long level_t_ns[MS_MAX_LEVEL + 2];
  unsigned long long level_mid_ns[MS_MAX_LEVEL + 2];  // end of the pull/push phase
  unsigned char level_pull[MS_MAX_LEVEL + 2];
  unsigned long long level_rows[MS_MAX_LEVEL + 2];  // counting launches: offset reads of the level
  unsigned long long level_sect[MS_MAX_LEVEL + 2];  // counting launches: adjacency sectors of the level
};

struct MsParams {
  const uint64_t* __restrict__ off;
  const uint32_t* __restrict__ deg;  // off[v + 1] - off[v]
  const uint32_t* __restrict__ col;
  const uint32_t* __restrict__ reorder;
  uint32_t* V;
  uint32_t* F[2];            // frontier masks by level parity: level l reads F[(l - 1) & 1], writes F[l & 1]
  uint32_t* N;
  uint8_t* L;                // [nlv][W] levels, 255 unreached
  const int64_t* roots;      // [nroots] original ids (device)
  const int* nroots_dev;     // number of roots of this launch (device, set with the roots)
  const uint2* hub_tab;      // pull: [nhub_chunks] (hub row, chunk index within the row)
  int64_t nhub_chunks;
  const uint32_t* hubs;      // pull: the hub rows themselves
  int64_t nhubs;
  const uint2* push_tab;     // push: [npush_chunks] the same for rows over MS_PUSH_HUB_DEG
  int64_t npush_chunks;
  // Sparse levels.  fb[l % 3] marks the vertices whose frontier mask level l
  // set (l = 0: the roots); `touched` marks the vertices a sparse push level
  // gave N bits (clear between levels).  A push level is sparse when the last
  // frontier's degree sum is at most sparse_limit.
  uint32_t* fb[3];           // [3][nwords]
  uint32_t* touched;         // [nwords]
  int64_t nwords;            // (nlv + 31) / 32
  int64_t sparse_limit;
  int64_t nlv;
  double alpha;
  MsCtl* ctl;
};

template <int NW>
struct Mask {
  uint32_t w[NW];
};

template <int NW>
__device__ __forceinline__ Mask<NW> load_mask(const uint32_t* p) {
  Mask<NW> m;
  if constexpr (NW == 4) {
    const uint4 x = __ldcg(reinterpret_cast<const uint4*>(p));
    m.w[0] = x.x; m.w[1] = x.y; m.w[2] = x.z; m.w[3] = x.w;
  } else if constexpr (NW == 2) {
    const uint2 x = __ldcg(reinterpret_cast<const uint2*>(p));
    m.w[0] = x.x; m.w[1] = x.y;
  } else {
    m.w[0] = __ldcg(p);
  }
  return m;
}

template <int NW>
__device__ __forceinline__ void store_mask(uint32_t* p, const Mask<NW>& m) {
  if constexpr (NW == 4) *reinterpret_cast<uint4*>(p) = make_uint4(m.w[0], m.w[1], m.w[2], m.w[3]);
  else if constexpr (NW == 2) *reinterpret_cast<uint2*>(p) = make_uint2(m.w[0], m.w[1]);
  else *p = m.w[0];
}

// Frontier masks gathered by the pull phase use plain loads, which may hit
// L1: hub rows recur in many adjacency lists.  The masks are rewritten by the
// apply pass of the same launch; the grid barrier between that pass and the
// next level (an acquire-release arrival on one side, an acquire fence once
// the arrival count is seen complete on the other) orders those writes before
// these loads.
template <int NW>
__device__ __forceinline__ Mask<NW> gather_mask(const uint32_t* p) {
  Mask<NW> m;
  if constexpr (NW == 4) {
    const uint4 x = *reinterpret_cast<const uint4*>(p);
    m.w[0] = x.x; m.w[1] = x.y; m.w[2] = x.z; m.w[3] = x.w;
  } else if constexpr (NW == 2) {
    const uint2 x = *reinterpret_cast<const uint2*>(p);
    m.w[0] = x.x; m.w[1] = x.y;
  } else {
    m.w[0] = *p;
  }
  return m;
}

// lanes [0, nroots) of word k
__device__ __forceinline__ uint32_t active_word(int nroots, int k) {
  const int lo = k * 32;
  if (nroots >= lo + 32) return ~0u;
  if (nroots <= lo) return 0u;
  return (1u << (nroots - lo)) - 1u;
}

template <int NW>
__device__ __forceinline__ bool covers(const Mask<NW>& acc, const Mask<NW>& need) {
  bool ok = true;
#pragma unroll
  for (int k = 0; k < NW; ++k) ok &= (acc.w[k] & need.w[k]) == need.w[k];
  return ok;
}

constexpr int MS_GROUPS = 4;           // dense push: groups of 32 rows whose frontier masks load together
constexpr int MS_WIN = 128;            // push: virtual edges a warp takes per window (4 per lane)
// Pull: rows up to MS_SMALL_DEG entries are walked by one thread, longer ones
// by a whole warp with a coverage check per step, and only rows of more than
// MS_HUB_DEG entries are split into chunks for several warps.  A chunk is
// scanned to its end whatever the row's coverage, while a walked row stops as
// soon as its needed lanes are found (at once for most high-degree rows), so
// splitting pays only for the very largest rows: with hub rows from 1024
// entries (1024-entry chunks) and single-thread rows up to 128, 64 roots took
// 1010 / 3719 / 16090 us at SCALE 22 / 24 / 26, against 894 / 2971 / 11349 us
// with these values.
constexpr int MS_SMALL_DEG = 256;      // pull: rows up to this long are walked by one thread
constexpr int MS_UNROLL = 4;           // pull: neighbours each thread loads per step
constexpr int MS_HUB_DEG = 1 << 20;    // pull: rows longer than this are hub rows, split across warps
constexpr int MS_HUB_CHUNK = 16384;    // pull: edges of a hub row one warp takes at a time
constexpr int MS_PUSH_HUB_DEG = 256;   // push: the same two, smaller: a push walks every edge of its
constexpr int MS_PUSH_CHUNK = 256;     //   frontier rows, so short chunks spread the few hub rows wider


// byte mask of the 4 lanes whose bits are set in nib (bit i -> byte i)
__device__ __forceinline__ uint32_t nibble_bytes(uint32_t nib) {
  return ((nib * 0x00204081u) & 0x01010101u) * 0xFFu;
}

// level bytes of a row: for each 16-lane group with new lanes, write the
// group's 16 bytes (new lanes = level, unvisited lanes = 255, lanes visited
// before keep their byte, read back only when the group has such lanes).
// Groups without visited lanes are never written; the output pass reads
// them as 255 from the visited mask.
template <int NW>
__device__ __forceinline__ void write_levels(uint8_t* row, const Mask<NW>& nw, const Mask<NW>& vv, uint32_t lvl4) {
#pragma unroll
  for (int g = 0; g < 2 * NW; ++g) {
    const uint32_t bits = (nw.w[g >> 1] >> ((g & 1) * 16)) & 0xFFFFu;
    if (!bits) continue;
    const uint32_t old = (vv.w[g >> 1] >> ((g & 1) * 16)) & 0xFFFFu;
    uint4* dst = reinterpret_cast<uint4*>(row) + g;
    uint4 o = make_uint4(~0u, ~0u, ~0u, ~0u);
    if (old) o = __ldcg(dst);
    uint32_t w[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t bm = nibble_bytes((bits >> (4 * i)) & 0xFu);
      w[i] = (w[i] & ~bm) | (lvl4 & bm);
    }
    *dst = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// 32-byte sectors spanned by the k adjacency entries (4 bytes each) at b
__device__ __forceinline__ unsigned long long sector_span(uint64_t b, uint64_t k) {
  return k ? ((b + k - 1) >> 3) - (b >> 3) + 1 : 0;
}

// Per-thread counters of a level, flushed once per block at its end; fb is
// the level's frontier bitmap, track whether its push marks touched vertices.
template <int NW>
struct LevelAcc {
  unsigned long long nnew, nf, mf, mu;
  unsigned long long rows, sect;  // counting launches only
  Mask<NW> lanes;  // lanes that found vertices
  uint32_t* fb;
  bool track;
  __device__ void clear() {
    nnew = nf = mf = mu = rows = sect = 0;
#pragma unroll
    for (int k = 0; k < NW; ++k) lanes.w[k] = 0;
  }
};

// Vertex v (visited lanes vv, still-needed lanes need) found lanes nw this
// level: its next-frontier mask (always written: the buffer holds an older
// level), visited mask, level bytes and the counters of the direction rule.
// Returns whether v found lanes (then it is marked in the level's frontier bitmap).
template <int NW>
__device__ __forceinline__ bool settle(const MsParams& p, uint32_t* Fn, int64_t v, const Mask<NW>& vv,
                                       const Mask<NW>& need, const Mask<NW>& nw, uint32_t deg, uint32_t lvl4,
                                       LevelAcc<NW>& a) {
  constexpr int W = 32 * NW;
  store_mask<NW>(Fn + v * NW, nw);
  bool anynew = false, left = false;
#pragma unroll
  for (int k = 0; k < NW; ++k) {
    anynew |= nw.w[k] != 0;
    left |= (need.w[k] & ~nw.w[k]) != 0;
  }
  if (anynew) {
    Mask<NW> vn;
#pragma unroll
    for (int k = 0; k < NW; ++k) vn.w[k] = vv.w[k] | nw.w[k];
    store_mask<NW>(p.V + v * NW, vn);
    write_levels<NW>(p.L + v * W, nw, vv, lvl4);
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      a.lanes.w[k] |= nw.w[k];
      a.nnew += __popc(nw.w[k]);
    }
    ++a.nf;
    a.mf += deg;
  }
  if (left) a.mu += deg;  // still has unvisited live lanes after this level
  return anynew;
}

// pull over non-hub rows.  A row of at most MS_SMALL_DEG edges is walked by
// its own thread, MS_UNROLL neighbours per step; a longer one by the whole
// warp, 32 * MS_UNROLL neighbours per step (rows taken in turn).  Either stops
// once the row's unvisited lanes are all found; under VERTEX_REORDERING=2 a
// row lists its highest-degree neighbours first, which find most of them.
// Each row is its own only writer, so it settles at once (next frontier,
// visited mask, levels): pull levels need no separate apply pass over all
// vertices, only one over the hub rows.
// INTO_N (a level that pulls some lanes and pushes the others): a row's
// finds go into its next mask N, beside the push's, for the apply pass to
// settle, instead of settling here.
template <int NW, bool INTO_N, bool COUNT, bool SP>
__device__ void ms_pull_rows(const MsParams& p, const Mask<NW>& act, const uint32_t* Fc, uint32_t* Fn,
                             uint32_t lvl4, LevelAcc<NW>& la) {
  const int lane = threadIdx.x & 31;
  for (int64_t base = gwarp_id() * 32; base < p.nlv; base += gwarp_count() * 32) {
    const int64_t v = base + lane;
    Mask<NW> need, acc, vv;
    bool any = false;
    uint32_t deg = 0;
    uint64_t rb = 0;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      acc.w[k] = 0;
      need.w[k] = 0;
      vv.w[k] = 0;
    }
    if (v < p.nlv) {
      vv = load_mask<NW>(p.V + v * NW);
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        need.w[k] = act.w[k] & ~vv.w[k];
        any |= need.w[k] != 0;
      }
      if (any) {
        rb = __ldg(p.off + v);
        deg = __ldg(p.deg + v);
      }
    }
    if (any && deg <= (uint32_t)MS_SMALL_DEG) {
      const uint64_t re = rb + deg;
      uint64_t e = rb;
      for (; e < re; e += MS_UNROLL) {
        uint32_t nb[MS_UNROLL];
#pragma unroll
        for (int t = 0; t < MS_UNROLL; ++t) nb[t] = e + t < re ? __ldg(p.col + e + t) : NO_VERTEX;
#pragma unroll
        for (int t = 0; t < MS_UNROLL; ++t)
          if (nb[t] != NO_VERTEX) {
            const Mask<NW> f = gather_mask<NW>(Fc + (int64_t)nb[t] * NW);
#pragma unroll
            for (int q = 0; q < NW; ++q) acc.w[q] |= f.w[q];
          }
        if (covers<NW>(acc, need)) break;
      }
      if constexpr (COUNT) {
        const uint64_t k = (e + MS_UNROLL < re ? e + MS_UNROLL : re) - rb;
        ++la.rows;
        la.sect += sector_span(rb, k);
      }
    }
    unsigned rows = __ballot_sync(FULL_MASK, any && deg > (uint32_t)MS_SMALL_DEG && deg <= (uint32_t)MS_HUB_DEG);
    while (rows) {
      const int src = __ffs(rows) - 1;
      rows &= rows - 1;
      const uint64_t b = __shfl_sync(FULL_MASK, rb, src);
      const uint64_t e = b + __shfl_sync(FULL_MASK, deg, src);
      Mask<NW> nd, a;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        nd.w[k] = __shfl_sync(FULL_MASK, need.w[k], src);
        a.w[k] = 0;
      }
      uint64_t j = b;
      for (; j < e; j += 32 * MS_UNROLL) {
        uint32_t nb[MS_UNROLL];
#pragma unroll
        for (int t = 0; t < MS_UNROLL; ++t) {
          const uint64_t i = j + t * 32 + lane;
          nb[t] = i < e ? __ldg(p.col + i) : NO_VERTEX;
        }
        Mask<NW> x;
#pragma unroll
        for (int k = 0; k < NW; ++k) x.w[k] = 0;
#pragma unroll
        for (int t = 0; t < MS_UNROLL; ++t)
          if (nb[t] != NO_VERTEX) {
            const Mask<NW> f = gather_mask<NW>(Fc + (int64_t)nb[t] * NW);
#pragma unroll
            for (int q = 0; q < NW; ++q) x.w[q] |= f.w[q];
          }
#pragma unroll
        for (int k = 0; k < NW; ++k) a.w[k] |= __reduce_or_sync(FULL_MASK, x.w[k]);
        if (covers<NW>(a, nd)) break;
      }
      if (lane == src) {
        acc = a;
        if constexpr (COUNT) {
          ++la.rows;
          la.sect += sector_span(b, (j + 32 * MS_UNROLL < e ? j + 32 * MS_UNROLL : e) - b);
        }
      }
    }
    // hub rows settle after the hub phase (deg is 0 here for rows without needed lanes)
    bool app = false;
    if (v < p.nlv && deg <= (uint32_t)MS_HUB_DEG) {
      Mask<NW> nw;
#pragma unroll
      for (int k = 0; k < NW; ++k) nw.w[k] = acc.w[k] & need.w[k];
      if constexpr (INTO_N) {
#pragma unroll
        for (int k = 0; k < NW; ++k)
          if (nw.w[k]) atomicOr(p.N + v * NW + k, nw.w[k]);
      } else {
        app = settle<NW>(p, Fn, v, vv, need, nw, deg, lvl4, la);
      }
    }
    if constexpr (SP && !INTO_N) {  // the warp's 32 vertices are one word of the frontier bitmap
      const unsigned word = __ballot_sync(FULL_MASK, app);
      if (lane == 0 && base < p.nlv) la.fb[base >> 5] = word;
    }
  }
}

// Hub rows are split into fixed-size chunks (MS_HUB_CHUNK edges for pull,
// MS_PUSH_CHUNK for push), listed as (row, chunk index within the row).  Warp
// w owns chunks w, w + nwarps, ...; it reads 32 of its chunk headers at once
// (one per lane) and works, in turn, only on the chunks whose row takes part
// in the level.  A pull chunk stops early once its row's lanes are found, so
// pull chunks are long; a push chunk walks all its edges, so push chunks are
// short and spread the hub rows of a small frontier over more warps.
template <int CHUNK>
__device__ __forceinline__ void hub_bounds(const MsParams& p, uint32_t h, uint32_t k, uint64_t* b, uint64_t* e) {
  const uint64_t rb = __ldg(p.off + h);
  const uint64_t re = rb + __ldg(p.deg + h);
  *b = rb + (uint64_t)k * CHUNK;
  *e = *b + CHUNK < re ? *b + CHUNK : re;
}

// pull over hub rows: each chunk ORs its neighbours' frontier masks, stopping
// once the row's unvisited lanes are covered, into the row's next mask
template <int NW, bool COUNT>
__device__ void ms_pull_hubs(const MsParams& p, const Mask<NW>& act, const uint32_t* Fc, LevelAcc<NW>& la) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = gwarp_count();
  for (int64_t c0 = gwarp_id(); c0 < p.nhub_chunks; c0 += 32 * nwarps) {
    const int64_t c = c0 + lane * nwarps;
    uint2 hd = make_uint2(0, 0);
    Mask<NW> need;
    bool any = false;
#pragma unroll
    for (int k = 0; k < NW; ++k) need.w[k] = 0;
    if (c < p.nhub_chunks) {
      hd = __ldg(p.hub_tab + c);
      const Mask<NW> vv = load_mask<NW>(p.V + (int64_t)hd.x * NW);
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        need.w[k] = act.w[k] & ~vv.w[k];
        any |= need.w[k] != 0;
      }
    }
    unsigned todo = __ballot_sync(FULL_MASK, any);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t h = __shfl_sync(FULL_MASK, hd.x, src);
      const uint32_t kk = __shfl_sync(FULL_MASK, hd.y, src);
      Mask<NW> nd, a;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        nd.w[k] = __shfl_sync(FULL_MASK, need.w[k], src);
        a.w[k] = 0;
      }
      uint64_t b, e;
      hub_bounds<MS_HUB_CHUNK>(p, h, kk, &b, &e);
      uint64_t j = b;
      for (; j < e; j += 32 * MS_UNROLL) {
        uint32_t nb[MS_UNROLL];
#pragma unroll
        for (int t = 0; t < MS_UNROLL; ++t) {
          const uint64_t i = j + t * 32 + lane;
          nb[t] = i < e ? __ldg(p.col + i) : NO_VERTEX;
        }
        Mask<NW> x;
#pragma unroll
        for (int k = 0; k < NW; ++k) x.w[k] = 0;
#pragma unroll
        for (int t = 0; t < MS_UNROLL; ++t)
          if (nb[t] != NO_VERTEX) {
            const Mask<NW> f = gather_mask<NW>(Fc + (int64_t)nb[t] * NW);
#pragma unroll
            for (int q = 0; q < NW; ++q) x.w[q] |= f.w[q];
          }
#pragma unroll
        for (int k = 0; k < NW; ++k) a.w[k] |= __reduce_or_sync(FULL_MASK, x.w[k]);
        if (covers<NW>(a, nd)) break;
      }
      if constexpr (COUNT)
        if (lane == 0) {
          ++la.rows;
          la.sect += sector_span(b, (j + 32 * MS_UNROLL < e ? j + 32 * MS_UNROLL : e) - b);
        }
      if (lane < NW) {
        uint32_t x = 0;
#pragma unroll
        for (int k = 0; k < NW; ++k)
          if (k == lane) x = a.w[k] & nd.w[k];
        if (x) atomicOr(p.N + (int64_t)h * NW + lane, x);
      }
    }
  }
}

// The lanes of fo that w still lacks go into N[w]; with track, w is marked
// touched when it got some.
template <int NW>
__device__ __forceinline__ void push_to(const MsParams& p, uint32_t w, const Mask<NW>& fo, bool track) {
  const Mask<NW> vw = load_mask<NW>(p.V + (int64_t)w * NW);
  bool any = false;
#pragma unroll
  for (int q = 0; q < NW; ++q) {
    const uint32_t add = fo.w[q] & ~vw.w[q];
    if (add) {
      atomicOr(p.N + (int64_t)w * NW + q, add);
      any = true;
    }
  }
  if (any && track) atomicOr(p.touched + (w >> 5), 1u << (w & 31));
}

// push from hub frontier rows: every neighbour of the chunk gets the lanes it
// still lacks
template <int NW, bool COUNT>
__device__ void ms_push_hubs(const MsParams& p, const uint32_t* Fc, const Mask<NW>& qm, LevelAcc<NW>& la) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = gwarp_count();
  for (int64_t c0 = gwarp_id(); c0 < p.npush_chunks; c0 += 32 * nwarps) {
    const int64_t c = c0 + lane * nwarps;
    uint2 hd = make_uint2(0, 0);
    Mask<NW> f;
    bool any = false;
#pragma unroll
    for (int k = 0; k < NW; ++k) f.w[k] = 0;
    if (c < p.npush_chunks) {
      hd = __ldg(p.push_tab + c);
      f = load_mask<NW>(Fc + (int64_t)hd.x * NW);
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        f.w[k] &= qm.w[k];
        any |= f.w[k] != 0;
      }
    }
    unsigned todo = __ballot_sync(FULL_MASK, any);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t h = __shfl_sync(FULL_MASK, hd.x, src);
      const uint32_t kk = __shfl_sync(FULL_MASK, hd.y, src);
      Mask<NW> fo;
#pragma unroll
      for (int k = 0; k < NW; ++k) fo.w[k] = __shfl_sync(FULL_MASK, f.w[k], src);
      uint64_t b, e;
      hub_bounds<MS_PUSH_CHUNK>(p, h, kk, &b, &e);
      if constexpr (COUNT)
        if (lane == 0) {
          ++la.rows;
          la.sect += sector_span(b, e - b);
        }
      for (uint64_t j = b; j < e; j += 32 * MS_UNROLL) {
        uint32_t nb[MS_UNROLL];
#pragma unroll
        for (int t = 0; t < MS_UNROLL; ++t) {
          const uint64_t i = j + t * 32 + lane;
          nb[t] = i < e ? __ldg(p.col + i) : NO_VERTEX;
        }
#pragma unroll
        for (int t = 0; t < MS_UNROLL; ++t)
          if (nb[t] != NO_VERTEX) push_to<NW>(p, nb[t], fo, la.track);
      }
    }
  }
}

// push from non-hub frontier rows (graphs without sparse levels: every
// vertex's frontier mask is read): the frontier masks of MS_GROUPS groups of
// 32 rows are loaded together; each group holding frontier rows has their
// edges walked as one list, MS_WIN at a time; every neighbour gets the lanes
// it still lacks.
template <int NW, bool COUNT>
__device__ void ms_push_rows_dense(const MsParams& p, const uint32_t* Fc, const Mask<NW>& qm, LevelAcc<NW>& la) {
  const int lane = threadIdx.x & 31;
  for (int64_t base = gwarp_id() * (32 * MS_GROUPS); base < p.nlv; base += gwarp_count() * (32 * MS_GROUPS)) {
    Mask<NW> fg[MS_GROUPS];
#pragma unroll
    for (int g = 0; g < MS_GROUPS; ++g) {
      const int64_t v = base + g * 32 + lane;
      if (v < p.nlv) {
        fg[g] = load_mask<NW>(Fc + v * NW);
#pragma unroll
        for (int k = 0; k < NW; ++k) fg[g].w[k] &= qm.w[k];
      } else {
#pragma unroll
        for (int k = 0; k < NW; ++k) fg[g].w[k] = 0;
      }
    }
#pragma unroll
    for (int g = 0; g < MS_GROUPS; ++g) {
      const int64_t v = base + g * 32 + lane;
      const Mask<NW> f = fg[g];
      bool any = false;
#pragma unroll
      for (int k = 0; k < NW; ++k) any |= f.w[k] != 0;
      if (!__any_sync(FULL_MASK, any)) continue;
      uint64_t cur = 0, re = 0;
      if (any) {
        cur = __ldg(p.off + v);
        re = cur + __ldg(p.deg + v);
        if (re - cur > (uint64_t)MS_PUSH_HUB_DEG) cur = re;  // hub row: the hub phase pushes it
        if constexpr (COUNT)
          if (re > cur) {
            ++la.rows;
            la.sect += sector_span(cur, re - cur);
          }
      }
      for (;;) {
        const uint32_t rem = (uint32_t)((re - cur) < (uint64_t)MS_WIN ? (re - cur) : (uint64_t)MS_WIN);
        const uint32_t incl = warp_incl_scan(rem);
        const uint32_t excl = incl - rem;
        const uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
        if (total == 0) break;
#pragma unroll
        for (int j = 0; j < MS_WIN / 32; ++j) {
          const uint32_t k = j * 32 + lane;
          const int o = owner_lane(excl, k);
          const uint64_t co = __shfl_sync(FULL_MASK, cur, o);
          const uint32_t exo = __shfl_sync(FULL_MASK, excl, o);
          Mask<NW> fo;
#pragma unroll
          for (int q = 0; q < NW; ++q) fo.w[q] = __shfl_sync(FULL_MASK, f.w[q], o);
          if (k < total) {
            const int64_t w = __ldg(p.col + co + (k - exo));
            const Mask<NW> vw = load_mask<NW>(p.V + w * NW);
#pragma unroll
            for (int q = 0; q < NW; ++q) {
              const uint32_t add = fo.w[q] & ~vw.w[q];
              if (add) atomicOr(p.N + w * NW + q, add);
            }
          }
        }
        cur += excl >= (uint32_t)MS_WIN ? 0u : min(rem, (uint32_t)MS_WIN - excl);
      }
    }
  }
}

// push from non-hub frontier rows: the rows marked in fbc (the last level's
// frontier bitmap), gathered 32 at a time from each warp's 32 words, so that
// a small frontier costs a pass over its bitmap and not over every vertex;
// each batch of rows has its edges walked as one list, MS_WIN at a time;
// every neighbour gets the lanes it still lacks.
template <int NW, bool COUNT>
__device__ void ms_push_rows_marked(const MsParams& p, const uint32_t* Fc, const uint32_t* fbc, const Mask<NW>& qm,
                             LevelAcc<NW>& la) {
  const int lane = threadIdx.x & 31;
  for (int64_t wb = gwarp_id() * 32; wb < p.nwords; wb += gwarp_count() * 32) {
    const int64_t wi = wb + lane;
    const uint32_t mw = wi < p.nwords ? __ldcg(fbc + wi) : 0u;
    const uint32_t c = __popc(mw);
    const uint32_t incl_w = warp_incl_scan(c);
    const uint32_t excl_w = incl_w - c;
    const uint32_t nrows = __shfl_sync(FULL_MASK, incl_w, 31);
    for (uint32_t b0 = 0; b0 < nrows; b0 += 32) {
      const uint32_t idx = b0 + lane;
      const int ow = owner_lane(excl_w, idx);
      const uint32_t mwo = __shfl_sync(FULL_MASK, mw, ow);
      const uint32_t exw = __shfl_sync(FULL_MASK, excl_w, ow);
      Mask<NW> f;
      bool any = false;
#pragma unroll
      for (int k = 0; k < NW; ++k) f.w[k] = 0;
      uint64_t cur = 0, re = 0;
      if (idx < nrows) {
        const int64_t v = (wb + ow) * 32 + select_bit(mwo, idx - exw);
        f = load_mask<NW>(Fc + v * NW);
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          f.w[k] &= qm.w[k];
          any |= f.w[k] != 0;
        }
        if (any) {
          cur = __ldg(p.off + v);
          re = cur + __ldg(p.deg + v);
          if (re - cur > (uint64_t)MS_PUSH_HUB_DEG) cur = re;  // hub row: the hub phase pushes it
          if constexpr (COUNT)
            if (re > cur) {
              ++la.rows;
              la.sect += sector_span(cur, re - cur);
            }
        }
      }
      for (;;) {
        const uint32_t rem = (uint32_t)((re - cur) < (uint64_t)MS_WIN ? (re - cur) : (uint64_t)MS_WIN);
        const uint32_t incl = warp_incl_scan(rem);
        const uint32_t excl = incl - rem;
        const uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
        if (total == 0) break;
#pragma unroll
        for (int j = 0; j < MS_WIN / 32; ++j) {
          const uint32_t k = j * 32 + lane;
          const int o = owner_lane(excl, k);
          const uint64_t co = __shfl_sync(FULL_MASK, cur, o);
          const uint32_t exo = __shfl_sync(FULL_MASK, excl, o);
          Mask<NW> fo;
#pragma unroll
          for (int q = 0; q < NW; ++q) fo.w[q] = __shfl_sync(FULL_MASK, f.w[q], o);
          if (k < total) push_to<NW>(p, __ldg(p.col + co + (k - exo)), fo, la.track);
        }
        cur += excl >= (uint32_t)MS_WIN ? 0u : min(rem, (uint32_t)MS_WIN - excl);
      }
    }
  }
}

// apply after a push level: new = N & needed lanes; settle every vertex (its
// next-frontier mask is always written).  U vertices per thread per step,
// loads first; each warp's 32 vertices of a step are one word of the
// frontier bitmap.
template <int NW, bool SP>
__device__ void ms_apply(const MsParams& p, const Mask<NW>& act, uint32_t* Fn, uint32_t lvl4, LevelAcc<NW>& la) {
  constexpr int U = NW == 4 ? 2 : 4;
  const int lane = threadIdx.x & 31;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v0w = tid - lane; v0w < p.nlv; v0w += nthreads * U) {  // v0w: the warp's first vertex (uniform)
    const int64_t v0 = v0w + lane;
    Mask<NW> n[U], vv[U];
    uint32_t dg[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t v = v0 + u * nthreads;
      if (v < p.nlv) {
        n[u] = load_mask<NW>(p.N + v * NW);
        vv[u] = load_mask<NW>(p.V + v * NW);
        dg[u] = __ldg(p.deg + v);
      } else {
        dg[u] = 0;
#pragma unroll
        for (int k = 0; k < NW; ++k) n[u].w[k] = vv[u].w[k] = 0;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t v = v0 + u * nthreads;
      bool app = false;
      if (v < p.nlv) {
        Mask<NW> need, nw;
        bool anyn = false;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          need.w[k] = act.w[k] & ~vv[u].w[k];
          nw.w[k] = n[u].w[k] & need.w[k];
          anyn |= n[u].w[k] != 0;
        }
        if (anyn) {
          Mask<NW> zero;
#pragma unroll
          for (int k = 0; k < NW; ++k) zero.w[k] = 0;
          store_mask<NW>(p.N + v * NW, zero);
        }
        app = settle<NW>(p, Fn, v, vv[u], need, nw, dg[u], lvl4, la);
      }
      if constexpr (SP) {
        const unsigned word = __ballot_sync(FULL_MASK, app);
        const int64_t vw = v0w + u * nthreads;  // a multiple of 32
        if (lane == 0 && vw < p.nlv) la.fb[vw >> 5] = word;
      }
    }
  }
}

// apply after a sparse push level: only the touched vertices have N bits, so
// only they settle (each warp gathers the marked vertices of its 32 words,
// 32 at a time, and clears the words); every other vertex's next-frontier
// mask is clear already (the push phase cleared the masks the buffer held
// from two levels before, and this level's frontier bitmap).  Mu, the degree
// sum of vertices with needed lanes left, is not summed here (the caller
// keeps the last one).
template <int NW>
__device__ void ms_apply_marked(const MsParams& p, const Mask<NW>& act, uint32_t* Fn, uint32_t lvl4,
                                LevelAcc<NW>& la) {
  const int lane = threadIdx.x & 31;
  for (int64_t wb = gwarp_id() * 32; wb < p.nwords; wb += gwarp_count() * 32) {
    const int64_t wi = wb + lane;
    const uint32_t mw = wi < p.nwords ? __ldcg(p.touched + wi) : 0u;
    if (mw) p.touched[wi] = 0;
    const uint32_t c = __popc(mw);
    const uint32_t incl = warp_incl_scan(c);
    const uint32_t excl = incl - c;
    const uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
    for (uint32_t b0 = 0; b0 < total; b0 += 32) {
      const uint32_t idx = b0 + lane;
      const int o = owner_lane(excl, idx);
      const uint32_t mwo = __shfl_sync(FULL_MASK, mw, o);
      const uint32_t exo = __shfl_sync(FULL_MASK, excl, o);
      if (idx < total) {
        const int64_t v = (wb + o) * 32 + select_bit(mwo, idx - exo);
        const Mask<NW> n = load_mask<NW>(p.N + v * NW);
        const Mask<NW> vv = load_mask<NW>(p.V + v * NW);
        Mask<NW> need, nw, zero;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          need.w[k] = act.w[k] & ~vv.w[k];
          nw.w[k] = n.w[k] & need.w[k];
          zero.w[k] = 0;
        }
        store_mask<NW>(p.N + v * NW, zero);
        if (settle<NW>(p, Fn, v, vv, need, nw, __ldg(p.deg + v), lvl4, la))
          atomicOr(la.fb + (v >> 5), 1u << (v & 31));
      }
    }
  }
}

// the next-frontier masks of the vertices marked in fb_old (the level two
// before, whose masks the buffer still holds) cleared, and fb_new (this
// level's frontier bitmap, last written three levels before) cleared
template <int NW>
__device__ void ms_clear_marked(const MsParams& p, uint32_t* Fn, const uint32_t* fb_old, uint32_t* fb_new) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  Mask<NW> zero;
#pragma unroll
  for (int k = 0; k < NW; ++k) zero.w[k] = 0;
  for (int64_t wi = tid; wi < p.nwords; wi += nthreads) {
    uint32_t m = fb_old ? __ldcg(fb_old + wi) : 0u;
    fb_new[wi] = 0;
    while (m) {
      const int b = __ffs(m) - 1;
      m &= m - 1;
      store_mask<NW>(Fn + (wi * 32 + b) * NW, zero);
    }
  }
}

// after a pull level: the hub rows, whose chunks ORed into N
template <int NW, bool SP>
__device__ void ms_settle_hubs(const MsParams& p, const Mask<NW>& act, uint32_t* Fn, uint32_t lvl4,
                               LevelAcc<NW>& la) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = tid; i < p.nhubs; i += nthreads) {
    const uint32_t h = __ldg(p.hubs + i);
    const Mask<NW> n = load_mask<NW>(p.N + (int64_t)h * NW);
    const Mask<NW> vv = load_mask<NW>(p.V + (int64_t)h * NW);
    Mask<NW> need, nw;
    bool anyn = false;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      need.w[k] = act.w[k] & ~vv.w[k];
      nw.w[k] = n.w[k] & need.w[k];
      anyn |= n.w[k] != 0;
    }
    if (anyn) {
      Mask<NW> zero;
#pragma unroll
      for (int k = 0; k < NW; ++k) zero.w[k] = 0;
      store_mask<NW>(p.N + (int64_t)h * NW, zero);
    }
    const bool app = settle<NW>(p, Fn, h, vv, need, nw, __ldg(p.deg + h), lvl4, la);
    if constexpr (SP)
      if (app) atomicOr(la.fb + (h >> 5), 1u << (h & 31));  // the pull phase wrote its bit clear
  }
}

// Lane survey before a level that would pull: the frontier degree sum of each
// lane, estimated from every MS_SURVEY_STEP-th vertex.  A lane with a small
// frontier finds few vertices at this level, yet while any of its vertices
// stay unfound every row that still needs it is scanned to its end; such
// lanes are pushed instead.  Per 32 sampled vertices a warp reduces each
// lane bit's degrees (lane b of the warp keeps bits b, b + 32, ...), then
// the block adds them up in shared memory and once into ctl->lane_deg.
constexpr int MS_SURVEY_STEP = 8;
constexpr int MS_SURVEY_DIV = 64;  // a lane is pushed when its frontier degree sum is under entries / this
constexpr int MS_SURVEY_LEVELS = 1;  // pull levels that survey (the first ones)
template <int NW>
__device__ void ms_lane_survey(const MsParams& p, const uint32_t* Fc, unsigned long long* sh_lane) {
  const int lane = threadIdx.x & 31;
  unsigned long long acc[NW];
#pragma unroll
  for (int k = 0; k < NW; ++k) acc[k] = 0;
  const int64_t nsample = (p.nlv + MS_SURVEY_STEP - 1) / MS_SURVEY_STEP;
  for (int64_t base = gwarp_id() * 32; base < nsample; base += gwarp_count() * 32) {
    const int64_t v = (base + lane) * MS_SURVEY_STEP;
    Mask<NW> f;
    uint32_t d = 0;
#pragma unroll
    for (int k = 0; k < NW; ++k) f.w[k] = 0;
    if (v < p.nlv) {
      f = load_mask<NW>(Fc + v * NW);
      d = __ldg(p.deg + v);
    }
    bool any = false;
#pragma unroll
    for (int k = 0; k < NW; ++k) any |= f.w[k] != 0;
    if (!__any_sync(FULL_MASK, any)) continue;
#pragma unroll
    for (int k = 0; k < NW; ++k)
      for (int b = 0; b < 32; ++b) {
        const unsigned sum = __reduce_add_sync(FULL_MASK, ((f.w[k] >> b) & 1u) ? d : 0u);
        if (lane == b) acc[k] += sum;
      }
  }
#pragma unroll
  for (int k = 0; k < NW; ++k)
    if (acc[k]) atomicAdd(&sh_lane[k * 32 + lane], acc[k]);
}

// the level's counters into the block accumulators, and the lanes that found
// vertices (the others have finished their BFS) into alive_out
template <int NW, bool COUNT>
__device__ void flush_level(const LevelAcc<NW>& la, unsigned long long* sh_acc, unsigned* sh_or,
                            unsigned* alive_out) {
  if constexpr (COUNT) {
    block_add(sh_acc, M_ROWS, la.rows);
    block_add(sh_acc, M_SECT, la.sect);
  }
  block_add(sh_acc, M_NEW, la.nnew);
  block_add(sh_acc, M_NF, la.nf);
  block_add(sh_acc, M_MF, la.mf);
  block_add(sh_acc, M_MU, la.mu);
#pragma unroll
  for (int k = 0; k < NW; ++k) {
    const unsigned x = __reduce_or_sync(FULL_MASK, la.lanes.w[k]);
    if ((threadIdx.x & 31) == 0 && x) atomicOr(&sh_or[k], x);
  }
  __syncthreads();
  if (threadIdx.x < NW) {
    if (sh_or[threadIdx.x]) atomicOr(&alive_out[threadIdx.x], sh_or[threadIdx.x]);
    sh_or[threadIdx.x] = 0;
  }
}

// COUNT: a counting launch, which also records each level's offset reads and
// adjacency sectors (the bytes model of the batched form); compiled apart so
// that the timed launches carry none of it.
// SP: sparse levels (frontier and touched bitmaps) are kept; without, every
// level works on every vertex (smaller graphs, where that costs less).
template <int NW, bool COUNT, bool SP>
__global__ void __launch_bounds__(MS_THREADS, MS_MIN_BLOCKS) msbfs_kernel(MsParams p) {
  constexpr int W = 32 * NW;
  __shared__ unsigned long long sh_cnt[M_NUM];
  __shared__ unsigned long long sh_acc[M_NUM];
  __shared__ unsigned sh_flag;
  __shared__ unsigned sh_or[4];
  MsCtl* ctl = p.ctl;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  if (threadIdx.x < M_NUM) sh_acc[threadIdx.x] = 0;
  if (threadIdx.x < 4) sh_or[threadIdx.x] = 0;
  const int nroots = *p.nroots_dev;
  Mask<NW> act;
#pragma unroll
  for (int k = 0; k < NW; ++k) act.w[k] = active_word(nroots, k);

  if (tid == 0) ctl->t0_ns = globaltimer();
  {
    Mask<NW> zero;
#pragma unroll
    for (int k = 0; k < NW; ++k) zero.w[k] = 0;
    for (int64_t v = tid; v < p.nlv; v += nthreads) {  // SP: level 1 may settle only the vertices it touches
      store_mask<NW>(p.V + v * NW, zero);               // (otherwise F[1] is written whole by level 1)
      store_mask<NW>(p.F[0] + v * NW, zero);
      if constexpr (SP) store_mask<NW>(p.F[1] + v * NW, zero);
      store_mask<NW>(p.N + v * NW, zero);
    }
    if constexpr (SP)
      for (int64_t w = tid; w < p.nwords; w += nthreads) {
        p.touched[w] = 0;
        p.fb[0][w] = 0;
      }
  }
  if (blockIdx.x == 0 && threadIdx.x < 3 * M_NUM) (&ctl->cnt[0][0])[threadIdx.x] = 0;
  if (blockIdx.x == 0 && threadIdx.x < 12) (&ctl->alive[0][0])[threadIdx.x] = 0;
  if (!grid_sync<M_NUM>(&ctl->bar, nullptr, sh_acc, nullptr, sh_cnt, &sh_flag)) return;

  // roots: lane i starts at reorder[root_i] (a root outside the CSR range has
  // no edges; its level 0 is written by the output pass)
  if (tid < nroots) {
    const uint32_t r = __ldg(p.reorder + p.roots[tid]);
    if ((int64_t)r < p.nlv) {
      atomicOr(p.V + (int64_t)r * NW + tid / 32, 1u << (tid & 31));
      atomicOr(p.F[0] + (int64_t)r * NW + tid / 32, 1u << (tid & 31));
      p.L[(int64_t)r * W + tid] = 0;
      if constexpr (SP) atomicOr(p.fb[0] + (r >> 5), 1u << (r & 31));  // level 0's frontier bitmap
    }
  }
  if (!grid_sync<M_NUM>(&ctl->bar, nullptr, sh_acc, nullptr, sh_cnt, &sh_flag)) return;

  if (tid == 0) ctl->t_init_ns = globaltimer();
  bool pull = false;  // the first frontier is a handful of roots
  int surveys = 0;
  unsigned phase = 0, pulls = 0;
  int level = 1;
  __shared__ unsigned long long sh_lane[MS_MAX_LANES];
  __shared__ uint32_t sh_qm[4];
  const unsigned long long survey_thr = __ldg(p.off + p.nlv) / ((unsigned long long)MS_SURVEY_DIV * MS_SURVEY_STEP);
  unsigned long long mu_last = __ldg(p.off + p.nlv);  // every vertex needs every lane
  unsigned long long mf_last = 0;                     // level 1: the roots' rows
  for (;; ++level) {
    unsigned long long* cnt = ctl->cnt[phase % 3];
    unsigned* alive = ctl->alive[phase % 3];
    if (blockIdx.x == 0 && threadIdx.x < M_NUM) ctl->cnt[(phase + 1) % 3][threadIdx.x] = 0;
    if (blockIdx.x == 0 && threadIdx.x < 4) ctl->alive[(phase + 1) % 3][threadIdx.x] = 0;
    const uint32_t* Fc = p.F[(level - 1) & 1];
    uint32_t* Fn = p.F[level & 1];
    const uint32_t lvl4 = (uint32_t)level * 0x01010101u;
    LevelAcc<NW> la;
    la.clear();
    la.fb = p.fb[level % 3];
    // The first level that would pull surveys the lanes' frontiers: lanes
    // whose frontier degree sum is under 1/MS_SURVEY_DIV of the graph's entries are
    // pushed at that level, the others pulled (a mixed level: both phases
    // leave their finds in N and the apply pass settles every vertex).
    Mask<NW> qm, pm;  // lanes pushed, lanes pulled
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      qm.w[k] = pull ? 0u : ~0u;
      pm.w[k] = act.w[k];
    }
    const bool survey = pull && surveys < MS_SURVEY_LEVELS;
    if (survey) {
      ++surveys;
      for (int i = threadIdx.x; i < MS_MAX_LANES; i += blockDim.x) sh_lane[i] = 0;
      __syncthreads();
      ms_lane_survey<NW>(p, Fc, sh_lane);
      __syncthreads();
      if (threadIdx.x < W && sh_lane[threadIdx.x]) atomicAdd(&ctl->lane_deg[threadIdx.x], sh_lane[threadIdx.x]);
      if (!grid_sync<M_NUM>(&ctl->bar, nullptr, sh_acc, nullptr, sh_cnt, &sh_flag)) return;
      if (threadIdx.x < NW) {
        uint32_t aw = 0;  // act.w[threadIdx.x], selected so that act stays in registers
#pragma unroll
        for (int k = 0; k < NW; ++k)
          if (k == (int)threadIdx.x) aw = act.w[k];
        uint32_t q = 0;
        for (int b = 0; b < 32; ++b) {
          const int k = threadIdx.x * 32 + b;
          if (((aw >> b) & 1u) && __ldcg(&ctl->lane_deg[k]) < survey_thr) q |= 1u << b;
        }
        sh_qm[threadIdx.x] = q;
      }
      __syncthreads();
      bool anyp = false;
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        qm.w[k] = sh_qm[k];
        pm.w[k] = act.w[k] & ~qm.w[k];
        anyp |= pm.w[k] != 0;
      }
      if (!anyp) pull = false;  // every live lane is small: a push level
    }
    bool mixed = false;
    if (pull) {
#pragma unroll
      for (int k = 0; k < NW; ++k) mixed |= qm.w[k] != 0;
    }
    // A push level is sparse when the last frontier's degree sum (which
    // bounds the vertices it can touch) is at most sparse_limit: it marks the
    // vertices it touches and settles only those, after clearing, during the
    // push, the masks Fn still holds from two levels before (marked in that
    // level's frontier bitmap) and its own frontier bitmap.
    const bool sparse = SP && !pull && !mixed && (int64_t)mf_last <= p.sparse_limit;
    const uint32_t* fbc = p.fb[(level - 1) % 3];
    la.track = sparse;
    if (pull && !mixed) {
      ms_pull_rows<NW, false, COUNT, SP>(p, act, Fc, Fn, lvl4, la);
      ms_pull_hubs<NW, COUNT>(p, act, Fc, la);
    } else if (mixed) {
      if constexpr (SP) ms_push_rows_marked<NW, COUNT>(p, Fc, fbc, qm, la);
      else ms_push_rows_dense<NW, COUNT>(p, Fc, qm, la);
      ms_push_hubs<NW, COUNT>(p, Fc, qm, la);
      ms_pull_rows<NW, true, COUNT, SP>(p, pm, Fc, Fn, lvl4, la);
      ms_pull_hubs<NW, COUNT>(p, pm, Fc, la);
    } else {
      if constexpr (SP) ms_push_rows_marked<NW, COUNT>(p, Fc, fbc, qm, la);
      else ms_push_rows_dense<NW, COUNT>(p, Fc, qm, la);
      ms_push_hubs<NW, COUNT>(p, Fc, qm, la);
      // (level 1: Fn is clear from the start)
      if (sparse) ms_clear_marked<NW>(p, Fn, level > 1 ? p.fb[(level - 2) % 3] : nullptr, la.fb);
    }
    pulls += pull;
    if (!grid_sync<M_NUM>(&ctl->bar, nullptr, sh_acc, nullptr, sh_cnt, &sh_flag)) return;
    if (tid == 0) ctl->level_mid_ns[level] = globaltimer();
    // every block read the survey's sums before this barrier; the next
    // survey adds after the level's closing one
    if (survey && blockIdx.x == 0)
      for (int i = threadIdx.x; i < MS_MAX_LANES; i += blockDim.x) ctl->lane_deg[i] = 0;
    if (pull && !mixed) ms_settle_hubs<NW, SP>(p, act, Fn, lvl4, la);
    else if (sparse) ms_apply_marked<NW>(p, act, Fn, lvl4, la);
    else ms_apply<NW, SP>(p, act, Fn, lvl4, la);
    flush_level<NW, COUNT>(la, sh_acc, sh_or, alive);
    if (!grid_sync_sum<M_NUM>(cnt, &ctl->bar, sh_acc, sh_cnt)) return;
    ++phase;
    const unsigned long long nnew = sh_cnt[M_NEW];
    if (tid == 0) {
      ctl->level_new[level] = nnew;
      ctl->level_t_ns[level] = globaltimer();
      ctl->level_pull[level] = pull ? (mixed ? 2 : 1) : 0;
      if constexpr (COUNT) {
        ctl->level_rows[level] = sh_cnt[M_ROWS];
        ctl->level_sect[level] = sh_cnt[M_SECT];
      }
    }
    // a lane that found nothing this level has finished: it no longer needs anything
    {
      volatile const unsigned* va = alive;
#pragma unroll
      for (int k = 0; k < NW; ++k) act.w[k] &= va[k];
    }
    if (nnew == 0) break;
    if (level >= MS_MAX_LEVEL) {
      if (tid == 0) atomicOr(&ctl->bar.err, (unsigned)MS_ERR_DEPTH);
      break;
    }
    const unsigned long long mu = sparse ? mu_last : sh_cnt[M_MU];
    mu_last = mu;
    mf_last = sh_cnt[M_MF];
    pull = (double)sh_cnt[M_MF] > (double)mu / p.alpha;
  }
  if (tid == 0) {
    ctl->num_levels = (unsigned)level;
    ctl->pull_levels = pulls;
    ctl->t_end_ns = globaltimer();
  }
}

// 4x4 byte transpose: c[j] byte v = a[v] byte j
__device__ __forceinline__ void transpose4x4(const uint32_t a[4], uint32_t c[4]) {
  const uint32_t t0 = __byte_perm(a[0], a[1], 0x5140u), t1 = __byte_perm(a[0], a[1], 0x7362u);
  const uint32_t t2 = __byte_perm(a[2], a[3], 0x5140u), t3 = __byte_perm(a[2], a[3], 0x7362u);
  c[0] = __byte_perm(t0, t2, 0x5410u);
  c[1] = __byte_perm(t0, t2, 0x7632u);
  c[2] = __byte_perm(t1, t3, 0x5410u);
  c[3] = __byte_perm(t1, t3, 0x7632u);
}

// levels [nlv][W] (reordered) -> out[lane][orig] (nroots rows of nolv bytes).
// Four consecutive original vertices per thread: their rows' visited masks and
// the level bytes of their visited 16-lane groups (unvisited lanes read as
// 255).  Each 32-bit word of a row holds 4 lanes of one vertex; a 4x4 byte
// transpose in registers turns the 4 vertices' words into 4 words of one lane
// x 4 vertices, so every store instruction of a warp writes 128 consecutive
// bytes of one lane's output row (nolv is a multiple of 65536, so the
// 4-vertex steps never straddle the end).
constexpr int TR_BLOCK = 256;
template <int NW>
__global__ void __launch_bounds__(TR_BLOCK) ms_transpose_kernel(const uint8_t* __restrict__ L,
                                                                const uint32_t* __restrict__ V,
                                                                const uint32_t* __restrict__ reorder, int64_t nlv,
                                                                int64_t nolv, const int* nroots_dev,
                                                                uint8_t* __restrict__ out) {
  constexpr int W = 32 * NW;
  constexpr int CHUNKS = W / 16;
  const int nroots = *nroots_dev;
  for (int64_t u0 = ((int64_t)blockIdx.x * TR_BLOCK + threadIdx.x) * 4; u0 < nolv;
       u0 += (int64_t)gridDim.x * TR_BLOCK * 4) {
    const uint4 rr = __ldg(reinterpret_cast<const uint4*>(reorder + u0));
    const uint32_t r[4] = {rr.x, rr.y, rr.z, rr.w};
    uint32_t vb[4][NW];
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int k = 0; k < NW; ++k) vb[v][k] = (int64_t)r[v] < nlv ? __ldg(V + (int64_t)r[v] * NW + k) : 0u;
    // one 16-lane group at a time (keeps the registers, hence occupancy, low)
#pragma unroll 1
    for (int q = 0; q < CHUNKS; ++q) {
      uint4 x[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        uint32_t word = vb[v][0];
#pragma unroll
        for (int k = 1; k < NW; ++k) word = (q >> 1) == k ? vb[v][k] : word;
        const uint32_t bits = (word >> ((q & 1) * 16)) & 0xFFFFu;
        x[v] = make_uint4(~0u, ~0u, ~0u, ~0u);
        if (bits) {
          x[v] = __ldg(reinterpret_cast<const uint4*>(L + (int64_t)r[v] * W) + q);
          x[v].x |= ~nibble_bytes(bits & 0xFu);
          x[v].y |= ~nibble_bytes((bits >> 4) & 0xFu);
          x[v].z |= ~nibble_bytes((bits >> 8) & 0xFu);
          x[v].w |= ~nibble_bytes((bits >> 12) & 0xFu);
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int lb = 4 * (4 * q + i);  // lanes lb .. lb + 3
        if (lb >= nroots) break;
        uint32_t a[4], c[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) a[v] = i == 0 ? x[v].x : i == 1 ? x[v].y : i == 2 ? x[v].z : x[v].w;
        transpose4x4(a, c);
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (lb + j < nroots) *reinterpret_cast<uint32_t*>(out + (int64_t)(lb + j) * nolv + u0) = c[j];
      }
    }
  }
}

// a root outside the CSR range (no edges) reached only itself; its self-loop
// occurrences are its edge count
__global__ void ms_root_stats_fixup_kernel(const int64_t* roots, const int* nroots_dev, const uint32_t* reorder,
                                           int64_t nlv, const uint32_t* endp, unsigned long long* reached,
                                           unsigned long long* e2) {
  const int i = threadIdx.x;
  if (i >= *nroots_dev) return;
  const uint32_t r = reorder[roots[i]];
  if ((int64_t)r >= nlv) {
    reached[i] = 1;
    e2[i] = endp[r];
  }
}

// every root is its own level 0 (also a root outside the CSR range)
__global__ void ms_root_fixup_kernel(const int64_t* roots, const int* nroots_dev, int64_t nolv, uint8_t* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < *nroots_dev) out[(int64_t)i * nolv + roots[i]] = 0;
}

__global__ void ms_degree_kernel(const uint64_t* __restrict__ off, int64_t nlv, uint32_t* __restrict__ deg) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nlv; v += (int64_t)gridDim.x * blockDim.x)
    deg[v] = (uint32_t)(off[v + 1] - off[v]);
}


// per lane: reached vertices and the sum of endpoint occurrences (2 x nedge)
template <int NW>
__global__ void __launch_bounds__(256) ms_stats_kernel(const uint32_t* __restrict__ V,
                                                       const uint32_t* __restrict__ endp, int64_t nlv, int nroots,
                                                       unsigned long long* reached, unsigned long long* e2) {
  __shared__ unsigned long long s_r[MS_MAX_LANES], s_e[MS_MAX_LANES];
  for (int i = threadIdx.x; i < MS_MAX_LANES; i += blockDim.x) s_r[i] = s_e[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < nlv;
       base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = base + lane;
    Mask<NW> m;
    uint32_t e = 0;
    if (v < nlv) {
      m = load_mask<NW>(V + v * NW);
      e = __ldg(endp + v);
    } else {
#pragma unroll
      for (int k = 0; k < NW; ++k) m.w[k] = 0;
    }
    for (int l = 0; l < nroots; ++l) {
      const uint32_t bit = (m.w[l >> 5] >> (l & 31)) & 1u;
      const unsigned rs = __reduce_add_sync(FULL_MASK, bit);
      const unsigned es = __reduce_add_sync(FULL_MASK, bit ? e : 0u);
      if (lane == 0 && rs) {
        atomicAdd(&s_r[l], (unsigned long long)rs);
        atomicAdd(&s_e[l], (unsigned long long)es);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nroots; i += blockDim.x) {
    if (s_r[i]) atomicAdd(&reached[i], s_r[i]);
    if (s_e[i]) atomicAdd(&e2[i], s_e[i]);
  }
}

// hub list: vertices whose rows exceed `thresh`, with their chunk counts
__global__ void hub_flag_kernel(const uint64_t* __restrict__ off, int64_t nlv, uint64_t thresh, uint32_t* flags) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nlv; r += (int64_t)gridDim.x * blockDim.x)
    flags[r] = (off[r + 1] - off[r]) > thresh ? 1u : 0u;
}

__global__ void hub_compact_kernel(const uint64_t* __restrict__ off, int64_t nlv, const uint32_t* __restrict__ flags,
                                   const uint64_t* __restrict__ pos, uint64_t chunk, uint32_t* hubs,
                                   uint32_t* chunks) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nlv; r += (int64_t)gridDim.x * blockDim.x)
    if (flags[r]) {
      hubs[pos[r]] = (uint32_t)r;
      chunks[pos[r]] = (uint32_t)((off[r + 1] - off[r] + chunk - 1) / chunk);
    }
}

// chunk table: hub i's chunks [chunk0[i], chunk0[i + 1]) -> (hubs[i], k)
__global__ void hub_tab_kernel(const uint32_t* __restrict__ hubs, const uint64_t* __restrict__ chunk0, int64_t nhubs,
                               uint2* __restrict__ tab) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nhubs; i += (int64_t)gridDim.x * blockDim.x)
    for (uint64_t c = chunk0[i]; c < chunk0[i + 1]; ++c) tab[c] = make_uint2(hubs[i], (uint32_t)(c - chunk0[i]));
}

}  // namespace g500

using namespace g500;

struct g500_msbfs {
  g500_graph* g = nullptr;
  cudaStream_t stream = nullptr;
  int lane_width = 64;
  double alpha = 15.0;
  int use_graph = 1;
  int count = 0;                    // counting launches (no CUDA graph): per-level offset reads and sectors
  unsigned grid[3] = {0, 0, 0};     // co-resident blocks per lane width (NW = 1, 2, 4)

  uint32_t *V = nullptr, *F = nullptr, *N = nullptr;  // [nlv][4] words (room for 128 lanes)
  uint8_t* L = nullptr;                               // [nlv][128]
  uint8_t* out = nullptr;                             // [128][nolv]
  MsCtl* ctl = nullptr;                               // [4] one per batch
  int64_t* roots_dev = nullptr;                       // [4][128]
  int* nroots_dev = nullptr;                          // [4]
  int64_t* staging = nullptr;                         // pinned: [4][128] roots + [4] counts
  MsCtl* h_ctl = nullptr;                             // pinned [4]
  unsigned long long* stats_dev = nullptr;            // [2][128]
  unsigned long long* h_stats = nullptr;              // pinned [2][128]: reached, 2 * nedge per lane
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_done = nullptr;
  unsigned grid_full[3] = {0, 0, 0};                  // the whole device's co-resident blocks
  int want_stats = 0;                                 // root statistics enqueued with every one-launch call
  int in_flight = 0, fl_batches = 0, fl_stats = 0, stats_valid = 0;
  std::vector<int64_t> fl_roots, last_roots;
  std::chrono::steady_clock::time_point t_launch;
  cudaGraphExec_t graphs[3][4] = {};                  // [log2(W/32)][batch]
  uint32_t* deg = nullptr;                            // [nlv] row lengths
  uint2* hub_tab = nullptr;                           // pull: [nhub_chunks] (hub row, chunk index)
  int64_t nhub_chunks = 0;
  uint32_t* hub_rows = nullptr;                       // pull: the rows longer than MS_HUB_DEG
  int64_t nhub_rows = 0;
  uint2* push_tab = nullptr;                          // push: [npush_chunks]
  int64_t npush_chunks = 0;
  uint32_t* marks = nullptr;                          // [4][nwords]: three frontier bitmaps, the touched bitmap
  int64_t nwords = 0;
  int64_t sparse_limit = 0;                           // g500_msbfs_set_sparse (-1: never sparse)
  int last_nroots = 0;
  int last_batches = 0;
};

static int nw_index(int w) { return w == 32 ? 0 : (w == 64 ? 1 : 2); }

static void ms_drop_graphs(g500_msbfs* m) {
  for (auto& row : m->graphs)
    for (auto& e : row)
      if (e) {
        cudaGraphExecDestroy(e);
        e = nullptr;
      }
}

static int ms_free(g500_msbfs* m) {
  if (!m) return G500_OK;
  cudaSetDevice(m->g->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  ms_drop_graphs(m);
  dev_free(m->V);
  dev_free(m->F);
  dev_free(m->N);
  dev_free(m->L);
  dev_free(m->out);
  dev_free(m->ctl);
  dev_free(m->roots_dev);
  dev_free(m->nroots_dev);
  dev_free(m->stats_dev);
  dev_free(m->deg);
  dev_free(m->hub_tab);
  dev_free(m->hub_rows);
  dev_free(m->push_tab);
  dev_free(m->marks);
  if (m->staging) cudaFreeHost(m->staging);
  if (m->h_ctl) cudaFreeHost(m->h_ctl);
  if (m->h_stats) cudaFreeHost(m->h_stats);
  if (m->ev0) cudaEventDestroy(m->ev0);
  if (m->ev1) cudaEventDestroy(m->ev1);
  if (m->ev_done) cudaEventDestroy(m->ev_done);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return G500_OK;
}

template <int NW>
static const void* ms_kernel_ptr() { return (const void*)msbfs_kernel<NW, false, true>; }

// Chunk table of the rows longer than `thresh`, `chunk` edges per chunk, so
// that warps can share a hub's row.
static int ms_build_hubs(g500_msbfs* m, uint64_t thresh, uint64_t chunk, uint2** tab, int64_t* ntab,
                         uint32_t** rows_out = nullptr, int64_t* nrows_out = nullptr) {
  g500_graph* g = m->g;
  cudaStream_t s = m->stream;
  const int64_t nlv = g->nlv;
  if (nlv == 0) return G500_OK;
  uint32_t* flags = nullptr;
  uint64_t* pos = nullptr;
  uint32_t* hubs = nullptr;
  uint32_t* chunks = nullptr;
  uint64_t* chunk0 = nullptr;
  void* tmp = nullptr;
  int st = dev_alloc_n(&flags, nlv, "hub flags");
  if (st == G500_OK) st = dev_alloc_n(&pos, nlv + 1, "hub positions");
  if (st == G500_OK) st = dev_alloc(&tmp, scan_tmp_bytes(nlv + 1), "scan scratch");
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(nlv, 256), (int64_t)num_sms() * 8);
  if (st == G500_OK) {
    hub_flag_kernel<<<grid, 256, 0, s>>>(g->d_offsets, nlv, thresh, flags);
    st = exclusive_scan_u32(flags, pos, nlv, tmp, s);
  }
  uint64_t H = 0;
  if (st == G500_OK) {
    cudaError_t e = cudaMemcpyAsync(&H, pos + nlv, sizeof(H), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_error(e, "hub count", __FILE__, __LINE__);
  }
  if (st == G500_OK) st = dev_alloc_n(&hubs, std::max<int64_t>((int64_t)H, 1), "hub list");
  if (st == G500_OK) st = dev_alloc_n(&chunks, std::max<int64_t>((int64_t)H, 1), "hub chunks");
  if (st == G500_OK) st = dev_alloc_n(&chunk0, (int64_t)H + 1, "hub chunk prefix");
  if (st == G500_OK && H > 0) {
    hub_compact_kernel<<<grid, 256, 0, s>>>(g->d_offsets, nlv, flags, pos, chunk, hubs, chunks);
    st = exclusive_scan_u32(chunks, chunk0, (int64_t)H, tmp, s);
    uint64_t tc = 0;
    if (st == G500_OK) {
      cudaError_t e = cudaMemcpyAsync(&tc, chunk0 + H, sizeof(tc), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) st = cuda_error(e, "hub chunks", __FILE__, __LINE__);
    }
    if (st == G500_OK) st = dev_alloc_n(tab, std::max<int64_t>((int64_t)tc, 1), "hub chunk table");
    if (st == G500_OK) {
      const unsigned hg = (unsigned)std::min<int64_t>(ceil_div((int64_t)H, 256), 1024);
      hub_tab_kernel<<<hg, 256, 0, s>>>(hubs, chunk0, (int64_t)H, *tab);
      cudaError_t e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) st = cuda_error(e, "hub chunk table", __FILE__, __LINE__);
      *ntab = (int64_t)tc;
    }
  }
  dev_free(flags);
  if (rows_out && st == G500_OK) {
    *rows_out = hubs;  // the handle keeps the hub rows
    *nrows_out = (int64_t)H;
  } else {
    dev_free(hubs);
  }
  dev_free(pos);
  dev_free(chunks);
  dev_free(chunk0);
  dev_free(tmp);
  return st;
}

// Enqueue one batch: roots upload, control reset, the persistent kernel, the
// transpose into out + batch * W * nolv, and the root fix-up.
static int ms_enqueue_batch(g500_msbfs* m, int b, cudaStream_t s) {
  g500_graph* g = m->g;
  const int W = m->lane_width;
  const int ni = nw_index(W);
  G500_CUDA(cudaMemcpyAsync(m->roots_dev + b * MS_MAX_LANES, m->staging + b * MS_MAX_LANES,
                            sizeof(int64_t) * MS_MAX_LANES, cudaMemcpyHostToDevice, s));
  G500_CUDA(cudaMemcpyAsync(m->nroots_dev + b, reinterpret_cast<int*>(m->staging + 4 * MS_MAX_LANES) + b,
                            sizeof(int), cudaMemcpyHostToDevice, s));
  G500_CUDA(cudaMemsetAsync(m->ctl + b, 0, sizeof(MsCtl), s));
  MsParams p;
  p.off = g->d_offsets;
  p.deg = m->deg;
  p.col = g->d_cols;
  p.reorder = g->d_reorder;
  p.V = m->V;
  p.F[0] = m->F;
  p.F[1] = m->F + std::max<int64_t>(g->nlv, 1) * 4;
  p.hubs = m->hub_rows;
  p.nhubs = m->nhub_rows;
  p.N = m->N;
  p.L = m->L;
  p.roots = m->roots_dev + b * MS_MAX_LANES;
  p.nroots_dev = m->nroots_dev + b;
  p.nlv = g->nlv;
  p.hub_tab = m->hub_tab;
  p.nhub_chunks = m->nhub_chunks;
  p.push_tab = m->push_tab;
  p.npush_chunks = m->npush_chunks;
  for (int i = 0; i < 3; ++i) p.fb[i] = m->marks + i * m->nwords;
  p.touched = m->marks + 3 * m->nwords;
  p.nwords = m->nwords;
  p.sparse_limit = m->sparse_limit;
  p.alpha = m->alpha;
  p.ctl = m->ctl + b;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(m->grid[ni]);
  cfg.blockDim = dim3(MS_THREADS);
  cfg.stream = s;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeCooperative;
  attr.val.cooperative = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  const bool sp = m->sparse_limit >= 0;
  if (m->count) {  // the counting variant has the timed kernel's grid (same launch bounds)
    if (W == 32) G500_CUDA(cudaLaunchKernelEx(&cfg, sp ? msbfs_kernel<1, true, true> : msbfs_kernel<1, true, false>, p));
    else if (W == 64) G500_CUDA(cudaLaunchKernelEx(&cfg, sp ? msbfs_kernel<2, true, true> : msbfs_kernel<2, true, false>, p));
    else G500_CUDA(cudaLaunchKernelEx(&cfg, sp ? msbfs_kernel<4, true, true> : msbfs_kernel<4, true, false>, p));
  } else {
    if (W == 32) G500_CUDA(cudaLaunchKernelEx(&cfg, sp ? msbfs_kernel<1, false, true> : msbfs_kernel<1, false, false>, p));
    else if (W == 64) G500_CUDA(cudaLaunchKernelEx(&cfg, sp ? msbfs_kernel<2, false, true> : msbfs_kernel<2, false, false>, p));
    else G500_CUDA(cudaLaunchKernelEx(&cfg, sp ? msbfs_kernel<4, false, true> : msbfs_kernel<4, false, false>, p));
  }
  uint8_t* out = m->out + (int64_t)b * W * g->nolv;
  const unsigned tg = (unsigned)std::min<int64_t>(ceil_div(g->nolv, 4 * TR_BLOCK), (int64_t)num_sms() * 8);
  if (W == 32) ms_transpose_kernel<1><<<tg, TR_BLOCK, 0, s>>>(m->L, m->V, g->d_reorder, g->nlv, g->nolv, m->nroots_dev + b, out);
  else if (W == 64) ms_transpose_kernel<2><<<tg, TR_BLOCK, 0, s>>>(m->L, m->V, g->d_reorder, g->nlv, g->nolv, m->nroots_dev + b, out);
  else ms_transpose_kernel<4><<<tg, TR_BLOCK, 0, s>>>(m->L, m->V, g->d_reorder, g->nlv, g->nolv, m->nroots_dev + b, out);
  ms_root_fixup_kernel<<<1, MS_MAX_LANES, 0, s>>>(m->roots_dev + b * MS_MAX_LANES, m->nroots_dev + b, g->nolv, out);
  G500_CUDA(cudaGetLastError());
  return G500_OK;
}

extern "C" int g500_msbfs_create(g500_graph* g, g500_msbfs** out) {
  if (!g || !out) return set_error(G500_E_INVAL, "null argument");
  G500_CUDA(cudaSetDevice(g->device));
  g500_msbfs* m = new g500_msbfs();
  m->g = g;
  int st = G500_OK;
  auto chk = [&](cudaError_t e, const char* what) {
    if (st == G500_OK && e != cudaSuccess) st = cuda_error(e, what, __FILE__, __LINE__);
  };
  chk(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  const int64_t nlv = std::max<int64_t>(g->nlv, 1);
  if (st == G500_OK) st = dev_alloc_n(&m->V, nlv * 4, "msbfs visited masks");
  if (st == G500_OK) st = dev_alloc_n(&m->F, 2 * nlv * 4, "msbfs frontier masks");
  if (st == G500_OK) st = dev_alloc_n(&m->N, nlv * 4, "msbfs next masks");
  if (st == G500_OK) st = dev_alloc_n(&m->L, nlv * MS_MAX_LANES, "msbfs levels");
  if (st == G500_OK) st = dev_alloc_n(&m->deg, nlv, "msbfs row lengths");
  // sparse levels: frontier and touched bitmaps; from 2^22 vertices with
  // edges, a push level is sparse up to a last-frontier degree sum of nlv / 8
  // (on smaller graphs a pass over every vertex costs less than the sparse
  // level's extra steps)
  m->nwords = (nlv + 31) / 32;
  m->sparse_limit = nlv >= (int64_t(1) << 22) ? nlv / 8 : -1;
  if (st == G500_OK) st = dev_alloc_n(&m->marks, 4 * m->nwords, "msbfs frontier and touched bitmaps");
  if (st == G500_OK && g->nlv > 0) {
    const unsigned dgrid = (unsigned)std::min<int64_t>(ceil_div(g->nlv, 256), (int64_t)num_sms() * 8);
    ms_degree_kernel<<<dgrid, 256, 0, m->stream>>>(g->d_offsets, g->nlv, m->deg);
    chk(cudaGetLastError(), "row lengths");
  }
  if (st == G500_OK) st = dev_alloc_n(&m->out, (int64_t)MS_MAX_LANES * g->nolv, "msbfs output levels");
  if (st == G500_OK) st = dev_alloc_n(&m->ctl, 4, "msbfs control");
  if (st == G500_OK) st = dev_alloc_n(&m->roots_dev, 4 * MS_MAX_LANES, "msbfs roots");
  if (st == G500_OK) st = dev_alloc_n(&m->nroots_dev, 4, "msbfs root counts");
  if (st == G500_OK) st = dev_alloc_n(&m->stats_dev, 2 * MS_MAX_LANES, "msbfs stats");
  if (st == G500_OK)
    chk(cudaHostAlloc(&m->staging, sizeof(int64_t) * (4 * MS_MAX_LANES + 4), cudaHostAllocDefault), "cudaHostAlloc");
  if (st == G500_OK) chk(cudaHostAlloc(&m->h_ctl, sizeof(MsCtl) * 4, cudaHostAllocDefault), "cudaHostAlloc");
  chk(cudaEventCreate(&m->ev0), "cudaEventCreate");
  chk(cudaEventCreate(&m->ev1), "cudaEventCreate");
  chk(cudaEventCreateWithFlags(&m->ev_done, cudaEventDisableTiming), "cudaEventCreate");
  if (st == G500_OK)
    chk(cudaHostAlloc(&m->h_stats, sizeof(unsigned long long) * 2 * MS_MAX_LANES, cudaHostAllocDefault),
        "cudaHostAlloc");
  if (st == G500_OK)
    st = ms_build_hubs(m, MS_HUB_DEG, MS_HUB_CHUNK, &m->hub_tab, &m->nhub_chunks, &m->hub_rows, &m->nhub_rows);
  if (st == G500_OK) st = ms_build_hubs(m, MS_PUSH_HUB_DEG, MS_PUSH_CHUNK, &m->push_tab, &m->npush_chunks);
  const void* kernels[3] = {ms_kernel_ptr<1>(), ms_kernel_ptr<2>(), ms_kernel_ptr<4>()};
  for (int i = 0; i < 3 && st == G500_OK; ++i) {
    int per_sm = 0;
    chk(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernels[i], MS_THREADS, 0), "occupancy");
    if (st == G500_OK && per_sm <= 0) st = set_error(G500_E_DEVICE, "multi-source kernel cannot be co-scheduled");
    m->grid[i] = m->grid_full[i] = (unsigned)(num_sms() * std::max(per_sm, 1));
  }
  if (st != G500_OK) {
    ms_free(m);
    return st;
  }
  *out = m;
  return G500_OK;
}

extern "C" int g500_msbfs_set_params(g500_msbfs* m, int lane_width, double alpha, int use_cuda_graph) {
  if (!m) return set_error(G500_E_INVAL, "null handle");
  if (lane_width != 32 && lane_width != 64 && lane_width != 128)
    return set_error(G500_E_INVAL, "lane width %d not 32, 64 or 128", lane_width);
  if (!(alpha > 0)) return set_error(G500_E_INVAL, "alpha must be > 0");
  if (alpha != m->alpha) ms_drop_graphs(m);  // graphs are kept per lane width; alpha is captured in them
  m->lane_width = lane_width;
  m->alpha = alpha;
  m->use_graph = use_cuda_graph ? 1 : 0;
  return G500_OK;
}

// Per-lane reached / 2*nedge of the last launch into h_stats (enqueued on s).
static int ms_enqueue_stats(g500_msbfs* m, int nroots, cudaStream_t s) {
  g500_graph* g = m->g;
  G500_CUDA(cudaMemsetAsync(m->stats_dev, 0, sizeof(unsigned long long) * 2 * MS_MAX_LANES, s));
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(std::max<int64_t>(g->nlv, 1), 256), num_sms() * 8);
  const int W = m->lane_width;
  unsigned long long* r = m->stats_dev;
  unsigned long long* e = m->stats_dev + MS_MAX_LANES;
  if (g->nlv > 0) {
    if (W == 32) ms_stats_kernel<1><<<grid, 256, 0, s>>>(m->V, g->d_endp, g->nlv, nroots, r, e);
    else if (W == 64) ms_stats_kernel<2><<<grid, 256, 0, s>>>(m->V, g->d_endp, g->nlv, nroots, r, e);
    else ms_stats_kernel<4><<<grid, 256, 0, s>>>(m->V, g->d_endp, g->nlv, nroots, r, e);
  }
  ms_root_stats_fixup_kernel<<<1, MS_MAX_LANES, 0, s>>>(m->roots_dev, m->nroots_dev, g->d_reorder, g->nlv, g->d_endp,
                                                        r, e);
  G500_CUDA(cudaGetLastError());
  G500_CUDA(cudaMemcpyAsync(m->h_stats, m->stats_dev, sizeof(unsigned long long) * 2 * MS_MAX_LANES,
                            cudaMemcpyDeviceToHost, s));
  return G500_OK;
}

// Enqueue a whole call (every launch, the optional level copy, the control
// blocks' copy back, the optional root statistics) and record ev_done.
static int ms_launch(g500_msbfs* m, const int64_t* roots, int nroots, uint8_t* levels, int levels_on_device,
                     uint8_t* const* root_dsts = nullptr) {
  if (!m || !roots) return set_error(G500_E_INVAL, "null argument");
  if (m->in_flight) return set_error(G500_E_STATE, "the previous launch has not been waited for");
  g500_graph* g = m->g;
  if (nroots < 1 || nroots > MS_MAX_LANES)
    return set_error(G500_E_INVAL, "%d roots; 1..%d per call", nroots, MS_MAX_LANES);
  for (int i = 0; i < nroots; ++i)
    if (roots[i] < 0 || roots[i] >= g->nolv)
      return set_error(G500_E_INVAL, "root %lld outside [0, %lld)", (long long)roots[i], (long long)g->nolv);
  G500_CUDA(cudaSetDevice(g->device));
  m->t_launch = std::chrono::steady_clock::now();
  const int W = m->lane_width;
  const int ni = nw_index(W);
  const int batches = (nroots + W - 1) / W;
  int* counts = reinterpret_cast<int*>(m->staging + 4 * MS_MAX_LANES);
  for (int b = 0; b < 4; ++b) {
    const int n = b < batches ? std::min(W, nroots - b * W) : 0;
    counts[b] = n;
    for (int i = 0; i < MS_MAX_LANES; ++i) m->staging[b * MS_MAX_LANES + i] = i < n ? roots[b * W + i] : 0;
  }
  cudaStream_t s = m->stream;
  G500_CUDA(cudaEventRecord(m->ev0, s));
  for (int b = 0; b < batches; ++b) {
    if (m->use_graph && !m->count) {
      if (!m->graphs[ni][b]) {
        cudaGraph_t graph = nullptr;
        G500_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int st = ms_enqueue_batch(m, b, s);
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (st != G500_OK) {
          if (graph) cudaGraphDestroy(graph);
          return st;
        }
        if (e != cudaSuccess) return cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        e = cudaGraphInstantiate(&m->graphs[ni][b], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
          m->graphs[ni][b] = nullptr;
          return cuda_error(e, "cudaGraphInstantiate", __FILE__, __LINE__);
        }
      }
      G500_CUDA(cudaGraphLaunch(m->graphs[ni][b], s));
    } else {
      G500_TRY(ms_enqueue_batch(m, b, s));
    }
  }
  G500_CUDA(cudaEventRecord(m->ev1, s));
  if (levels) {
    G500_CUDA(cudaMemcpyAsync(levels, m->out, (size_t)nroots * g->nolv,
                              levels_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  }
  if (root_dsts)
    for (int i = 0; i < nroots; ++i)
      if (root_dsts[i])
        G500_CUDA(cudaMemcpyAsync(root_dsts[i], m->out + (int64_t)i * g->nolv, (size_t)g->nolv, cudaMemcpyDefault, s));
  G500_CUDA(cudaMemcpyAsync(m->h_ctl, m->ctl, sizeof(MsCtl) * batches, cudaMemcpyDeviceToHost, s));
  m->fl_stats = m->want_stats && batches == 1;
  if (m->fl_stats) G500_TRY(ms_enqueue_stats(m, nroots, s));
  G500_CUDA(cudaEventRecord(m->ev_done, s));
  m->fl_roots.assign(roots, roots + nroots);
  m->fl_batches = batches;
  m->in_flight = 1;
  return G500_OK;
}

// Wait for the launch in flight and report it.
static int ms_complete(g500_msbfs* m, g500_msbfs_stats* stats) {
  if (!m->in_flight) return set_error(G500_E_STATE, "no launch in flight");
  G500_CUDA(cudaSetDevice(m->g->device));
  m->in_flight = 0;
  cudaError_t ce = cudaEventSynchronize(m->ev_done);
  if (ce != cudaSuccess) return cuda_error(ce, "cudaEventSynchronize", __FILE__, __LINE__);
  const int batches = m->fl_batches;
  m->last_roots = m->fl_roots;
  m->last_nroots = (int)m->fl_roots.size();
  m->last_batches = batches;
  m->stats_valid = m->fl_stats;
  unsigned err = 0;
  for (int b = 0; b < batches; ++b) err |= m->h_ctl[b].bar.err;
  if (err & GRID_ERR_TIMEOUT) return set_error(G500_E_TIMEOUT, "grid barrier wait gave up (bounded spin)");
  if (err & MS_ERR_DEPTH) return set_error(G500_E_RANGE, "a BFS is deeper than %d levels (uint8 levels)", MS_MAX_LEVEL);
  if (stats) {
    float ms = 0;
    G500_CUDA(cudaEventElapsedTime(&ms, m->ev0, m->ev1));
    memset(stats, 0, sizeof(*stats));
    stats->device_ms = ms;
    stats->host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - m->t_launch).count();
    stats->lane_width = m->lane_width;
    stats->batches = batches;
    for (int b = 0; b < batches; ++b) {
      stats->num_levels = std::max<int32_t>(stats->num_levels, (int32_t)m->h_ctl[b].num_levels);
      stats->pull_levels += (int32_t)m->h_ctl[b].pull_levels;
      const MsCtl& c = m->h_ctl[b];
      if (c.t_init_ns >= c.t0_ns) stats->init_ms += (double)(c.t_init_ns - c.t0_ns) * 1e-6;
      if (c.t_end_ns >= c.t_init_ns) stats->search_ms += (double)(c.t_end_ns - c.t_init_ns) * 1e-6;
    }
    stats->kernel_launches = 3 * batches + (m->fl_stats ? 2 : 0);
  }
  return G500_OK;
}

extern "C" int g500_msbfs_run(g500_msbfs* m, const int64_t* roots, int nroots, uint8_t* levels, int levels_on_device,
                              g500_msbfs_stats* stats) {
  G500_TRY(ms_launch(m, roots, nroots, levels, levels_on_device));
  return ms_complete(m, stats);
}

extern "C" int g500_msbfs_launch(g500_msbfs* m, const int64_t* roots, int nroots) {
  return ms_launch(m, roots, nroots, nullptr, 0);
}

namespace g500 {
int msbfs_launch_to(g500_msbfs* m, const int64_t* roots, int nroots, uint8_t* const* root_dsts) {
  return ms_launch(m, roots, nroots, nullptr, 0, root_dsts);
}
}  // namespace g500

extern "C" int g500_msbfs_poll(g500_msbfs* m, int* done) {
  if (!m || !done) return set_error(G500_E_INVAL, "null argument");
  if (!m->in_flight) return set_error(G500_E_STATE, "no launch in flight");
  const cudaError_t e = cudaEventQuery(m->ev_done);
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

extern "C" int g500_msbfs_wait(g500_msbfs* m, g500_msbfs_stats* stats) {
  if (!m) return set_error(G500_E_INVAL, "null handle");
  return ms_complete(m, stats);
}

extern "C" int g500_msbfs_set_root_stats(g500_msbfs* m, int on) {
  if (!m) return set_error(G500_E_INVAL, "null handle");
  m->want_stats = on ? 1 : 0;
  return G500_OK;
}

extern "C" int g500_msbfs_set_grid(g500_msbfs* m, int blocks) {
  if (!m) return set_error(G500_E_INVAL, "null handle");
  if (blocks < 0) return set_error(G500_E_INVAL, "negative block count");
  if (m->in_flight) return set_error(G500_E_STATE, "a launch is in flight");
  for (int i = 0; i < 3; ++i) {
    const unsigned want = blocks == 0 ? m->grid_full[i] : std::min<unsigned>((unsigned)blocks, m->grid_full[i]);
    if (want != m->grid[i]) {
      ms_drop_graphs(m);
      m->grid[i] = want;
    }
  }
  return G500_OK;
}

extern "C" int g500_msbfs_set_sparse(g500_msbfs* m, int on, int64_t limit) {
  if (!m) return set_error(G500_E_INVAL, "null handle");
  if (limit < 0) return set_error(G500_E_INVAL, "negative degree-sum limit");
  if (m->in_flight) return set_error(G500_E_STATE, "a launch is in flight");
  const int64_t want = !on ? -1 : (limit == 0 ? std::max<int64_t>(std::max<int64_t>(m->g->nlv, 1) / 8, 1) : limit);
  if (want != m->sparse_limit) {
    ms_drop_graphs(m);  // the captured launches carry the limit
    m->sparse_limit = want;
  }
  return G500_OK;
}

extern "C" int g500_msbfs_get_grid(const g500_msbfs* m, int lane_width, int* blocks, int* max_blocks) {
  if (!m) return set_error(G500_E_INVAL, "null handle");
  if (lane_width != 32 && lane_width != 64 && lane_width != 128)
    return set_error(G500_E_INVAL, "lane width %d not 32, 64 or 128", lane_width);
  if (blocks) *blocks = (int)m->grid[nw_index(lane_width)];
  if (max_blocks) *max_blocks = (int)m->grid_full[nw_index(lane_width)];
  return G500_OK;
}

extern "C" int g500_msbfs_workspace_bytes(const g500_graph* g, uint64_t* bytes) {
  if (!g || !bytes) return set_error(G500_E_INVAL, "null argument");
  const uint64_t nlv = (uint64_t)std::max<int64_t>(g->nlv, 1);
  // V, F, N (4 words each), L (128 bytes), row lengths, output rows, the
  // sparse-level bitmaps (4 bits), with room for the hub tables and control
  // blocks
  *bytes = nlv * (4 * 16 + MS_MAX_LANES + 4) + (uint64_t)MS_MAX_LANES * (uint64_t)g->nolv + (16ull << 20) +
           (uint64_t)g->nge / 64 + (nlv + 31) / 32 * 16;
  return G500_OK;
}

extern "C" int g500_msbfs_root_stats(g500_msbfs* m, int64_t* reached, int64_t* nedge) {
  if (!m) return set_error(G500_E_INVAL, "null handle");
  if (m->in_flight) return set_error(G500_E_STATE, "a launch is in flight");
  if (m->last_nroots == 0) return set_error(G500_E_STATE, "no run yet");
  if (m->last_batches != 1)
    return set_error(G500_E_STATE, "root statistics need the last run to fit one launch (roots <= lane width)");
  G500_CUDA(cudaSetDevice(m->g->device));
  const int n = m->last_nroots;
  if (!m->stats_valid) {
    G500_TRY(ms_enqueue_stats(m, n, m->stream));
    G500_CUDA(cudaStreamSynchronize(m->stream));
    m->stats_valid = 1;
  }
  for (int i = 0; i < n; ++i) {
    if (reached) reached[i] = (int64_t)m->h_stats[i];
    if (nedge) nedge[i] = (int64_t)(m->h_stats[MS_MAX_LANES + i] / 2);
  }
  return G500_OK;
}

extern "C" int g500_msbfs_device_levels(const g500_msbfs* m, const uint8_t** dev_levels) {
  if (!m || !dev_levels) return set_error(G500_E_INVAL, "null argument");
  *dev_levels = m->out;
  return G500_OK;
}

extern "C" int g500_msbfs_level_info(const g500_msbfs* m, int batch, g500_msbfs_level* out, int max_levels,
                                     int* num_levels) {
  if (!m || !num_levels) return set_error(G500_E_INVAL, "null argument");
  if (m->last_nroots == 0) return set_error(G500_E_STATE, "no run yet");
  if (batch < 0 || batch >= m->last_batches)
    return set_error(G500_E_INVAL, "launch %d outside [0, %d)", batch, m->last_batches);
  const MsCtl& c = m->h_ctl[batch];
  const int n = (int)std::min<unsigned>(c.num_levels, (unsigned)MS_MAX_LEVEL);
  *num_levels = n;
  for (int l = 1; l <= n && l <= max_levels; ++l) {
    g500_msbfs_level& r = out[l - 1];
    r.level = l;
    r.pull = c.level_pull[l];
    r.discovered = (int64_t)c.level_new[l];
    const unsigned long long prev = l == 1 ? c.t_init_ns : c.level_t_ns[l - 1];
    r.device_ms = c.level_t_ns[l] >= prev ? (double)(c.level_t_ns[l] - prev) * 1e-6 : 0.0;
    r.expand_ms = c.level_mid_ns[l] >= prev ? (double)(c.level_mid_ns[l] - prev) * 1e-6 : 0.0;
    r.rows_read = m->count ? (int64_t)c.level_rows[l] : -1;
    r.sectors = m->count ? (int64_t)c.level_sect[l] : -1;
  }
  return G500_OK;
}

extern "C" int g500_msbfs_set_count(g500_msbfs* m, int on) {
  if (!m) return set_error(G500_E_INVAL, "null argument");
  if (m->in_flight) return set_error(G500_E_STATE, "a launch is in flight");
  m->count = on ? 1 : 0;
  return G500_OK;
}

extern "C" int g500_msbfs_autotune(g500_msbfs* m, const int64_t* roots, int nroots, int reps,
                                   g500_msbfs_tune* out) {
  if (!m || !roots || nroots < 1) return set_error(G500_E_INVAL, "bad argument");
  if (reps < 1) reps = 1;
  static const int widths[] = {32, 64, 128};
  static const double alphas[] = {2.0, 6.0, 15.0, 50.0, 200.0};
  const int use_graph = m->use_graph;
  double best = 1e300;
  int bw = 64, tried = 0;
  double ba = 15.0;
  for (int w : widths) {
    for (double a : alphas) {
      G500_TRY(g500_msbfs_set_params(m, w, a, use_graph));
      double t = 1e300;
      for (int k = 0; k < reps; ++k) {
        g500_msbfs_stats st;
        G500_TRY(g500_msbfs_run(m, roots, nroots, nullptr, 0, &st));
        t = std::min(t, st.device_ms);
      }
      ++tried;
      if (t < best) {
        best = t;
        bw = w;
        ba = a;
      }
    }
  }
  G500_TRY(g500_msbfs_set_params(m, bw, ba, use_graph));
  if (out) {
    out->lane_width = bw;
    out->configs_tried = tried;
    out->alpha = ba;
    out->best_ms = best;
  }
  return G500_OK;
}

extern "C" int g500_msbfs_destroy(g500_msbfs* m) { return ms_free(m); }
