// Device helpers shared by the persistent BFS kernels: warp scans, lane
// selection, block-level counter accumulation and a bounded grid barrier for
// cooperative launches.
#pragma once

#include "g500_internal.cuh"

namespace g500 {

constexpr unsigned long long SPIN_LIMIT = 1ull << 25;  // ~ seconds of polls with __nanosleep(32)

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(FULL_MASK, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long x) {
#pragma unroll
  for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(FULL_MASK, x, o);
  return x;
}

// last lane whose exclusive prefix is <= k (prefixes are non-decreasing over lanes)
__device__ __forceinline__ int owner_lane(uint32_t excl, uint32_t k) {
  int o = 0;
#pragma unroll
  for (int step = 16; step; step >>= 1) {
    const uint32_t ex = __shfl_sync(FULL_MASK, excl, o + step);
    if (ex <= k) o += step;
  }
  return o;
}



__device__ __forceinline__ int64_t gwarp_id() { return ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int64_t gwarp_count() { return ((int64_t)gridDim.x * blockDim.x) >> 5; }

// position of the r-th (0-based) set bit of m (m has more than r set bits)
__device__ __forceinline__ uint32_t select_bit(uint32_t m, uint32_t r) {
  uint32_t pos = 0;
#pragma unroll
  for (int w = 16; w; w >>= 1) {
    const uint32_t lo = __popc(m & ((1u << w) - 1u));
    if (r >= lo) {
      r -= lo;
      m >>= w;
      pos += w;
    } else {
      m &= (1u << w) - 1u;
    }
  }
  return pos;
}

// Add a warp's value to the block accumulator of counter i (flushed to the
// level's global slot once per block at the next grid barrier).
__device__ __forceinline__ void block_add(unsigned long long* sh_acc, int i, unsigned long long v) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(&sh_acc[i], v);
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}


// Grid-wide barrier for a cooperative launch.  The block's accumulated
// counters are first added to flush_slot (one global atomic per non-zero
// counter per block).  Thread 0 then arrives on a counter with acquire-release
// semantics (the block's writes, ordered before it by __syncthreads, are
// released with it).  The counter only grows during a launch (it starts at
// zero): barrier k is complete once it reaches (k + 1) * gridDim.x, a target
// each block computes from the value its own arrival returned, so the last
// arrival has nothing more to publish.  The others poll the counter and take
// an acquire fence once it reached the target.  Polls are bounded; on
// timeout (or an error raised elsewhere, checked every 16 polls) the barrier
// reports failure and the caller returns.  On success thread 0 copies
// read_slot into sh_cnt for the block's next decision.
template <int NC>
__device__ bool grid_sync(GridBarrier* bar, unsigned long long* flush_slot, unsigned long long* sh_acc,
                          const unsigned long long* read_slot, unsigned long long* sh_cnt, unsigned* sh_flag,
                          unsigned long long spin_limit = SPIN_LIMIT) {
  __syncthreads();
  if (threadIdx.x < NC) {
    const unsigned long long v = sh_acc[threadIdx.x];
    if (flush_slot && v) atomicAdd(&flush_slot[threadIdx.x], v);
    sh_acc[threadIdx.x] = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* err = &bar->err;
    volatile unsigned* count = &bar->count;
    bool ok = true;
    const unsigned old = atom_add_acq_rel_gpu(&bar->count, 1u);
    const unsigned target = (old / gridDim.x + 1u) * gridDim.x;
    if (old + 1u != target) {
      // relaxed polls (an acquire per poll would invalidate L1 under the
      // other blocks of the SM), one acquire fence once the target is reached
      unsigned long long spins = 0;
      while ((int)(*count - target) < 0) {
        ++spins;
        if ((spins & 15) == 0 && *err) {
          ok = false;
          break;
        }
        if (spins > spin_limit) {
          atomicOr(&bar->err, (unsigned)GRID_ERR_TIMEOUT);
          ok = false;
          break;
        }
        __nanosleep(32);
      }
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
    }
    if (*err) ok = false;
    *sh_flag = ok ? 1u : 0u;
    if (ok && read_slot) {
      volatile const unsigned long long* vs = read_slot;
      for (int i = 0; i < NC; ++i) sh_cnt[i] = vs[i];
    }
  }
  __syncthreads();
  return *sh_flag != 0;
}

// Grid-wide barrier that also sums NC block counters, for a cooperative
// launch of fewer than 65536 blocks.  The counters ride on the arrivals:
// thread i < NC of every block adds (sh_acc[i] << 16) | 1 to slot[i] with
// release semantics (fire and forget), then polls slot[i] until its low 16
// bits count every block; the high 48 bits are then the grid's sum, copied to
// sh_cnt[i].  One reduction per counter instead of a reduction, an arrival
// and a read-back in turn: 2.1 us per barrier on 296 blocks of a B200 against
// 3.4 us for grid_sync with counters.  The NC words of slot must be zero
// before the first block arrives and stay untouched until every block has
// passed (the kernels rotate three slots and clear the next one a phase
// ahead).  Polls are bounded like grid_sync's; on timeout or an error raised
// elsewhere while a block waits, every block returns false.  An error raised
// before a barrier that still completes is not reported by it (that would
// cost one more round trip per barrier): the kernels decide to stop from the
// sums themselves (queue overflow, depth), and a block that gives up returns
// before arriving, so that the others time out or see the flag in their polls.
template <int NC>
__device__ bool grid_sync_sum(unsigned long long* slot, GridBarrier* bar, unsigned long long* sh_acc,
                              unsigned long long* sh_cnt, unsigned long long spin_limit = SPIN_LIMIT) {
  __syncthreads();
  bool fail = false;
  if (threadIdx.x < NC) {
    unsigned long long* w = slot + threadIdx.x;
    const unsigned long long v = (sh_acc[threadIdx.x] << 16) | 1ull;
    sh_acc[threadIdx.x] = 0;
    asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(w), "l"(v) : "memory");
    volatile const unsigned long long* vw = w;
    volatile const unsigned* err = &bar->err;
    unsigned long long x, spins = 0;
    while (((x = *vw) & 0xFFFFull) != (unsigned long long)gridDim.x) {
      ++spins;
      if ((spins & 15) == 0 && *err) {
        fail = true;
        break;
      }
      if (spins > spin_limit) {
        atomicOr(&bar->err, (unsigned)GRID_ERR_TIMEOUT);
        fail = true;
        break;
      }
      __nanosleep(32);
    }
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
    sh_cnt[threadIdx.x] = x >> 16;
  }
  return !__syncthreads_or(fail);
}

}  // namespace g500
