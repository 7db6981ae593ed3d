// Device primitives used by graph construction: error plumbing, allocation,
// an exclusive prefix sum (the reference's prefix_sum role,
// graph_constructor.hpp:404-408 and :486-491) and a stable LSD radix sort
// (the role of sort2 / std::sort in graph_constructor.hpp:318-322, :1376-1412).
#include "g500_internal.cuh"

#include <algorithm>
#include <mutex>

namespace g500 {

static thread_local std::string tl_error;

const char* last_error_text() { return tl_error.c_str(); }

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  tl_error = buf;
  return code;
}

int cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  int code = (e == cudaErrorMemoryAllocation) ? G500_E_NOMEM : G500_E_DEVICE;
  return set_error(code, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}

int num_sms() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  return n;
}

int dev_alloc(void** p, size_t bytes, const char* what) {
  *p = nullptr;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return set_error(e == cudaErrorMemoryAllocation ? G500_E_NOMEM : G500_E_DEVICE,
                     "cudaMalloc(%zu bytes) for %s failed: %s", bytes, what, cudaGetErrorString(e));
  }
  return G500_OK;
}

void dev_free(void* p) {
  if (p) cudaFree(p);
}

// ---------------------------------------------------------------------------
// exclusive scan
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <typename T>
__device__ __forceinline__ uint64_t load_val(const T* in, int64_t i, int64_t n) {
  return i < n ? (uint64_t)in[i] : 0ull;
}

// Block-wide exclusive scan of one value per thread; returns the prefix and
// the block total.
__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* total, uint64_t* sh_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t y = __shfl_up_sync(FULL_MASK, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint64_t w = lane < (SCAN_THREADS / 32) ? sh_warp[lane] : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t y = __shfl_up_sync(FULL_MASK, w, o);
      if (lane >= o) w += y;
    }
    if (lane < (SCAN_THREADS / 32)) sh_warp[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  uint64_t warp_prefix = warp ? sh_warp[warp - 1] : 0ull;
  *total = sh_warp[SCAN_THREADS / 32 - 1];
  return warp_prefix + x - v;
}

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) scan_reduce_kernel(const T* in, int64_t n, uint64_t* partial) {
  __shared__ uint64_t sh_warp[SCAN_THREADS / 32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  uint64_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) s += load_val(in, base + k * SCAN_THREADS + threadIdx.x, n);
  uint64_t total;
  block_exclusive_scan(s, &total, sh_warp);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(SCAN_THREADS) scan_tile_kernel(const T* in, uint64_t* out, int64_t n,
                                                                 const uint64_t* block_offsets) {
  __shared__ uint64_t tile[SCAN_TILE];
  __shared__ uint64_t sh_warp[SCAN_THREADS / 32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int idx = k * SCAN_THREADS + threadIdx.x;
    tile[idx] = load_val(in, base + idx, n);
  }
  __syncthreads();
  uint64_t v[SCAN_ITEMS], s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    v[k] = tile[threadIdx.x * SCAN_ITEMS + k];
    s += v[k];
  }
  uint64_t total;
  uint64_t run = block_exclusive_scan(s, &total, sh_warp) + (block_offsets ? block_offsets[blockIdx.x] : 0ull);
  __syncthreads();
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    tile[threadIdx.x * SCAN_ITEMS + k] = run;
    run += v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int64_t i = base + k * SCAN_THREADS + threadIdx.x;
    if (i < n) out[i] = tile[k * SCAN_THREADS + threadIdx.x];
  }
  const int64_t last = base + SCAN_TILE;
  if (threadIdx.x == 0 && last >= n && base < n + 1)
    out[n] = (block_offsets ? block_offsets[blockIdx.x] : 0ull) + total;
}

size_t scan_tmp_bytes(int64_t n) {
  size_t bytes = 0;
  int64_t m = n;
  while (m > SCAN_TILE) {
    m = ceil_div(m, SCAN_TILE);
    bytes += sizeof(uint64_t) * (size_t)(2 * m + 2);
  }
  return bytes + 256;
}

template <typename T>
static int exclusive_scan_impl(const T* in, uint64_t* out, int64_t n, void* tmp, cudaStream_t s) {
  if (n <= 0) {
    G500_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), s));
    return G500_OK;
  }
  int64_t nb = ceil_div(n, SCAN_TILE);
  if (nb == 1) {
    scan_tile_kernel<T><<<1, SCAN_THREADS, 0, s>>>(in, out, n, nullptr);
    G500_CUDA(cudaGetLastError());
    return G500_OK;
  }
  uint64_t* partial = reinterpret_cast<uint64_t*>(tmp);
  uint64_t* partial_scan = partial + nb + 1;
  void* rest = partial_scan + nb + 1;
  scan_reduce_kernel<T><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, partial);
  G500_CUDA(cudaGetLastError());
  G500_TRY(exclusive_scan_impl<uint64_t>(partial, partial_scan, nb, rest, s));
  scan_tile_kernel<T><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, partial_scan);
  G500_CUDA(cudaGetLastError());
  return G500_OK;
}

int exclusive_scan_u32(const uint32_t* in, uint64_t* out, int64_t n, void* tmp, cudaStream_t s) {
  return exclusive_scan_impl<uint32_t>(in, out, n, tmp, s);
}
int exclusive_scan_u64(const uint64_t* in, uint64_t* out, int64_t n, void* tmp, cudaStream_t s) {
  return exclusive_scan_impl<uint64_t>(in, out, n, tmp, s);
}

// ---------------------------------------------------------------------------
// LSD radix sort, 8-bit digits
// ---------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 16;  // keys per lane per tile
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_BINS = 256;

static int rs_num_blocks(int64_t n) {
  int64_t tiles = ceil_div(n, RS_TILE);
  int64_t cap = (int64_t)num_sms() * 8;
  return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, cap));
}

// Each block owns a contiguous run of whole tiles: [tile_begin, tile_end).
__device__ __forceinline__ void rs_block_range(int64_t n, int64_t* b, int64_t* e) {
  int64_t tiles = (n + RS_TILE - 1) / RS_TILE;
  int64_t per = (tiles + gridDim.x - 1) / gridDim.x;
  int64_t t0 = per * blockIdx.x, t1 = min(tiles, t0 + per);
  *b = min(n, t0 * RS_TILE);
  *e = min(n, t1 * RS_TILE);
}

__global__ void __launch_bounds__(RS_THREADS) rs_upsweep_kernel(const uint64_t* keys, int64_t n, int shift,
                                                               uint32_t* hist /* [RS_BINS][grid] */) {
  __shared__ uint32_t wh[RS_WARPS][RS_BINS];
  for (int i = threadIdx.x; i < RS_WARPS * RS_BINS; i += RS_THREADS) (&wh[0][0])[i] = 0;
  __syncthreads();
  int64_t b, e;
  rs_block_range(n, &b, &e);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t base = b; base < e; base += RS_THREADS) {
    int64_t i = base + threadIdx.x;
    unsigned d = i < e ? (unsigned)((keys[i] >> shift) & 0xFF) : 0x100u;
    unsigned peers = __match_any_sync(FULL_MASK, d);
    if (d != 0x100u && (__ffs(peers) - 1) == lane) wh[warp][d] += __popc(peers);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < RS_BINS; d += RS_THREADS) {
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) s += wh[w][d];
    hist[(int64_t)d * gridDim.x + blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(RS_THREADS) rs_downsweep_kernel(const uint64_t* keys, uint64_t* out, int64_t n,
                                                                 int shift, const uint64_t* offsets /* scanned hist */) {
  __shared__ unsigned long long run[RS_BINS];  // global output position of the next key of each digit
  __shared__ uint32_t tile_total[RS_BINS];
  __shared__ uint32_t wc[RS_WARPS][RS_BINS];   // per-warp digit counts, then per-warp digit offsets
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < RS_BINS; d += RS_THREADS) run[d] = offsets[(int64_t)d * gridDim.x + blockIdx.x];
  for (int i = threadIdx.x; i < RS_WARPS * RS_BINS; i += RS_THREADS) (&wc[0][0])[i] = 0;
  __syncthreads();
  int64_t b, e;
  rs_block_range(n, &b, &e);
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int64_t tile = b; tile < e; tile += RS_TILE) {
    uint64_t k[RS_ITEMS];
    unsigned rank[RS_ITEMS];
    // keys of warp w: tile + w*512 + j*32 + lane, so (warp, j, lane) order is index order
    const int64_t wbase = tile + (int64_t)warp * (RS_ITEMS * 32);
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
      int64_t i = wbase + j * 32 + lane;
      k[j] = i < e ? keys[i] : 0ull;
      unsigned d = i < e ? (unsigned)((k[j] >> shift) & 0xFF) : 0x100u;
      unsigned peers = __match_any_sync(FULL_MASK, d);
      unsigned r = __popc(peers & lt_mask);
      unsigned before = (d != 0x100u) ? wc[warp][d] : 0u;
      __syncwarp();
      if (d != 0x100u && r == 0) wc[warp][d] = before + __popc(peers);
      __syncwarp();
      rank[j] = before + r;
    }
    __syncthreads();
    for (int d = threadIdx.x; d < RS_BINS; d += RS_THREADS) {
      uint32_t acc = 0;
#pragma unroll
      for (int w = 0; w < RS_WARPS; ++w) {
        uint32_t c = wc[w][d];
        wc[w][d] = acc;
        acc += c;
      }
      tile_total[d] = acc;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < RS_ITEMS; ++j) {
      int64_t i = wbase + j * 32 + lane;
      if (i < e) {
        unsigned d = (unsigned)((k[j] >> shift) & 0xFF);
        out[run[d] + wc[warp][d] + rank[j]] = k[j];
      }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < RS_BINS; d += RS_THREADS) {
      run[d] += tile_total[d];
#pragma unroll
      for (int w = 0; w < RS_WARPS; ++w) wc[w][d] = 0;
    }
    __syncthreads();
  }
}

size_t sort_tmp_bytes(int64_t n) {
  int g = rs_num_blocks(n);
  size_t hist = sizeof(uint32_t) * (size_t)g * RS_BINS;
  size_t offs = sizeof(uint64_t) * ((size_t)g * RS_BINS + 1);
  return hist + offs + scan_tmp_bytes((int64_t)g * RS_BINS) + 1024;
}

int radix_sort_u64(uint64_t* keys, uint64_t* alt, int64_t n, int lo_bit, int hi_bit, void* tmp,
                   cudaStream_t s, uint64_t** result) {
  *result = keys;
  if (n <= 1 || hi_bit <= lo_bit) return G500_OK;
  const int g = rs_num_blocks(n);
  uint32_t* hist = reinterpret_cast<uint32_t*>(tmp);
  uint64_t* offs = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(hist + (size_t)g * RS_BINS) + 255) & ~uintptr_t(255));
  void* scan_tmp = reinterpret_cast<void*>(
      (reinterpret_cast<uintptr_t>(offs + (size_t)g * RS_BINS + 1) + 255) & ~uintptr_t(255));
  uint64_t* src = keys;
  uint64_t* dst = alt;
  for (int shift = lo_bit; shift < hi_bit; shift += 8) {
    rs_upsweep_kernel<<<g, RS_THREADS, 0, s>>>(src, n, shift, hist);
    G500_CUDA(cudaGetLastError());
    G500_TRY(exclusive_scan_u32(hist, offs, (int64_t)g * RS_BINS, scan_tmp, s));
    rs_downsweep_kernel<<<g, RS_THREADS, 0, s>>>(src, dst, n, shift, offs);
    G500_CUDA(cudaGetLastError());
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  *result = src;
  return G500_OK;
}

}  // namespace g500
