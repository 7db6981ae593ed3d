// pred to a pageable host buffer for g500_bfs_run (the reference's driver
// allocates pred with plain host memory, main.cc:74-75): the int64 entries
// cross PCIe as 32-bit packed entries into a pinned staging buffer, in
// chunks, and host threads expand each chunk into the caller's array while
// the next one is still being copied.  The runtime's own pageable copy goes
// through its staging buffers at about half the pinned rate (SCALE 22: 1.96
// ms for the 34 MB pred against 0.92 ms this way, 0.83 ms by DMA into pinned
// memory, which stays the path for a pinned pred).  The caller's array holds
// the same int64 values either way (bfs.hpp:1203, :2470 encoding: parent |
// level << 48, -1 unreached).
//
// Packed entry: parent original id in the low PACK_BITS bits, the level
// above it; 0xFFFFFFFF = unreached.  Graphs with more than 2^PACK_BITS ids,
// and runs with a level of 31 or more, copy the int64 entries instead.
#include "g500_internal.cuh"

#include <algorithm>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

namespace g500 {
namespace {

constexpr int PACK_BITS = 27;
constexpr uint32_t PACK_UNREACHED = 0xFFFFFFFFu;
constexpr int PACK_MAX_LEVEL = 30;  // level 31 with an all-ones parent would read as unreached
constexpr int PRED_CHUNKS = 8;

__global__ void __launch_bounds__(256) pack_pred_kernel(const int64_t* __restrict__ pred, int64_t n,
                                                        uint32_t* __restrict__ out, unsigned* overflow) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  bool bad = false;
  for (int64_t i = 2 * tid; i < n; i += 2 * nthreads) {  // n is even (a multiple of 65536)
    const longlong2 v = __ldcs(reinterpret_cast<const longlong2*>(pred + i));
    uint32_t e[2];
    const long long x[2] = {v.x, v.y};
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      if (x[k] == -1) {
        e[k] = PACK_UNREACHED;
      } else {
        const uint64_t parent = (uint64_t)x[k] & ((1ull << 48) - 1);
        const uint64_t level = (uint64_t)x[k] >> 48;
        bad |= parent >= (1ull << PACK_BITS) || level > (uint64_t)PACK_MAX_LEVEL;
        e[k] = (uint32_t)parent | ((uint32_t)level << PACK_BITS);
      }
    }
    __stcs(reinterpret_cast<uint2*>(out + i), make_uint2(e[0], e[1]));
  }
  if (bad) atomicOr(overflow, 1u);
}

}  // namespace

// Host threads that expand the chunks: each waits for a chunk's copy event
// and expands its slice of it, so one wake-up per run serves every chunk.
class PredExpander {
 public:
  PredExpander(int device, int nthreads) : device_(device), n_(nthreads) {
    for (int t = 1; t < nthreads; ++t) th_.emplace_back([this, t] { loop(t); });
  }
  ~PredExpander() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }

  // expand src[0, n) into dst; chunk k = [bounds[k], bounds[k+1]) is ready
  // once ev[k] has completed
  void run(const uint32_t* src, int64_t* dst, const int64_t* bounds, cudaEvent_t* ev, int nchunks) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      src_ = src;
      dst_ = dst;
      bounds_ = bounds;
      ev_ = ev;
      nchunks_ = nchunks;
      pending_ = n_ - 1;
      ++gen_;
    }
    cv_.notify_all();
    work(0);
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [&] { return pending_ == 0; });
  }

 private:
  void loop(int t) {
    cudaSetDevice(device_);
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      work(t);
      {
        std::lock_guard<std::mutex> lk(mu_);
        --pending_;
      }
      cv_done_.notify_one();
    }
  }

  void work(int t) {
    for (int k = 0; k < nchunks_; ++k) {
      const int64_t b = bounds_[k], len = bounds_[k + 1] - b;
      const int64_t lo = b + len * t / n_, hi = b + len * (t + 1) / n_;
      cudaEventSynchronize(ev_[k]);
      const uint32_t* s = src_;
      int64_t* d = dst_;
      for (int64_t i = lo; i < hi; ++i) {
        const uint32_t e = s[i];
        d[i] = e == PACK_UNREACHED ? -1 : (int64_t)(e & ((1u << PACK_BITS) - 1u)) | ((int64_t)(e >> PACK_BITS) << 48);
      }
    }
  }

  int device_ = 0, n_ = 1;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, cv_done_;
  bool stop_ = false;
  uint64_t gen_ = 0;
  int pending_ = 0;
  const uint32_t* src_ = nullptr;
  int64_t* dst_ = nullptr;
  const int64_t* bounds_ = nullptr;
  cudaEvent_t* ev_ = nullptr;
  int nchunks_ = 0;
};

void pred_expander_free(g500_bfs* b) {
  delete b->expander;
  b->expander = nullptr;
  for (auto& e : b->ev_chunk)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  dev_free(b->d_pack);
  dev_free(b->d_pack_ovf);
  if (b->h_pack) cudaFreeHost(b->h_pack);
  b->h_pack = nullptr;
}

int pred_to_host_packed(g500_bfs* b, int64_t* host_pred, cudaStream_t s, bool* packed) {
  g500_graph* g = b->g;
  *packed = false;
  const int64_t n = g->nolv;
  if (n > (1ll << PACK_BITS) || n % 2 != 0 || b->pack_host_off) return G500_OK;
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, host_pred) != cudaSuccess) {
    cudaGetLastError();  // not a pointer the runtime knows: pageable
    attr.type = cudaMemoryTypeUnregistered;
  }
  if (attr.type != cudaMemoryTypeUnregistered) return G500_OK;  // pinned (or device): one DMA copy is faster
  if (!b->d_pack) {
    G500_TRY(dev_alloc_n(&b->d_pack, n, "packed pred"));
    G500_TRY(dev_alloc_n(&b->d_pack_ovf, 1, "packed pred overflow flag"));
    // the overflow flag lands after the entries
    G500_CUDA(cudaHostAlloc(&b->h_pack, sizeof(uint32_t) * (size_t)(n + 64), cudaHostAllocDefault));
    for (auto& e : b->ev_chunk) G500_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    const int hw = (int)std::thread::hardware_concurrency();
    b->expander = new PredExpander(g->device, std::max(1, std::min(hw > 0 ? hw : 1, 16)));
  }
  G500_CUDA(cudaMemsetAsync(b->d_pack_ovf, 0, sizeof(unsigned), s));
  const unsigned grid = (unsigned)std::min<int64_t>(ceil_div(n / 2, 256), (int64_t)num_sms() * 8);
  pack_pred_kernel<<<grid, 256, 0, s>>>(b->d_pred, n, b->d_pack, b->d_pack_ovf);
  G500_CUDA(cudaGetLastError());
  volatile uint32_t* h_ovf = b->h_pack + n;
  *h_ovf = 0;
  G500_CUDA(cudaMemcpyAsync(b->h_pack + n, b->d_pack_ovf, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  int64_t bounds[PRED_CHUNKS + 1];
  for (int k = 0; k <= PRED_CHUNKS; ++k) bounds[k] = (n * k / PRED_CHUNKS) & ~(int64_t)63;
  bounds[PRED_CHUNKS] = n;
  for (int k = 0; k < PRED_CHUNKS; ++k) {
    const int64_t lo = bounds[k], len = bounds[k + 1] - lo;
    if (len > 0)
      G500_CUDA(cudaMemcpyAsync(b->h_pack + lo, b->d_pack + lo, sizeof(uint32_t) * (size_t)len,
                                cudaMemcpyDeviceToHost, s));
    G500_CUDA(cudaEventRecord(b->ev_chunk[k], s));
  }
  // the flag arrived with the first chunk's event
  G500_CUDA(cudaEventSynchronize(b->ev_chunk[0]));
  if (*h_ovf) {  // a level or an id beyond the packed fields: the caller gets the int64 copy instead
    G500_CUDA(cudaStreamSynchronize(s));
    return G500_OK;
  }
  b->expander->run(b->h_pack, host_pred, bounds, b->ev_chunk, PRED_CHUNKS);
  *packed = true;
  return G500_OK;
}

}  // namespace g500
