// Library-wide C entry points: error text, pinned memory, and edge generation.
#include "g500_internal.cuh"

namespace g500 {
const char* last_error_text();
}

using namespace g500;

extern "C" int g500_abi_version(void) { return G500_ABI_VERSION; }

extern "C" const char* g500_last_error(void) { return g500::last_error_text(); }

extern "C" int g500_host_alloc(uint64_t bytes, void** out) {
  if (!out) return set_error(G500_E_INVAL, "null output");
  *out = nullptr;
  cudaError_t e = cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocPortable);
  if (e != cudaSuccess) {
    *out = nullptr;
    return cuda_error(e, "cudaHostAlloc", __FILE__, __LINE__);
  }
  return G500_OK;
}

extern "C" int g500_host_free(void* p) {
  if (p) G500_CUDA(cudaFreeHost(p));
  return G500_OK;
}

extern "C" int g500_scramble_values(int scale, uint64_t s1, uint64_t s2, uint64_t* v0, uint64_t* v1) {
  (void)scale;
  if (!v0 || !v1) return set_error(G500_E_INVAL, "null output");
  scramble_values_host(s1, s2, v0, v1);
  return G500_OK;
}

namespace {
// Edges [start, end) of a graph of `total` edges into out (device or host
// memory); host output is generated on the device in chunks and copied back.
template <typename Edge, typename Gen>
int gen_edges_to(int scale, int64_t total, int64_t start, int64_t end, Edge* out, int out_on_device, void* stream,
                 Gen gen) {
  if (start < 0 || end < start) return set_error(G500_E_INVAL, "bad edge range [%lld, %lld)", (long long)start,
                                                 (long long)end);
  if (end > total)
    return set_error(G500_E_RANGE, "edge range ends past the graph's %lld edges", (long long)total);
  if (!out && end > start) return set_error(G500_E_INVAL, "null output");
  if (end == start) return G500_OK;
  (void)scale;
  cudaStream_t s = (cudaStream_t)stream;
  cudaStream_t own = nullptr;
  if (!s) {
    G500_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
    s = own;
  }
  int st = G500_OK;
  if (out_on_device) {
    st = gen(start, end, out, s);
    if (own) {
      cudaError_t e = cudaStreamSynchronize(own);
      if (st == G500_OK && e != cudaSuccess) st = cuda_error(e, "generation", __FILE__, __LINE__);
    }
  } else {
    // generate into device memory chunk by chunk and copy back
    const int64_t chunk = int64_t(1) << 26;
    Edge* d = nullptr;
    st = dev_alloc_n(&d, std::min<int64_t>(chunk, end - start), "generation staging");
    for (int64_t b = start; st == G500_OK && b < end; b += chunk) {
      int64_t e = std::min<int64_t>(end, b + chunk);
      st = gen(b, e, d, s);
      if (st == G500_OK) {
        cudaError_t ce = cudaMemcpyAsync(out + (b - start), d, sizeof(Edge) * (e - b), cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
        if (ce != cudaSuccess) st = cuda_error(ce, "generation copy", __FILE__, __LINE__);
      }
    }
    dev_free(d);
  }
  if (own) cudaStreamDestroy(own);
  return st;
}
}  // namespace

extern "C" int g500_gen_edges(int scale, int edgefactor, uint64_t s1, uint64_t s2, int64_t start, int64_t end,
                              g500_packed_edge* out, int out_on_device, void* stream) {
  if (scale < 1 || scale > 48) return set_error(G500_E_INVAL, "scale %d not in 1..48", scale);
  if (edgefactor < 1) return set_error(G500_E_INVAL, "edgefactor %d < 1", edgefactor);
  return gen_edges_to(scale, (int64_t(1) << scale) * edgefactor, start, end, out, out_on_device, stream,
                      [&](int64_t b, int64_t e, g500_packed_edge* o, cudaStream_t s) {
                        return gen_edges_device(scale, s1, s2, b, e, o, s);
                      });
}

extern "C" int g500_gen_edges_spec2012(int scale, int edgefactor, uint64_t s1, uint64_t s2, int64_t start,
                                       int64_t end, g500_weighted_edge* out, int out_on_device, void* stream) {
  if (scale < 1 || scale > 48) return set_error(G500_E_INVAL, "scale %d not in 1..48", scale);
  if (edgefactor < 1) return set_error(G500_E_INVAL, "edgefactor %d < 1", edgefactor);
  const int64_t n = int64_t(1) << scale;
  return gen_edges_to(scale, n * edgefactor + n - 1, start, end, out, out_on_device, stream,
                      [&](int64_t b, int64_t e, g500_weighted_edge* o, cudaStream_t s) {
                        return gen_edges_spec2012_device(scale, s1, s2, b, e, o, s);
                      });
}
