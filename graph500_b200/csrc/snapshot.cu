// CSR snapshots: a constructed graph written to a file and read back, so that
// a serving process can bring its resident graphs up without regenerating
// and re-sorting them.  The reference has no such format; its only on-disk
// state is the generator's TMPFILE spill of the edge list
// (graph_generator.hpp:67-83), which still needs construction afterwards.
//
// File layout (little endian): a fixed header (magic, version, the graph's
// scalars, the byte length of every array that follows), then the arrays in
// header order.  A reader refuses a file whose magic, version or lengths do
// not match what the header's scalars imply.
#include "g500_internal.cuh"

#include <cstdio>
#include <cstring>
#include <memory>

namespace g500 {
namespace {

constexpr char SNAP_MAGIC[8] = {'G', '5', '0', '0', 'C', 'S', 'R', '1'};
constexpr uint32_t SNAP_VERSION = 2;  // 2: first[] carries FIRST_MORE
constexpr size_t SNAP_CHUNK = 64u << 20;  // staging buffer for the copies

enum SnapArray { S_OFFSETS, S_COLS, S_FIRST, S_REORDER, S_INVERT, S_VIS_INIT, S_ENDP, S_HAS_EDGE, S_EDGES, S_NUM };

struct SnapHeader {
  char magic[8];
  uint32_t version;
  int32_t reorder_mode;
  int32_t log_bits;
  int32_t first_flags;
  int64_t log_orig_global_verts, nolv, nlv, ngv, nge, max_used_vertex, num_edges, device_bytes;
  double gen_seconds, build_seconds;
  uint64_t bytes[S_NUM];
};

struct FileCloser {
  void operator()(FILE* f) const {
    if (f) std::fclose(f);
  }
};
using File = std::unique_ptr<FILE, FileCloser>;

void expected_bytes(const SnapHeader& h, uint64_t out[S_NUM]) {
  out[S_OFFSETS] = 8ull * (uint64_t)(h.nlv + 1);
  out[S_COLS] = 4ull * (uint64_t)h.nge;
  out[S_FIRST] = 4ull * (uint64_t)h.nlv;
  out[S_REORDER] = 4ull * (uint64_t)h.nolv;
  out[S_INVERT] = 4ull * (uint64_t)h.nolv;
  out[S_VIS_INIT] = 4ull * (uint64_t)std::max<int64_t>(h.nlv / 32, 1);
  out[S_ENDP] = 4ull * (uint64_t)h.nolv;
  out[S_HAS_EDGE] = 4ull * (uint64_t)(h.nolv / 32);
  out[S_EDGES] = sizeof(g500_packed_edge) * (uint64_t)h.num_edges;
}

// device -> file through the pinned staging buffer
int write_device(FILE* f, const void* dev, uint64_t bytes, void* stage, cudaStream_t s) {
  const char* p = static_cast<const char*>(dev);
  for (uint64_t off = 0; off < bytes; off += SNAP_CHUNK) {
    const size_t n = (size_t)std::min<uint64_t>(SNAP_CHUNK, bytes - off);
    G500_CUDA(cudaMemcpyAsync(stage, p + off, n, cudaMemcpyDeviceToHost, s));
    G500_CUDA(cudaStreamSynchronize(s));
    if (std::fwrite(stage, 1, n, f) != n) return set_error(G500_E_IO, "snapshot write failed");
  }
  return G500_OK;
}

// file -> device through the pinned staging buffer
int read_device(FILE* f, void* dev, uint64_t bytes, void* stage, cudaStream_t s) {
  char* p = static_cast<char*>(dev);
  for (uint64_t off = 0; off < bytes; off += SNAP_CHUNK) {
    const size_t n = (size_t)std::min<uint64_t>(SNAP_CHUNK, bytes - off);
    if (std::fread(stage, 1, n, f) != n) return set_error(G500_E_IO, "snapshot file is truncated");
    G500_CUDA(cudaMemcpyAsync(p + off, stage, n, cudaMemcpyHostToDevice, s));
    G500_CUDA(cudaStreamSynchronize(s));
  }
  return G500_OK;
}

struct Pinned {
  void* p = nullptr;
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

}  // namespace
}  // namespace g500

using namespace g500;

extern "C" int g500_graph_save(const g500_graph* g, const char* path) {
  if (!g || !path) return set_error(G500_E_INVAL, "null argument");
  G500_CUDA(cudaSetDevice(g->device));
  SnapHeader h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, SNAP_MAGIC, sizeof(h.magic));
  h.version = SNAP_VERSION;
  h.reorder_mode = g->reorder_mode;
  h.log_bits = g->log_bits;
  h.first_flags = g->first_flags ? 1 : 0;
  h.log_orig_global_verts = g->log_orig_global_verts;
  h.nolv = g->nolv;
  h.nlv = g->nlv;
  h.ngv = g->ngv;
  h.nge = g->nge;
  h.max_used_vertex = g->max_used_vertex;
  h.num_edges = g->d_edges ? g->num_edges : 0;
  h.device_bytes = g->device_bytes;
  h.gen_seconds = g->gen_seconds;
  h.build_seconds = g->build_seconds;
  expected_bytes(h, h.bytes);
  if (g->h_has_edge_orig.size() * 4 != h.bytes[S_HAS_EDGE]) return set_error(G500_E_STATE, "graph is incomplete");
  File f(std::fopen(path, "wb"));
  if (!f) return set_error(G500_E_IO, "cannot create %s", path);
  if (std::fwrite(&h, sizeof(h), 1, f.get()) != 1) return set_error(G500_E_IO, "snapshot write failed");
  Pinned stage;
  G500_CUDA(cudaHostAlloc(&stage.p, SNAP_CHUNK, cudaHostAllocDefault));
  cudaStream_t s = g->stream;
  const void* dev[S_NUM] = {g->d_offsets, g->d_cols, g->d_first, g->d_reorder, g->d_invert,
                            g->d_vis_init, g->d_endp, nullptr, g->d_edges};
  for (int a = 0; a < S_NUM; ++a) {
    if (h.bytes[a] == 0) continue;
    if (a == S_HAS_EDGE) {
      if (std::fwrite(g->h_has_edge_orig.data(), 1, h.bytes[a], f.get()) != h.bytes[a])
        return set_error(G500_E_IO, "snapshot write failed");
    } else {
      G500_TRY(write_device(f.get(), dev[a], h.bytes[a], stage.p, s));
    }
  }
  if (std::fflush(f.get()) != 0) return set_error(G500_E_IO, "snapshot write failed");
  return G500_OK;
}

extern "C" int g500_graph_load(const char* path, int device, g500_graph** out) {
  if (!path || !out) return set_error(G500_E_INVAL, "null argument");
  File f(std::fopen(path, "rb"));
  if (!f) return set_error(G500_E_IO, "cannot open %s", path);
  SnapHeader h;
  if (std::fread(&h, sizeof(h), 1, f.get()) != 1) return set_error(G500_E_IO, "%s: no snapshot header", path);
  if (memcmp(h.magic, SNAP_MAGIC, sizeof(h.magic)) != 0) return set_error(G500_E_IO, "%s is not a graph snapshot", path);
  if (h.version != SNAP_VERSION) return set_error(G500_E_IO, "%s: snapshot version %u, expected %u", path, h.version, SNAP_VERSION);
  uint64_t want[S_NUM];
  if (h.nolv < 0 || h.nlv < 0 || h.nge < 0 || h.num_edges < 0 || h.nlv > h.nolv || h.nolv % 32 != 0)
    return set_error(G500_E_IO, "%s: inconsistent snapshot header", path);
  expected_bytes(h, want);
  for (int a = 0; a < S_NUM; ++a)
    if (want[a] != h.bytes[a]) return set_error(G500_E_IO, "%s: inconsistent snapshot header (array %d)", path, a);
  g500_graph* g = nullptr;
  G500_TRY(new_graph(device, h.reorder_mode, &g));
  g->log_bits = h.log_bits;
  g->first_flags = h.first_flags != 0;
  g->log_orig_global_verts = h.log_orig_global_verts;
  g->nolv = h.nolv;
  g->nlv = h.nlv;
  g->ngv = h.ngv;
  g->nge = h.nge;
  g->max_used_vertex = h.max_used_vertex;
  g->device_bytes = h.device_bytes;
  g->gen_seconds = h.gen_seconds;
  g->build_seconds = h.build_seconds;
  int st = dev_alloc_n(&g->d_offsets, h.nlv + 1, "offsets");
  if (st == G500_OK) st = dev_alloc_n(&g->d_cols, std::max<int64_t>(h.nge, 1), "cols");
  if (st == G500_OK) st = dev_alloc_n(&g->d_first, std::max<int64_t>(h.nlv, 1), "first neighbours");
  if (st == G500_OK) st = dev_alloc_n(&g->d_reorder, std::max<int64_t>(h.nolv, 1), "reorder_map");
  if (st == G500_OK) st = dev_alloc_n(&g->d_invert, std::max<int64_t>(h.nolv, 1), "invert_map");
  if (st == G500_OK) st = dev_alloc_n(&g->d_vis_init, std::max<int64_t>(h.nlv / 32, 1), "visited init bitmap");
  if (st == G500_OK) st = dev_alloc_n(&g->d_endp, std::max<int64_t>(h.nolv, 1), "endpoint counts");
  if (st == G500_OK && h.num_edges > 0) {
    st = dev_alloc_n(&g->d_edges, h.num_edges, "edge list");
    g->owns_edges = true;
    g->num_edges = h.num_edges;
  }
  Pinned stage;
  if (st == G500_OK) {
    const cudaError_t e = cudaHostAlloc(&stage.p, SNAP_CHUNK, cudaHostAllocDefault);
    if (e != cudaSuccess) st = cuda_error(e, "cudaHostAlloc", __FILE__, __LINE__);
  }
  void* dev[S_NUM] = {g->d_offsets, g->d_cols, g->d_first, g->d_reorder, g->d_invert,
                      g->d_vis_init, g->d_endp, nullptr, g->d_edges};
  for (int a = 0; a < S_NUM && st == G500_OK; ++a) {
    if (h.bytes[a] == 0) continue;
    if (a == S_HAS_EDGE) {
      g->h_has_edge_orig.assign((size_t)(h.bytes[a] / 4), 0u);
      if (std::fread(g->h_has_edge_orig.data(), 1, h.bytes[a], f.get()) != h.bytes[a])
        st = set_error(G500_E_IO, "%s is truncated", path);
    } else {
      st = read_device(f.get(), dev[a], h.bytes[a], stage.p, g->stream);
    }
  }
  if (st == G500_OK && std::fgetc(f.get()) != EOF) st = set_error(G500_E_IO, "%s: bytes after the last array", path);
  if (st != G500_OK) {
    graph_destroy_internal(g);
    return st;
  }
  *out = g;
  return G500_OK;
}
