// Kronecker (R-MAT) edge generation on the device, bit-exact to the
// reference's RmatGraphGenerator<.., 5700, 1900>::generateRange
// (generator/graph_generator.hpp:612-627, :651-704) driven by
// generate_graph_spec2010 (mpi/benchmark_helper.hpp:308-314).
//
// Edge i draws from the splittable MRG stream A^(i * 2^64) * seed
// (graph_generator.hpp:623: mrg_skip(&st, 0, i, 0)).  Instead of jumping from
// the seed for every edge, thread t of T owns edges start+t, start+t+T, ...
// and advances its stream by the fixed matrix P = A^(T * 2^64) per edge: one
// 5x5 matrix-vector product instead of up to eight.  Modular arithmetic is
// exact, so the streams are identical to the reference's.
#include "g500_internal.cuh"

#include <mutex>

namespace g500 {

static constexpr uint32_t MRG_P = 0x7FFFFFFFu;
static constexpr uint32_t MRG_X = 107374182u;  // splittable_mrg.c:29-34
static constexpr uint32_t MRG_Y = 104480u;

// ------------------------------------------------------------------ host
static inline uint32_t hmul(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) % MRG_P); }

void mat5_mul_host(const Mat5& a, const Mat5& b, Mat5* r) {
  Mat5 t;
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      uint64_t acc = 0;
      for (int k = 0; k < 5; ++k) acc = (acc + (uint64_t)a.m[i * 5 + k] * b.m[k * 5 + j]) % MRG_P;
      t.m[i * 5 + j] = (uint32_t)acc;
    }
  *r = t;
}

static void mat5_apply_host(const Mat5& a, uint32_t z[5]) {
  uint32_t o[5];
  for (int i = 0; i < 5; ++i) {
    uint64_t acc = 0;
    for (int k = 0; k < 5; ++k) acc = (acc + (uint64_t)a.m[i * 5 + k] * z[k]) % MRG_P;
    o[i] = (uint32_t)acc;
  }
  for (int i = 0; i < 5; ++i) z[i] = o[i];
}

// skip[b][v] = A^(v * 256^b), the byte-indexed jump table of splittable_mrg.c
// (generated there by dump_mrg_powers, :213-247); computed once here.
static std::vector<Mat5>* g_skip = nullptr;
static std::once_flag g_skip_once;

static void build_skip_table() {
  std::call_once(g_skip_once, [] {
    std::vector<Mat5>* t = new std::vector<Mat5>(24 * 256);
    Mat5 base;
    memset(&base, 0, sizeof(base));
    base.m[0] = MRG_X;
    base.m[4] = MRG_Y;
    for (int i = 1; i < 5; ++i) base.m[i * 5 + i - 1] = 1;
    for (int b = 0; b < 24; ++b) {
      Mat5& id = (*t)[b * 256];
      memset(&id, 0, sizeof(id));
      for (int i = 0; i < 5; ++i) id.m[i * 5 + i] = 1;
      (*t)[b * 256 + 1] = base;
      for (int v = 2; v < 256; ++v) mat5_mul_host((*t)[b * 256 + v - 1], base, &(*t)[b * 256 + v]);
      mat5_mul_host((*t)[b * 256 + 255], base, &base);
    }
    g_skip = t;
  });
}

void mrg_skip_matrix_host(int byte_index, int val, Mat5* out) {
  build_skip_table();
  *out = (*g_skip)[byte_index * 256 + (val & 255)];
}

// make_mrg_seed, graph_generator.hpp:327-333
void mrg_seed_host(uint64_t s1, uint64_t s2, uint32_t z[5]) {
  z[0] = (uint32_t)((s1 & 0x3FFFFFFF) + 1);
  z[1] = (uint32_t)(((s1 >> 30) & 0x3FFFFFFF) + 1);
  z[2] = (uint32_t)((s2 & 0x3FFFFFFF) + 1);
  z[3] = (uint32_t)(((s2 >> 30) & 0x3FFFFFFF) + 1);
  z[4] = (uint32_t)(((s2 >> 60) << 4) + (s1 >> 60) + 1);
}

// mrg_skip, splittable_mrg.c:185-200
void mrg_skip_host(uint32_t z[5], uint64_t hi, uint64_t mid, uint64_t lo) {
  build_skip_table();
  uint64_t parts[3] = {lo, mid, hi};
  for (int p = 0; p < 3; ++p)
    for (int b = 0; parts[p]; ++b, parts[p] >>= 8) {
      int v = (int)(parts[p] & 0xFF);
      if (v) mat5_apply_host((*g_skip)[(p * 8 + b) * 256 + v], z);
    }
}

// mrg_get_uint_orig, splittable_mrg.c:170-177, :266-269
uint32_t mrg_next_host(uint32_t z[5]) {
  uint32_t ne = (uint32_t)(((uint64_t)hmul(z[0], MRG_X) + hmul(z[4], MRG_Y)) % MRG_P);
  z[4] = z[3]; z[3] = z[2]; z[2] = z[1]; z[1] = z[0]; z[0] = ne;
  return ne;
}

// graph_generator.hpp:375-384
void scramble_values_host(uint64_t s1, uint64_t s2, uint64_t* v0, uint64_t* v1) {
  uint32_t z[5];
  mrg_seed_host(s1, s2, z);
  mrg_skip_host(z, 50, 7, 0);
  uint64_t a = mrg_next_host(z);
  a *= UINT64_C(0xFFFFFFFF);
  a += mrg_next_host(z);
  uint64_t b = mrg_next_host(z);
  b *= UINT64_C(0xFFFFFFFF);
  b += mrg_next_host(z);
  *v0 = a;
  *v1 = b;
}

// ---------------------------------------------------------------- device
struct GenParams {
  uint32_t step[25];   // P = A^(T * 2^64)
  uint32_t seed[5];
  uint64_t val0, val1; // scramble words
  int scale;
  int64_t start, end;
  uint32_t a_num, bc_num;  // R-MAT initiator numerators of 10000 (A; B = C)
  int64_t n_init;          // initial edges before the R-MAT ones (binary tree: N - 1)
};

// Mersenne folding: x mod (2^31 - 1) without a division.
__device__ __forceinline__ uint64_t fold31(uint64_t x) { return (x & MRG_P) + (x >> 31); }
__device__ __forceinline__ uint32_t reduce31(uint64_t x) {  // x < 2^62
  x = fold31(x);
  x = fold31(x);
  return (uint32_t)(x >= MRG_P ? x - MRG_P : x);
}

__device__ __forceinline__ void mat5_apply_dev(const uint32_t* __restrict__ m, uint32_t z[5]) {
  uint32_t o[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) acc += fold31((uint64_t)m[i * 5 + k] * z[k]);  // each < 2^32
    o[i] = reduce31(acc);
  }
#pragma unroll
  for (int i = 0; i < 5; ++i) z[i] = o[i];
}

__device__ __forceinline__ uint32_t mrg_next_dev(uint32_t z[5]) {
  uint32_t ne = reduce31(fold31((uint64_t)z[0] * MRG_X) + fold31((uint64_t)z[4] * MRG_Y));
  z[4] = z[3]; z[3] = z[2]; z[2] = z[1]; z[1] = z[0]; z[0] = ne;
  return ne;
}

// graph_generator.hpp:457-469; __brevll is the 64-bit bit reversal of :405-451
__device__ __forceinline__ uint64_t scramble_dev(uint64_t v, int scale, uint64_t val0, uint64_t val1) {
  v += val0 + val1;
  v *= (val0 | 0x4519840211493211ull);
  v = __brevll(v) >> (64 - scale);
  v *= (val1 | 0x3050852102C843A5ull);
  v = __brevll(v) >> (64 - scale);
  return v;
}

// generate_4way_bernoulli, graph_generator.hpp:651-677 (no noise): spec 2010
// A = .57, B = C = .19 (numerators 5700 / 1900); spec 2012 A = .55, B = C = .01
__device__ __forceinline__ int bernoulli4_dev(uint32_t z[5], uint32_t a_num, uint32_t bc_num) {
  uint32_t val = mrg_next_dev(z);
  while (val < 7295u) val = mrg_next_dev(z);  // 0xFFFFFFFF % 10000
  val %= 10000u;
  if (val < bc_num) return 1;
  val -= bc_num;
  if (val < bc_num) return 2;
  val -= bc_num;
  if (val < a_num) return 0;
  return 3;
}

__device__ __forceinline__ void put_edge(g500_packed_edge* out, int64_t i, uint64_t v0, uint64_t v1) {
  g500_packed_edge pe;
  pe.v0_low = (uint32_t)v0;
  pe.v1_low = (uint32_t)v1;
  pe.high = (uint32_t)(((v0 >> 32) & 0xFFFF) | ((v1 >> 16) & 0xFFFF0000u));
  out[i] = pe;
}

// WeightedEdge (primitives.hpp:87-106): the packed layout and a weight, which
// generateWeight sets to the constant 0xBEEF (graph_generator.hpp:495-503)
__device__ __forceinline__ void put_edge(g500_weighted_edge* out, int64_t i, uint64_t v0, uint64_t v1) {
  g500_weighted_edge w;  // 4-byte aligned: a caller's buffer need not be 16-byte aligned
  w.v0_low = (uint32_t)v0;
  w.v1_low = (uint32_t)v1;
  w.high = (uint32_t)(((v0 >> 32) & 0xFFFF) | ((v1 >> 16) & 0xFFFF0000u));
  w.weight = 0xBEEF;
  out[i] = w;
}

// Thread t of T owns edges start + t, start + t + T, ...: edges below n_init
// are the binary-tree initial edges (scramble(i + 1), scramble((i + 1) / 2))
// (generateInitialEdge, graph_generator.hpp:513-520), the others R-MAT edges
// from the stream of their own index (generateRange, :612-627).
template <typename Edge>
__global__ void __launch_bounds__(256) gen_edges_kernel(GenParams p, const uint32_t* __restrict__ skip_mid,
                                                        Edge* __restrict__ out) {
  __shared__ uint32_t step[25];
  if (threadIdx.x < 25) step[threadIdx.x] = p.step[threadIdx.x];
  __syncthreads();
  const int64_t T = (int64_t)gridDim.x * blockDim.x;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t ei = p.start + t;
  if (ei >= p.end) return;
  // stream of edge ei: A^(ei * 2^64) seed, via the middle-exponent bytes 8..15
  uint32_t z[5] = {p.seed[0], p.seed[1], p.seed[2], p.seed[3], p.seed[4]};
  uint64_t e = (uint64_t)ei;
  for (int b = 0; e; ++b, e >>= 8) {
    int v = (int)(e & 0xFF);
    if (v) mat5_apply_dev(skip_mid + ((size_t)b * 256 + v) * 25, z);
  }
  for (; ei < p.end; ei += T) {
    if (ei < p.n_init) {
      put_edge(out, ei - p.start, scramble_dev((uint64_t)(ei + 1), p.scale, p.val0, p.val1),
               scramble_dev((uint64_t)((ei + 1) / 2), p.scale, p.val0, p.val1));
    } else {
      uint32_t s[5] = {z[0], z[1], z[2], z[3], z[4]};
      // make_one_edge, graph_generator.hpp:681-704
      int64_t base_src = 0, base_tgt = 0;
      for (int lvl = p.scale - 1; lvl >= 0; --lvl) {
        int sq = bernoulli4_dev(s, p.a_num, p.bc_num);
        int so = sq >> 1, to = sq & 1;
        if (base_src == base_tgt && so > to) { int x = so; so = to; to = x; }
        base_src += (int64_t)so << lvl;
        base_tgt += (int64_t)to << lvl;
      }
      put_edge(out, ei - p.start, scramble_dev((uint64_t)base_src, p.scale, p.val0, p.val1),
               scramble_dev((uint64_t)base_tgt, p.scale, p.val0, p.val1));
    }
    mat5_apply_dev(step, z);
  }
}

static uint32_t* g_skip_mid_dev[64] = {nullptr};  // per device: bytes 8..15 of the jump table
static std::mutex g_skip_mu;

static int skip_mid_table(uint32_t** out) {
  int dev = 0;
  G500_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(G500_E_INVAL, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_skip_mu);
  if (!g_skip_mid_dev[dev]) {
    build_skip_table();
    std::vector<uint32_t> h((size_t)8 * 256 * 25);
    for (int b = 0; b < 8; ++b)
      for (int v = 0; v < 256; ++v)
        memcpy(&h[((size_t)b * 256 + v) * 25], (*g_skip)[(8 + b) * 256 + v].m, sizeof(uint32_t) * 25);
    uint32_t* d = nullptr;
    G500_TRY(dev_alloc_n(&d, (int64_t)h.size(), "MRG jump table"));
    cudaError_t e = cudaMemcpy(d, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      dev_free(d);
      return cuda_error(e, "cudaMemcpy(jump table)", __FILE__, __LINE__);
    }
    g_skip_mid_dev[dev] = d;
  }
  *out = g_skip_mid_dev[dev];
  return G500_OK;
}

template <typename Edge>
static int gen_device(int scale, uint64_t s1, uint64_t s2, int64_t start, int64_t end, uint32_t a_num,
                      uint32_t bc_num, int64_t n_init, Edge* out, cudaStream_t s) {
  if (end <= start) return G500_OK;
  uint32_t* skip_mid = nullptr;
  G500_TRY(skip_mid_table(&skip_mid));
  const int threads = 256;
  int64_t n = end - start;
  int64_t blocks = std::min<int64_t>(ceil_div(n, threads), (int64_t)num_sms() * 8);
  const uint64_t T = (uint64_t)blocks * threads;
  GenParams p;
  // P = A^(T * 2^64): product of the middle-exponent byte matrices of T
  Mat5 P;
  memset(&P, 0, sizeof(P));
  for (int i = 0; i < 5; ++i) P.m[i * 5 + i] = 1;
  uint64_t e = T;
  for (int b = 0; e; ++b, e >>= 8) {
    int v = (int)(e & 0xFF);
    if (v) {
      Mat5 M;
      mrg_skip_matrix_host(8 + b, v, &M);
      mat5_mul_host(M, P, &P);
    }
  }
  memcpy(p.step, P.m, sizeof(p.step));
  mrg_seed_host(s1, s2, p.seed);
  scramble_values_host(s1, s2, &p.val0, &p.val1);
  p.scale = scale;
  p.start = start;
  p.end = end;
  p.a_num = a_num;
  p.bc_num = bc_num;
  p.n_init = n_init;
  gen_edges_kernel<Edge><<<(unsigned)blocks, threads, 0, s>>>(p, skip_mid, out);
  G500_CUDA(cudaGetLastError());
  return G500_OK;
}

// generate_graph_spec2010 (benchmark_helper.hpp:308-314)
int gen_edges_device(int scale, uint64_t s1, uint64_t s2, int64_t start, int64_t end,
                     g500_packed_edge* out, cudaStream_t s) {
  return gen_device(scale, s1, s2, start, end, 5700u, 1900u, 0, out, s);
}

// generate_graph_spec2012 (benchmark_helper.hpp:316-322): RmatGraphGenerator<
// WeightedEdge, 5500, 100> with InitialEdgeType::BINARY_TREE (N - 1 initial edges)
int gen_edges_spec2012_device(int scale, uint64_t s1, uint64_t s2, int64_t start, int64_t end,
                              g500_weighted_edge* out, cudaStream_t s) {
  return gen_device(scale, s1, s2, start, end, 5500u, 100u, (int64_t(1) << scale) - 1, out, s);
}

}  // namespace g500
