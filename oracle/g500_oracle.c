/*
 * g500_oracle.c -- CPU restatement of the suzumura/graph500 BFS hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): imported by tests/, by
 * __graft_entry__.smoke() and by the cpu_baseline leg of bench.py.  The CUDA
 * library never links or calls it.
 *
 * Written from the reference's algorithm description; no reference source is
 * included.  Each function names the reference lines it follows.
 */
#include "g500_oracle.h"

#include <stdlib.h>
#include <string.h>
#include <math.h>

#define MRG_P 0x7FFFFFFFu            /* modulus 2^31 - 1 */
#define MRG_X 107374182u             /* splittable_mrg.c:29-34 multiplier x */
#define MRG_Y 104480u                /*                        multiplier y */

/* ------------------------------------------------------------------------- */
/* Splittable MRG                                                             */
/* ------------------------------------------------------------------------- */

/* mod_arith_64bit.h:26-30: (a*b) mod 2^31-1 using a 64-bit product. */
static inline uint32_t mulmod(uint32_t a, uint32_t b) {
  return (uint32_t)(((uint64_t)a * b) % MRG_P);
}
static inline uint32_t addmod(uint32_t a, uint32_t b) {
  return (uint32_t)(((uint64_t)a + b) % MRG_P);
}

/* Dense 5x5 matrices mod p.  splittable_mrg.c:21-28 defines the one-step
 * transition A (first row x 0 0 0 y, then the shift rows). */
typedef struct { uint32_t m[25]; } mat5;

static void mat5_identity(mat5* r) {
  memset(r, 0, sizeof(*r));
  for (int i = 0; i < 5; ++i) r->m[i * 5 + i] = 1;
}
static void mat5_A(mat5* r) {
  memset(r, 0, sizeof(*r));
  r->m[0] = MRG_X;
  r->m[4] = MRG_Y;
  for (int i = 1; i < 5; ++i) r->m[i * 5 + (i - 1)] = 1;
}
static void mat5_mul(const mat5* a, const mat5* b, mat5* r) {
  mat5 t;
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      uint64_t acc = 0;
      for (int k = 0; k < 5; ++k) acc = (acc + (uint64_t)a->m[i * 5 + k] * b->m[k * 5 + j]) % MRG_P;
      t.m[i * 5 + j] = (uint32_t)acc;
    }
  *r = t;
}
static void mat5_apply(const mat5* a, orc_mrg_state* st) {
  uint32_t z[5] = {st->z1, st->z2, st->z3, st->z4, st->z5}, o[5];
  for (int i = 0; i < 5; ++i) {
    uint64_t acc = 0;
    for (int k = 0; k < 5; ++k) acc = (acc + (uint64_t)a->m[i * 5 + k] * z[k]) % MRG_P;
    o[i] = (uint32_t)acc;
  }
  st->z1 = o[0]; st->z2 = o[1]; st->z3 = o[2]; st->z4 = o[3]; st->z5 = o[4];
}

/* Jump table: skip[b][v] = A^(v * 256^b) for the 24 bytes of a 192-bit
 * exponent (the table mrg_transitions.c holds, splittable_mrg.c:213-247 says
 * how it is made).  Computed here at first use. */
static mat5 g_skip[24][256];
static int g_skip_ready = 0;

static void build_skip_table(void) {
  if (g_skip_ready) return;
#pragma omp critical(orc_skip_table)
  {
    if (!g_skip_ready) {
      mat5 base;
      mat5_A(&base); /* A^(256^0) */
      for (int b = 0; b < 24; ++b) {
        mat5_identity(&g_skip[b][0]);
        g_skip[b][1] = base;
        for (int v = 2; v < 256; ++v) mat5_mul(&g_skip[b][v - 1], &base, &g_skip[b][v]);
        mat5_mul(&g_skip[b][255], &base, &base); /* A^(256^(b+1)) */
      }
      __sync_synchronize();
      g_skip_ready = 1;
    }
  }
}

void orc_mrg_skip_matrix(int byte_index, int val, uint32_t out[25]) {
  build_skip_table();
  memcpy(out, g_skip[byte_index][val & 255].m, sizeof(uint32_t) * 25);
}

/* splittable_mrg.c:185-200: apply A^exponent byte by byte (the 192-bit exponent
 * is exp_high:exp_mid:exp_low). */
void orc_mrg_skip(orc_mrg_state* st, uint64_t exp_high, uint64_t exp_mid, uint64_t exp_low) {
  build_skip_table();
  uint64_t parts[3] = {exp_low, exp_mid, exp_high};
  for (int p = 0; p < 3; ++p) {
    uint64_t e = parts[p];
    for (int b = 0; e; ++b, e >>= 8) {
      int v = (int)(e & 0xFF);
      if (v) mat5_apply(&g_skip[p * 8 + b][v], st);
    }
  }
}

/* splittable_mrg.c:170-177 and :266-269: one step of A, return z1. */
uint32_t orc_mrg_get_uint_orig(orc_mrg_state* st) {
  uint32_t ne = addmod(mulmod(st->z1, MRG_X), mulmod(st->z5, MRG_Y));
  st->z5 = st->z4; st->z4 = st->z3; st->z3 = st->z2; st->z2 = st->z1; st->z1 = ne;
  return ne;
}

/* splittable_mrg.c:272-276. */
double orc_mrg_get_double_orig(orc_mrg_state* st) {
  double a = (double)orc_mrg_get_uint_orig(st) * .000000000465661287524579692;
  double b = (double)orc_mrg_get_uint_orig(st) * .0000000000000000002168404346990492787;
  return a + b;
}

/* graph_generator.hpp:327-333. */
void orc_make_mrg_seed(uint64_t s1, uint64_t s2, orc_mrg_state* st) {
  st->z1 = (uint32_t)((s1 & 0x3FFFFFFF) + 1);
  st->z2 = (uint32_t)(((s1 >> 30) & 0x3FFFFFFF) + 1);
  st->z3 = (uint32_t)((s2 & 0x3FFFFFFF) + 1);
  st->z4 = (uint32_t)(((s2 >> 30) & 0x3FFFFFFF) + 1);
  st->z5 = (uint32_t)(((s2 >> 60) << 4) + (s1 >> 60) + 1);
}

/* graph_generator.hpp:338-354: two PRNG outputs per double, stream at
 * exponent 2*2^128 + 2*position. */
void orc_make_random_numbers(int64_t n, uint64_t s1, uint64_t s2, int64_t position, double* out) {
  orc_mrg_state st;
  orc_make_mrg_seed(s1, s2, &st);
  orc_mrg_skip(&st, 2, 0, (uint64_t)(2 * position));
  for (int64_t i = 0; i < n; ++i) out[i] = orc_mrg_get_double_orig(&st);
}

/* ------------------------------------------------------------------------- */
/* Kronecker generator                                                        */
/* ------------------------------------------------------------------------- */

int64_t orc_edge_v0(const orc_packed_edge* e) {
  return (int64_t)e->v0_low | ((int64_t)(e->high & 0xFFFF) << 32);     /* primitives.hpp:61 */
}
int64_t orc_edge_v1(const orc_packed_edge* e) {
  return (int64_t)e->v1_low | ((int64_t)(e->high >> 16) << 32);        /* primitives.hpp:62 */
}
static inline void edge_set(orc_packed_edge* e, int64_t v0, int64_t v1) { /* primitives.hpp:63-67 */
  e->v0_low = (uint32_t)v0;
  e->v1_low = (uint32_t)v1;
  e->high = (uint32_t)(((v0 >> 32) & 0xFFFF) | ((v1 >> 16) & 0xFFFF0000u));
}

/* graph_generator.hpp:375-384: the two scramble words come from the stream at
 * exponent 50*2^128 + 7*2^64; val = u1 * 0xFFFFFFFF + u2 (64-bit wrap). */
void orc_scramble_values(int scale, uint64_t s1, uint64_t s2, uint64_t* val0, uint64_t* val1) {
  (void)scale;
  orc_mrg_state st;
  orc_make_mrg_seed(s1, s2, &st);
  orc_mrg_skip(&st, 50, 7, 0);
  uint64_t a = orc_mrg_get_uint_orig(&st);
  a *= UINT64_C(0xFFFFFFFF);
  a += orc_mrg_get_uint_orig(&st);
  uint64_t b = orc_mrg_get_uint_orig(&st);
  b *= UINT64_C(0xFFFFFFFF);
  b += orc_mrg_get_uint_orig(&st);
  *val0 = a;
  *val1 = b;
}

/* graph_generator.hpp:405-451: full 64-bit bit reversal. */
static inline uint64_t bitreverse64(uint64_t x) {
  x = __builtin_bswap64(x);
  x = ((x >> 4) & UINT64_C(0x0F0F0F0F0F0F0F0F)) | ((x & UINT64_C(0x0F0F0F0F0F0F0F0F)) << 4);
  x = ((x >> 2) & UINT64_C(0x3333333333333333)) | ((x & UINT64_C(0x3333333333333333)) << 2);
  x = ((x >> 1) & UINT64_C(0x5555555555555555)) | ((x & UINT64_C(0x5555555555555555)) << 1);
  return x;
}

/* graph_generator.hpp:457-469. */
int64_t orc_scramble(int64_t v0, int scale, uint64_t val0, uint64_t val1) {
  uint64_t v = (uint64_t)v0;
  v += val0 + val1;
  v *= (val0 | UINT64_C(0x4519840211493211));
  v = bitreverse64(v) >> (64 - scale);
  v *= (val1 | UINT64_C(0x3050852102C843A5));
  v = bitreverse64(v) >> (64 - scale);
  return (int64_t)v;
}

/* graph_generator.hpp:651-677 with SPK_NOISE_LEVEL 0; initiator numerators
 * of 10000: spec 2010 A=5700, B=C=1900 (benchmark_helper.hpp:311), spec 2012
 * A=5500, B=C=100 (benchmark_helper.hpp:319). */
static inline int bernoulli4(orc_mrg_state* st, uint32_t a_num, uint32_t bc_num) {
  const uint32_t limit = 0xFFFFFFFFu % 10000u; /* 7295 */
  uint32_t val = orc_mrg_get_uint_orig(st);
  while (val < limit) val = orc_mrg_get_uint_orig(st);
  val %= 10000u;
  if (val < bc_num) return 1;
  val -= bc_num;
  if (val < bc_num) return 2;
  val -= bc_num;
  if (val < a_num) return 0;
  return 3;
}

/* make_one_edge (graph_generator.hpp:681-704): R-MAT descent with
 * clip-and-flip from the stream of edge ei (ei * 2^64, :622-625). */
static void rmat_edge(const orc_mrg_state* seed, int scale, uint64_t val0, uint64_t val1, int64_t ei,
                      uint32_t a_num, uint32_t bc_num, int64_t* src, int64_t* tgt) {
  orc_mrg_state st = *seed;
  orc_mrg_skip(&st, 0, (uint64_t)ei, 0);
  int64_t nverts = INT64_C(1) << scale, base_src = 0, base_tgt = 0;
  while (nverts > 1) {
    int square = bernoulli4(&st, a_num, bc_num);
    int src_off = square / 2, tgt_off = square % 2;
    if (base_src == base_tgt && src_off > tgt_off) { int t = src_off; src_off = tgt_off; tgt_off = t; }
    nverts /= 2;
    base_src += nverts * src_off;
    base_tgt += nverts * tgt_off;
  }
  *src = orc_scramble(base_src, scale, val0, val1);
  *tgt = orc_scramble(base_tgt, scale, val0, val1);
}

void orc_generate_edges(int scale, int edgefactor, uint64_t s1, uint64_t s2,
                        int64_t start, int64_t end, orc_packed_edge* out) {
  (void)edgefactor;
  build_skip_table();
  orc_mrg_state seed;
  orc_make_mrg_seed(s1, s2, &seed);
  uint64_t val0, val1;
  orc_scramble_values(scale, s1, s2, &val0, &val1);
#pragma omp parallel for schedule(static)
  for (int64_t ei = start; ei < end; ++ei) {
    int64_t a, b;
    rmat_edge(&seed, scale, val0, val1, ei, 5700u, 1900u, &a, &b);
    edge_set(&out[ei - start], a, b);
  }
}

/* generate_graph_spec2012 (benchmark_helper.hpp:316-322):
 * RmatGraphGenerator<WeightedEdge, 5500, 100> with BINARY_TREE initial edges.
 * Edge i < N - 1 is (scramble(i + 1), scramble((i + 1) / 2))
 * (graph_generator.hpp:385-392, :513-520); later edges are R-MAT edges of
 * their own index (:612-627); every weight is 0xBEEF (generateWeight,
 * :495-503, the random draw disabled). */
void orc_generate_edges_spec2012(int scale, int edgefactor, uint64_t s1, uint64_t s2,
                                 int64_t start, int64_t end, orc_weighted_edge* out) {
  (void)edgefactor;
  build_skip_table();
  orc_mrg_state seed;
  orc_make_mrg_seed(s1, s2, &seed);
  uint64_t val0, val1;
  orc_scramble_values(scale, s1, s2, &val0, &val1);
  const int64_t n_init = (INT64_C(1) << scale) - 1;
#pragma omp parallel for schedule(static)
  for (int64_t ei = start; ei < end; ++ei) {
    int64_t a, b;
    if (ei < n_init) {
      a = orc_scramble(ei + 1, scale, val0, val1);
      b = orc_scramble((ei + 1) / 2, scale, val0, val1);
    } else {
      rmat_edge(&seed, scale, val0, val1, ei, 5500u, 100u, &a, &b);
    }
    orc_packed_edge pe;
    edge_set(&pe, a, b);
    out[ei - start].v0_low = pe.v0_low;
    out[ei - start].v1_low = pe.v1_low;
    out[ei - start].high = pe.high;
    out[ei - start].weight = 0xBEEF;
  }
}

/* ------------------------------------------------------------------------- */
/* Graph construction (one rank)                                              */
/* ------------------------------------------------------------------------- */

struct orc_graph {
  int64_t info[ORC_INFO_COUNT];
  int64_t* degree;        /* by original id */
  uint32_t* reorder_map;  /* original -> reordered */
  uint32_t* invert_map;   /* reordered -> original */
  uint64_t* offsets;      /* reordered rows */
  uint32_t* cols;
};

static inline int msb_index(uint64_t v) { return 63 - __builtin_clzll(v); }
static inline int64_t roundup64(int64_t v, int64_t w) { return (v + w - 1) / w * w; }

static const int64_t* g_sort_degree; /* qsort context (single-threaded use) */
static int cmp_degree_desc(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  int64_t dx = g_sort_degree[x], dy = g_sort_degree[y];
  if (dx != dy) return dx > dy ? -1 : 1;
  return x < y ? -1 : (x > y ? 1 : 0);
}
static int cmp_u32(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* graph_constructor.hpp:554-574 (construct), restated for one rank:
 *  - searchMaxVertex (:735-763): OR of all ids -> log_orig_global_verts;
 *    initializeParameters (:659-674) with a 65536-vertex unit (bfs.hpp:109 and
 *    :557 give max(11, 16)).
 *  - calc_degree (:296-352): degree = non-self-loop endpoint occurrences,
 *    duplicates included; reorder 0 = identity, 1 = vertices with edges first,
 *    2 = degree descending.  The reference's std::sort is unstable; ties are
 *    broken here by ascending original id (a stable order).
 *  - num_local_verts = roundup(last reordered vertex with edges + 1, 65536).
 *  - scatterAndStore/sortEdges (:1183-1280, :1363-1442): both directions of
 *    every non-self-loop edge, rows sorted by reordered target, duplicates
 *    dropped.  The first entry of each row is the reference's isolated edge
 *    (:845-879); it stays in place here.
 *  - computeNumVertices (:1444-1464): vertices with >= 1 edge. */
orc_graph* orc_graph_build(const orc_packed_edge* edges, int64_t m, int reorder_mode) {
  orc_graph* g = (orc_graph*)calloc(1, sizeof(orc_graph));
  uint64_t orv = 0;
  for (int64_t i = 0; i < m; ++i) orv |= (uint64_t)(orc_edge_v0(&edges[i]) | orc_edge_v1(&edges[i]));
  int log_max = orv ? msb_index(orv) + 1 : 0;
  int64_t nolv = roundup64(INT64_C(1) << log_max, 65536);
  g->info[ORC_INFO_LOG_ORIG_GLOBAL_VERTS] = log_max;
  g->info[ORC_INFO_NUM_ORIG_LOCAL_VERTS] = nolv;

  g->degree = (int64_t*)calloc((size_t)nolv, sizeof(int64_t));
  for (int64_t i = 0; i < m; ++i) {
    int64_t a = orc_edge_v0(&edges[i]), b = orc_edge_v1(&edges[i]);
    if (a == b) continue;
    g->degree[a]++;
    g->degree[b]++;
  }
  g->invert_map = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)nolv);
  g->reorder_map = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)nolv);
  for (int64_t i = 0; i < nolv; ++i) g->invert_map[i] = (uint32_t)i;
  if (reorder_mode == 2) {
    g_sort_degree = g->degree;
    qsort(g->invert_map, (size_t)nolv, sizeof(uint32_t), cmp_degree_desc);
  } else if (reorder_mode == 1) {
    int64_t k = 0;
    for (int64_t i = 0; i < nolv; ++i) if (g->degree[i]) g->invert_map[k++] = (uint32_t)i;
    for (int64_t i = 0; i < nolv; ++i) if (!g->degree[i]) g->invert_map[k++] = (uint32_t)i;
  }
  for (int64_t i = 0; i < nolv; ++i) g->reorder_map[g->invert_map[i]] = (uint32_t)i;

  int64_t last = -1, nverts = 0;
  for (int64_t i = 0; i < nolv; ++i)
    if (g->degree[g->invert_map[i]]) { last = i; ++nverts; }
  int64_t nlv = roundup64(last + 1, 65536);
  g->info[ORC_INFO_NUM_LOCAL_VERTS] = nlv;
  g->info[ORC_INFO_NUM_GLOBAL_VERTS] = nverts;

  /* CSR over reordered ids */
  uint64_t* cnt = (uint64_t*)calloc((size_t)nlv + 1, sizeof(uint64_t));
  for (int64_t i = 0; i < m; ++i) {
    int64_t a = orc_edge_v0(&edges[i]), b = orc_edge_v1(&edges[i]);
    if (a == b) continue;
    cnt[g->reorder_map[a] + 1]++;
    cnt[g->reorder_map[b] + 1]++;
  }
  for (int64_t i = 0; i < nlv; ++i) cnt[i + 1] += cnt[i];
  uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(cnt[nlv] ? cnt[nlv] : 1));
  uint64_t* pos = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(nlv ? nlv : 1));
  memcpy(pos, cnt, sizeof(uint64_t) * (size_t)nlv);
  for (int64_t i = 0; i < m; ++i) {
    int64_t a = orc_edge_v0(&edges[i]), b = orc_edge_v1(&edges[i]);
    if (a == b) continue;
    uint32_t ra = g->reorder_map[a], rb = g->reorder_map[b];
    tmp[pos[ra]++] = rb;
    tmp[pos[rb]++] = ra;
  }
  g->offsets = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(nlv + 1));
  g->cols = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(cnt[nlv] ? cnt[nlv] : 1));
  uint64_t out = 0;
  for (int64_t r = 0; r < nlv; ++r) {
    g->offsets[r] = out;
    uint64_t b = cnt[r], e = cnt[r + 1];
    if (e > b) qsort(tmp + b, (size_t)(e - b), sizeof(uint32_t), cmp_u32);
    for (uint64_t j = b; j < e; ++j)
      if (j == b || tmp[j] != tmp[j - 1]) g->cols[out++] = tmp[j];
  }
  g->offsets[nlv] = out;
  g->info[ORC_INFO_NUM_GLOBAL_EDGES] = (int64_t)out;
  free(cnt); free(tmp); free(pos);
  g->info[ORC_INFO_MAX_USED_VERTEX] = orc_find_max_used_vertex(g);
  return g;
}

void orc_graph_free(orc_graph* g) {
  if (!g) return;
  free(g->degree); free(g->reorder_map); free(g->invert_map); free(g->offsets); free(g->cols);
  free(g);
}
void orc_graph_info(const orc_graph* g, int64_t info[ORC_INFO_COUNT]) {
  memcpy(info, g->info, sizeof(g->info));
}
const uint64_t* orc_graph_offsets(const orc_graph* g) { return g->offsets; }
const uint32_t* orc_graph_cols(const orc_graph* g) { return g->cols; }
const uint32_t* orc_graph_reorder_map(const orc_graph* g) { return g->reorder_map; }
const uint32_t* orc_graph_invert_map(const orc_graph* g) { return g->invert_map; }
const int64_t* orc_graph_degree(const orc_graph* g) { return g->degree; }

/* graph_constructor.hpp:101-110: the vertex has at least one non-self-loop
 * edge.  (The reference compares reorder_map[v] > num_local_verts, which for
 * a vertex with no edges and reorder_map[v] == num_local_verts reads one word
 * past has_edge_bitmap; here such vertices simply have no edge.) */
int orc_graph_has_edge(const orc_graph* g, int64_t v) {
  if (v < 0 || v >= g->info[ORC_INFO_NUM_ORIG_LOCAL_VERTS]) return 0;
  return g->degree[v] != 0;
}

/* benchmark_helper.hpp:475-508. */
int orc_find_roots(const orc_graph* g, int num_roots, uint64_t s1, uint64_t s2, int64_t* roots) {
  int64_t counter = 0;
  const int64_t nglobalverts = INT64_C(1) << g->info[ORC_INFO_LOG_ORIG_GLOBAL_VERTS];
  int k;
  for (k = 0; k < num_roots; ++k) {
    int64_t root;
    for (;;) {
      double d[2];
      orc_make_random_numbers(2, s1, s2, counter, d);
      root = (int64_t)((d[0] + d[1]) * nglobalverts) % nglobalverts;
      counter += 2;
      if (counter > 2 * nglobalverts) break;
      int dup = 0;
      for (int i = 0; i < k; ++i) if (roots[i] == root) { dup = 1; break; }
      if (dup) continue;
      if (orc_graph_has_edge(g, root)) break;
    }
    roots[k] = root;
  }
  return k;
}

/* benchmark_helper.hpp:510-528: the largest vertex id that has an edge (0 if none). */
int64_t orc_find_max_used_vertex(const orc_graph* g) {
  for (int64_t v = g->info[ORC_INFO_NUM_ORIG_LOCAL_VERTS] - 1; v > 0; --v)
    if (orc_graph_has_edge(g, v)) return v;
  return 0;
}

/* ------------------------------------------------------------------------- */
/* BFS                                                                        */
/* ------------------------------------------------------------------------- */

/* Level-synchronous BFS over the reordered CSR.  Levels are unique (they are
 * shortest-path distances), so any correct BFS gives the reference's
 * (pred >> 48) array (bfs.hpp:1203, :2470; validate.hpp:813). */
static void bfs_core(const orc_graph* g, int64_t root, uint16_t* lvl_r, uint32_t* parent_r) {
  const int64_t nlv = g->info[ORC_INFO_NUM_LOCAL_VERTS];
  for (int64_t i = 0; i < nlv; ++i) lvl_r[i] = 0xFFFF;
  uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(nlv ? nlv : 1));
  int64_t head = 0, tail = 0;
  uint32_t r = g->reorder_map[root];
  if ((int64_t)r < nlv) {
    lvl_r[r] = 0;
    if (parent_r) parent_r[r] = r;
    q[tail++] = r;
  }
  while (head < tail) {
    uint32_t u = q[head++];
    for (uint64_t j = g->offsets[u]; j < g->offsets[u + 1]; ++j) {
      uint32_t w = g->cols[j];
      if (lvl_r[w] == 0xFFFF) {
        lvl_r[w] = (uint16_t)(lvl_r[u] + 1);
        if (parent_r) parent_r[w] = u;
        q[tail++] = w;
      }
    }
  }
  free(q);
}

void orc_bfs_levels(const orc_graph* g, int64_t root, uint16_t* levels) {
  const int64_t nlv = g->info[ORC_INFO_NUM_LOCAL_VERTS];
  const int64_t nolv = g->info[ORC_INFO_NUM_ORIG_LOCAL_VERTS];
  uint16_t* lr = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)(nlv ? nlv : 1));
  bfs_core(g, root, lr, NULL);
  for (int64_t v = 0; v < nolv; ++v) {
    uint32_t r = g->reorder_map[v];
    levels[v] = ((int64_t)r < nlv) ? lr[r] : 0xFFFF;
  }
  /* a root without edges is still reached at level 0 */
  if (root >= 0 && root < nolv) levels[root] = 0;
  free(lr);
}

void orc_bfs_pred(const orc_graph* g, int64_t root, int64_t* pred) {
  const int64_t nlv = g->info[ORC_INFO_NUM_LOCAL_VERTS];
  const int64_t nolv = g->info[ORC_INFO_NUM_ORIG_LOCAL_VERTS];
  uint16_t* lr = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)(nlv ? nlv : 1));
  uint32_t* pr = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(nlv ? nlv : 1));
  bfs_core(g, root, lr, pr);
  for (int64_t v = 0; v < nolv; ++v) {
    uint32_t r = g->reorder_map[v];
    if ((int64_t)r < nlv && lr[r] != 0xFFFF)
      pred[v] = (int64_t)g->invert_map[pr[r]] | ((int64_t)lr[r] << 48);
    else
      pred[v] = -1;
  }
  pred[root] = root; /* first_expand, bfs.hpp:498: bare id at level 0 */
  free(lr); free(pr);
}

/* bfs.hpp:2651-2940: the level loop's direction rule, replayed on levels.
 * TD -> BU when growing and nq > num_global_verts / alpha (:2801-2807);
 * BU -> TD (and stop growing) when unvisited < num_global_verts / beta
 * (:2809-2823).  Per level it reports the counts of the algorithmic-bytes
 * model: TD reads each frontier row; BU scans every unvisited vertex with
 * edges until its first neighbour visited before this level (row order is
 * ascending reordered id, first entry first, bfs.hpp:1839-1967). */
int orc_dobfs_schedule(const orc_graph* g, int64_t root, double alpha, double beta,
                       orc_level_stats* out, int max_levels) {
  const int64_t nlv = g->info[ORC_INFO_NUM_LOCAL_VERTS];
  const int64_t ngv = g->info[ORC_INFO_NUM_GLOBAL_VERTS];
  uint16_t* lr = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)(nlv ? nlv : 1));
  bfs_core(g, root, lr, NULL);
  int forward = 1, growing = 1, nl = 0;
  int64_t prev_nq = 0, visited = 1;
  for (int level = 1; nl < max_levels; ++level) {
    orc_level_stats s;
    memset(&s, 0, sizeof(s));
    s.direction = forward;
    for (int64_t v = 0; v < nlv; ++v) {
      uint64_t b = g->offsets[v], e = g->offsets[v + 1];
      if (forward) {
        if (lr[v] == level - 1) {
          s.frontier++;
          s.edges_examined += (int64_t)(e - b);
          s.edge_sectors += (int64_t)((e - b + 7) / 8);
        }
      } else if (e > b && lr[v] >= level) { /* unvisited with edges */
        s.scanned++;
        int64_t k = 0;
        for (uint64_t j = b; j < e; ++j) { ++k; if (lr[g->cols[j]] == level - 1) break; }
        s.edges_examined += k;
        s.edge_sectors += (k + 7) / 8;
      }
      if (lr[v] == level) s.discovered++;
    }
    out[nl++] = s;
    int64_t nq = s.discovered;
    visited += nq;
    if (nq == 0) break;
    int64_t unvisited = ngv - visited;
    if (growing && nq > prev_nq) {
      if (forward && nq > ngv / alpha) forward = 0;
    } else {
      if (!forward && unvisited < (int64_t)(ngv / beta)) { forward = 1; growing = 0; }
    }
    prev_nq = nq;
  }
  free(lr);
  return nl;
}

/* ------------------------------------------------------------------------- */
/* Validation (validate.hpp:506-995, one rank)                                */
/* ------------------------------------------------------------------------- */

static inline int64_t pred_of(int64_t e) { return (int64_t)((uint64_t)e << 16) >> 16; } /* :809 */
static inline uint16_t depth_of(int64_t e) { return (uint16_t)((e >> 48) & 0xFFFF); }   /* :813 */

int orc_validate(const orc_packed_edge* edges, int64_t m, int64_t nglobalverts, int64_t nlocalverts,
                 int64_t root, const int64_t* pred, int64_t* edge_visit_count,
                 orc_validate_report* rep) {
  orc_validate_report r;
  memset(&r, 0, sizeof(r));
  *edge_visit_count = 0;
  /* check_value_ranges, :822-839 */
  for (int64_t i = 0; i < nlocalverts; ++i) {
    int64_t p = pred_of(pred[i]);
    if (p < -1 || p >= nglobalverts) r.range_errors++;
  }
  /* :513-515 only reports a root outside [0, nglobalverts) (its own entry then
   * fails the range check); a root outside pred[] cannot be checked at all */
  if (root < 0 || root >= nlocalverts) { r.root_errors++; goto done; }
  if (r.range_errors) goto done;
  /* root is its own parent, :529-537 */
  if (pred_of(pred[root]) != root) { r.root_errors++; goto done; }
  /* nothing else is its own parent, :542-571 */
  for (int64_t i = 0; i < nlocalverts; ++i)
    if (i != root && pred_of(pred[i]) != -1 && pred_of(pred[i]) == i) r.self_parent_errors++;
  if (r.self_parent_errors) goto done;
  /* check_bfs_depth_map_using_predecessors, :920-995 */
  if (depth_of(pred[root]) != 0) r.depth_errors++;
  for (int64_t i = 0; i < nlocalverts; ++i) {
    int64_t p = pred_of(pred[i]);
    uint16_t d = depth_of(pred[i]);
    if (p == -1 && d != 0xFFFF) r.depth_errors++;
    else if (p != -1 && d == 0xFFFF) r.depth_errors++;
  }
  for (int64_t i = 0; i < nlocalverts; ++i) {
    if (i == root) continue;
    if (pred_of(pred[i]) == -1) continue;
    int64_t pp = pred[pred_of(pred[i])];
    if (depth_of(pp) == 0xFFFF) r.depth_errors++;
    if ((int)depth_of(pred[i]) != (int)depth_of(pp) + 1) r.depth_errors++;
  }
  if (r.depth_errors) goto done;
  {
    /* edge loop, :598-776 */
    unsigned char* valid = (unsigned char*)calloc((size_t)(nlocalverts ? nlocalverts : 1), 1);
    int64_t count = 0;
    for (int64_t i = 0; i < m; ++i) {
      int64_t src = orc_edge_v0(&edges[i]), tgt = orc_edge_v1(&edges[i]);
      int64_t ps = pred[src], pt = pred[tgt];
      int sd = depth_of(ps), td = depth_of(pt);
      if (sd != 0xFFFF && td == 0xFFFF) r.edge_errors++;
      else if (sd == 0xFFFF && td != 0xFFFF) r.edge_errors++;
      else if (sd - td < -1 || sd - td > 1) r.edge_errors++;
      else if (sd != 0xFFFF) ++count;
      if (pred_of(ps) == tgt) valid[src] = 1;
      if (pred_of(pt) == src) valid[tgt] = 1;
    }
    /* every reached non-root vertex has an input edge to its parent, :780-792 */
    for (int64_t i = 0; i < nlocalverts; ++i) {
      if (pred_of(pred[i]) == -1 || i == root) continue;
      if (!valid[i]) r.missing_parent_edge_errors++;
    }
    free(valid);
    *edge_visit_count = count;
  }
done:
  if (rep) *rep = r;
  return (r.range_errors + r.root_errors + r.self_parent_errors + r.depth_errors + r.edge_errors +
          r.missing_parent_edge_errors) == 0;
}

/* ------------------------------------------------------------------------- */
/* Statistics (logfile.h:19-44)                                               */
/* ------------------------------------------------------------------------- */
static int cmp_double(const void* a, const void* b) {
  double x = *(const double*)a, y = *(const double*)b;
  return (x < y) ? -1 : (x == y) ? 0 : 1;
}
void orc_statistics(const double* x, int n, double r[ORC_S_LAST]) {
  double t = 0;
  for (int i = 0; i < n; ++i) t += x[i];
  t /= n;
  r[ORC_S_MEAN] = t;
  t = 0;
  for (int i = 0; i < n; ++i) t += (x[i] - r[ORC_S_MEAN]) * (x[i] - r[ORC_S_MEAN]);
  t /= n - 1;
  r[ORC_S_STD] = sqrt(t);
  double* xx = (double*)malloc(sizeof(double) * (size_t)n);
  memcpy(xx, x, sizeof(double) * (size_t)n);
  qsort(xx, (size_t)n, sizeof(double), cmp_double);
  r[ORC_S_MIN] = xx[0];
  r[ORC_S_Q1] = (xx[(n - 1) / 4] + xx[n / 4]) * .5;
  r[ORC_S_MEDIAN] = (xx[(n - 1) / 2] + xx[n / 2]) * .5;
  r[ORC_S_Q3] = (xx[n - 1 - (n - 1) / 4] + xx[n - 1 - n / 4]) * .5;
  r[ORC_S_MAX] = xx[n - 1];
  free(xx);
}
