/* CPU restatement of the EmptyHeaded storage-engine hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see eh_oracle.h).  Parity pinned against the
 * reference's golden counts and against the reference engine compiled from
 * its own sources.  Each function names the reference code it restates.
 */
#define _GNU_SOURCE
#include "eh_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <pthread.h>
#include <unistd.h>

/* ------------------------------------------------- tiny parallel for
 * Dynamic chunking over [0, n) with pthreads (the reference's par::for_range
 * with a block size, storage_engine/src/utils/parallel.cpp:42-79).  Thread
 * count: $EHO_THREADS, else the online CPU count. */
typedef void (*eho_body)(void* ctx, uint64_t begin, uint64_t end, int tid);
typedef struct {
  eho_body body;
  void* ctx;
  uint64_t n, chunk;
  uint64_t next;
  int tid;
} eho_job;
typedef struct { eho_job* job; int tid; } eho_arg;
static void* eho_worker(void* p) {
  eho_arg* a = (eho_arg*)p;
  eho_job* j = a->job;
  for (;;) {
    uint64_t b = __atomic_fetch_add(&j->next, j->chunk, __ATOMIC_RELAXED);
    if (b >= j->n) break;
    uint64_t e = b + j->chunk < j->n ? b + j->chunk : j->n;
    j->body(j->ctx, b, e, a->tid);
  }
  return NULL;
}
static int eho_threads(void) {
  const char* e = getenv("EHO_THREADS");
  if (e && atoi(e) > 0) return atoi(e);
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)(n > 256 ? 256 : n) : 1;
}
static void eho_parallel(uint64_t n, uint64_t chunk, eho_body body, void* ctx) {
  int nt = eho_threads();
  if (chunk == 0) chunk = 1;
  if ((uint64_t)nt > (n + chunk - 1) / chunk) nt = (int)((n + chunk - 1) / chunk);
  if (nt <= 1) { if (n) body(ctx, 0, n, 0); return; }
  eho_job job = {body, ctx, n, chunk, 0, 0};
  pthread_t th[256];
  eho_arg args[256];
  for (int t = 0; t < nt; t++) { args[t].job = &job; args[t].tid = t; }
  for (int t = 1; t < nt; t++) pthread_create(&th[t], NULL, eho_worker, &args[t]);
  eho_worker(&args[0]);
  for (int t = 1; t < nt; t++) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------ rng
 * splitmix64 (Steele, Lea, Flood 2014), used as a counter-based generator:
 * every random draw is a pure function of (seed, index), so the device
 * generator reproduces the same stream in any order. */
uint64_t eho_splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
uint64_t eho_rand64(uint64_t seed, uint64_t index) {
  return eho_splitmix64(eho_splitmix64(seed) ^ eho_splitmix64(index));
}

/* uniform integer in [0, n) from 32 random bits (multiply-shift) */
static inline uint32_t mulshift(uint32_t r, uint32_t n) { return (uint32_t)(((uint64_t)r * n) >> 32); }

/* Erdős–Rényi samples: pair i = (uniform, uniform) from one 64-bit draw */
typedef struct { uint64_t seed; uint32_t n; uint32_t* u; uint32_t* v; const uint32_t* t; int scale;
                 const uint64_t* cdf; } gen_ctx;
static void er_body(void* p, uint64_t b, uint64_t e, int tid) {
  gen_ctx* c = (gen_ctx*)p;
  (void)tid;
  for (uint64_t i = b; i < e; i++) {
    uint64_t h = eho_rand64(c->seed, i);
    c->u[i] = mulshift((uint32_t)h, c->n);
    c->v[i] = mulshift((uint32_t)(h >> 32), c->n);
  }
}
void eho_gen_er(uint64_t seed, uint32_t n, uint64_t m, uint32_t* u, uint32_t* v) {
  gen_ctx c = {seed, n, u, v, NULL, 0, NULL};
  eho_parallel(m, 1 << 16, er_body, &c);
}

/* R-MAT (Chakrabarti, Zhan, Faloutsos 2004): per level choose a quadrant
 * with probabilities a, b, c, d.  Thresholds are 32-bit fixed point so host
 * and device make identical choices. */
void eho_rmat_thresholds(double a, double b, double c, uint32_t t[3]) {
  const double s = 4294967296.0;
  t[0] = (uint32_t)floor(a * s);
  t[1] = (uint32_t)floor((a + b) * s);
  t[2] = (uint32_t)floor((a + b + c) * s);
}
static void rmat_body(void* p, uint64_t b, uint64_t e, int tid) {
  gen_ctx* c = (gen_ctx*)p;
  (void)tid;
  const int scale = c->scale;
  const uint32_t* t = c->t;
  const uint64_t seed = c->seed;
  uint32_t* u = c->u;
  uint32_t* v = c->v;
  const int words = (scale + 1) / 2;
  for (uint64_t i = b; i < e; i++) {
    uint32_t x = 0, y = 0;
    for (int w = 0; w < words; w++) {
      uint64_t h = eho_rand64(seed, (i << 5) | (uint64_t)w);
      for (int half = 0; half < 2; half++) {
        const int level = 2 * w + half;
        if (level >= scale) break;
        const uint32_t r = half ? (uint32_t)(h >> 32) : (uint32_t)h;
        const uint32_t bit = 1u << (scale - 1 - level);
        if (r < t[0]) {
        } else if (r < t[1]) {
          y |= bit;
        } else if (r < t[2]) {
          x |= bit;
        } else {
          x |= bit;
          y |= bit;
        }
      }
    }
    u[i] = x;
    v[i] = y;
  }
}
void eho_gen_rmat(uint64_t seed, int scale, uint64_t m, const uint32_t t[3], uint32_t* u, uint32_t* v) {
  gen_ctx c = {seed, 0, u, v, t, scale, NULL};
  eho_parallel(m, 1 << 16, rmat_body, &c);
}

/* Chung–Lu: node i has weight (i+1)^(-1/(gamma-1)); endpoints are drawn
 * independently proportional to weight through a 63-bit fixed-point CDF
 * (cdf[n-1] == 2^63). */
void eho_chunglu_cdf(uint32_t n, double gamma, uint64_t* cdf) {
  const double e = -1.0 / (gamma - 1.0);
  double total = 0.0;
  for (uint32_t i = 0; i < n; i++) total += pow((double)i + 1.0, e);
  double acc = 0.0;
  const double scale = 9223372036854775808.0 / total;
  for (uint32_t i = 0; i < n; i++) {
    acc += pow((double)i + 1.0, e);
    double c = acc * scale;
    cdf[i] = c >= 9223372036854775808.0 ? (1ull << 63) : (uint64_t)c;
  }
  cdf[n - 1] = 1ull << 63;
}
static inline uint32_t cdf_pick(const uint64_t* cdf, uint32_t n, uint64_t r63) {
  uint32_t lo = 0, hi = n - 1; /* first i with cdf[i] > r63 */
  while (lo < hi) {
    uint32_t mid = lo + (hi - lo) / 2;
    if (cdf[mid] > r63) hi = mid; else lo = mid + 1;
  }
  return lo;
}
static void chunglu_body(void* p, uint64_t b, uint64_t e, int tid) {
  gen_ctx* c = (gen_ctx*)p;
  (void)tid;
  for (uint64_t i = b; i < e; i++) {
    c->u[i] = cdf_pick(c->cdf, c->n, eho_rand64(c->seed, 2 * i) >> 1);
    c->v[i] = cdf_pick(c->cdf, c->n, eho_rand64(c->seed, 2 * i + 1) >> 1);
  }
}
void eho_gen_chunglu(uint64_t seed, uint32_t n, uint64_t m, const uint64_t* cdf, uint32_t* u, uint32_t* v) {
  gen_ctx c = {seed, n, u, v, NULL, 0, cdf};
  eho_parallel(m, 1 << 16, chunglu_body, &c);
}

/* ------------------------------------------------------------ radix sort */
static void radix_sort_u64(uint64_t* a, uint64_t n, int bits) {
  if (n < 2) return;
  uint64_t* tmp = (uint64_t*)malloc(n * sizeof(uint64_t));
  uint64_t *src = a, *dst = tmp;
  for (int shift = 0; shift < bits; shift += 11) {
    uint64_t cnt[2048];
    memset(cnt, 0, sizeof cnt);
    for (uint64_t i = 0; i < n; i++) cnt[(src[i] >> shift) & 2047]++;
    uint64_t s = 0;
    for (int d = 0; d < 2048; d++) { uint64_t c = cnt[d]; cnt[d] = s; s += c; }
    for (uint64_t i = 0; i < n; i++) dst[cnt[(src[i] >> shift) & 2047]++] = src[i];
    uint64_t* t = src; src = dst; dst = t;
  }
  if (src != a) memcpy(a, src, n * sizeof(uint64_t));
  free(tmp);
}
static int bits_for(uint64_t maxv) {
  int b = 1;
  while (b < 64 && (maxv >> b)) b++;
  return b;
}
static uint64_t sort_unique(uint64_t* k, uint64_t n) {
  uint64_t mx = 0;
  for (uint64_t i = 0; i < n; i++) if (k[i] > mx) mx = k[i];
  radix_sort_u64(k, n, bits_for(mx));
  uint64_t w = 0;
  for (uint64_t i = 0; i < n; i++) if (i == 0 || k[i] != k[i - 1]) k[w++] = k[i];
  return w;
}

/* --------------------------------------------------------- preprocessing */
uint64_t eho_preprocess(const uint32_t* u, const uint32_t* v, uint64_t m, int symmetric, uint32_t* out_src,
                        uint32_t* out_dst, uint32_t* nodes) {
  uint64_t* k = (uint64_t*)malloc((m ? m : 1) * sizeof(uint64_t));
  uint64_t e = 0;
  uint32_t maxid = 0;
  for (uint64_t i = 0; i < m; i++) {
    uint32_t a = u[i], b = v[i];
    if (a == b) continue;
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    if (hi > maxid) maxid = hi;
    k[e++] = ((uint64_t)lo << 32) | hi;
  }
  e = sort_unique(k, e);
  /* degree of every endpoint in the simple undirected graph */
  uint64_t nid = (uint64_t)maxid + 1;
  uint32_t* deg = (uint32_t*)calloc(nid, sizeof(uint32_t));
  for (uint64_t i = 0; i < e; i++) { deg[k[i] >> 32]++; deg[(uint32_t)k[i]]++; }
  /* relabel nodes of degree > 0 by (degree, id) ascending */
  uint64_t* order = (uint64_t*)malloc(nid * sizeof(uint64_t));
  uint64_t nn = 0;
  for (uint64_t x = 0; x < nid; x++) if (deg[x]) order[nn++] = ((uint64_t)deg[x] << 32) | x;
  radix_sort_u64(order, nn, 64);
  uint32_t* newid = deg; /* reuse: old id -> new id */
  for (uint64_t r = 0; r < nn; r++) newid[(uint32_t)order[r]] = (uint32_t)r;
  free(order);
  uint64_t rows = 0;
  uint64_t* o = (uint64_t*)malloc((symmetric ? 2 * e : e) * sizeof(uint64_t) + 8);
  for (uint64_t i = 0; i < e; i++) {
    uint32_t a = newid[k[i] >> 32], b = newid[(uint32_t)k[i]];
    uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    o[rows++] = ((uint64_t)lo << 32) | hi;
    if (symmetric) o[rows++] = ((uint64_t)hi << 32) | lo;
  }
  radix_sort_u64(o, rows, 64);
  for (uint64_t i = 0; i < rows; i++) { out_src[i] = (uint32_t)(o[i] >> 32); out_dst[i] = (uint32_t)o[i]; }
  *nodes = (uint32_t)nn;
  free(o);
  free(deg);
  free(k);
  return rows;
}

/* ------------------------------------------------------------- trie build
 * Trie.cpp:380-510 sorts row indices lexicographically (SortColumns
 * :173-186), then produce_ranges (:192-224) finds distinct head values and
 * encode_tail (:291-302) drops repeated child values inside each run. */
uint64_t eho_trie_build(const uint32_t* c0, const uint32_t* c1, uint64_t n, uint32_t* head, uint64_t* off,
                        uint32_t* vals, uint32_t* n_head) {
  uint64_t* k = (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < n; i++) k[i] = ((uint64_t)c0[i] << 32) | c1[i];
  uint64_t r = sort_unique(k, n);
  uint32_t nh = 0;
  for (uint64_t i = 0; i < r; i++) {
    uint32_t s = (uint32_t)(k[i] >> 32);
    if (i == 0 || s != (uint32_t)(k[i - 1] >> 32)) { head[nh] = s; off[nh] = i; nh++; }
    vals[i] = (uint32_t)k[i];
  }
  off[nh] = r;
  *n_head = nh;
  free(k);
  return r;
}

/* ----------------------------------------------------------------- layout */
int eho_is_sparse(uint64_t length, uint64_t range) {
  /* common::is_sparse, utils/common.hpp:60-66: bitset_length = 2,
     bitset_req = 128.0 */
  if (length > 2) return ((double)range / (double)length) > 128.0;
  return 1;
}
int eho_hybrid_type(const uint32_t* data, uint64_t len) {
  /* hybrid::get_type, layouts/hybrid.hpp:103-111: range = last - first */
  const uint64_t range = len > 1 ? (uint64_t)(data[len - 1] - data[0]) : 0;
  return eho_is_sparse(len, range) ? 1 /*UINTEGER*/ : 0 /*RANGE_BITSET*/;
}
uint64_t eho_range_bitset_bytes(const uint32_t* data, uint64_t len) {
  if (!len) return 0;
  const uint64_t words = (data[len - 1] >> 6) - (data[0] >> 6) + 1;
  return 8 + words * 12;
}
uint64_t eho_range_bitset_build(const uint32_t* data, uint64_t len, uint8_t* out) {
  /* range_bitset::build, layouts/range_bitset.hpp:123-157 */
  if (!len) return 0;
  const uint64_t start = data[0] >> 6;
  const uint64_t words = (data[len - 1] >> 6) - start + 1;
  uint64_t* w = (uint64_t*)(out + 8);
  uint32_t* rank = (uint32_t*)(w + words);
  memcpy(out, &start, 8);
  memset(w, 0, words * 8);
  for (uint64_t i = 0; i < len; i++) w[(data[i] >> 6) - start] |= 1ull << (data[i] & 63);
  uint32_t c = 0;
  for (uint64_t j = 0; j < words; j++) { rank[j] = c; c += (uint32_t)__builtin_popcountll(w[j]); }
  return 8 + words * 12;
}

/* ----------------------------------------------------------- intersection
 * The element set of A ∩ B does not depend on the layouts the reference
 * picked (set.hpp:9-167 dispatches on layout pairs; uinteger.hpp:1209-1261,
 * hetero.hpp:29-60 and bitset.hpp:619-661 all yield the common elements in
 * increasing order).  Linear merge. */
uint64_t eho_intersect(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb, uint32_t* out) {
  uint64_t i = 0, j = 0, c = 0;
  while (i < na && j < nb) {
    if (a[i] < b[j]) i++;
    else if (a[i] > b[j]) j++;
    else {
      if (out) out[c] = a[i];
      c++; i++; j++;
    }
  }
  return c;
}

/* index of value x in head, or -1 (TrieBlock::get_next_block, TrieBlock.hpp:86-111) */
static inline int64_t head_find(const uint32_t* head, uint32_t nh, uint32_t x) {
  uint32_t lo = 0, hi = nh;
  while (lo < hi) {
    uint32_t mid = lo + (hi - lo) / 2;
    if (head[mid] < x) lo = mid + 1; else hi = mid;
  }
  return (lo < nh && head[lo] == x) ? (int64_t)lo : -1;
}

/* ---------------------------------------------------------------- queries
 * TriangleAgg plan (order [a,b,c], QueryPlannerTest.scala:78-96) as the
 * generated loop nest runs it (EHGenerator.scala:273-480):
 *   a ∈ head ∩ head;  b ∈ N(a) ∩ head;  count_c = |N(b) ∩ N(a)|. */
typedef struct { const uint32_t* head; uint32_t nh; const uint64_t* off; const uint32_t* vals; uint64_t* per;
                 const uint64_t* T; uint64_t partial[256 * 8]; } q_ctx;
static void tri_body(void* p, uint64_t b, uint64_t e, int tid) {
  q_ctx* c = (q_ctx*)p;
  (void)tid;
  const uint32_t* head = c->head; const uint32_t nh = c->nh; const uint64_t* off = c->off;
  const uint32_t* vals = c->vals; uint64_t* per = c->per;
  for (uint64_t ia = b; ia < e; ia++) {
    const uint32_t* na = vals + off[ia];
    const uint64_t da = off[ia + 1] - off[ia];
    uint64_t acc = 0;
    for (uint64_t j = 0; j < da; j++) {
      int64_t ib = head_find(head, nh, na[j]);
      if (ib < 0) continue;
      acc += eho_intersect(vals + off[ib], off[ib + 1] - off[ib], na, da, NULL);
    }
    per[ia] = acc;
  }
}
void eho_triangle_per_vertex(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals,
                             uint64_t* per) {
  q_ctx* c = (q_ctx*)calloc(1, sizeof(q_ctx));
  c->head = head; c->nh = nh; c->off = off; c->vals = vals; c->per = per;
  eho_parallel(nh, 64, tri_body, c);
  free(c);
}
uint64_t eho_triangle(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals) {
  uint64_t* per = (uint64_t*)malloc((nh ? nh : 1) * sizeof(uint64_t));
  eho_triangle_per_vertex(head, nh, off, vals, per);
  uint64_t t = 0;
  for (uint32_t i = 0; i < nh; i++) t += per[i];
  free(per);
  return t;
}

/* Triangle(a,b,c) materialized: the generated loop nest visits a in head
 * order, b in N(a) ∩ head in order, c in N(a) ∩ N(b) in order, so the
 * tuples come out sorted by (a,b,c) (the output trie's Trie::foreach
 * order).  Writes at most cap tuples; returns the total. */
uint64_t eho_triangle_list(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals, uint32_t* a,
                           uint32_t* b, uint32_t* c, uint64_t cap) {
  uint64_t n = 0;
  uint32_t* tmp = NULL;
  uint64_t tcap = 0;
  for (uint32_t ia = 0; ia < nh; ia++) {
    const uint32_t* na = vals + off[ia];
    const uint64_t da = off[ia + 1] - off[ia];
    if (da > tcap) { free(tmp); tcap = da; tmp = (uint32_t*)malloc(tcap * sizeof(uint32_t)); }
    for (uint64_t j = 0; j < da; j++) {
      int64_t ib = head_find(head, nh, na[j]);
      if (ib < 0) continue;
      const uint64_t k = eho_intersect(vals + off[ib], off[ib + 1] - off[ib], na, da, tmp);
      for (uint64_t q = 0; q < k; q++, n++)
        if (n < cap) { a[n] = head[ia]; b[n] = na[j]; c[n] = tmp[q]; }
    }
  }
  free(tmp);
  return n;
}

/* FliqueAgg plan (order [a,b,c,d]): N-way intersections chain pairwise,
 * smallest input first (TrieBuilder.cpp:276-348).  Here: S = N(a) ∩ N(b)
 * restricted to head, then d ∈ S ∩ N(c). */
static void c4_body(void* p, uint64_t b, uint64_t e, int tid) {
  q_ctx* c = (q_ctx*)p;
  const uint32_t* head = c->head; const uint32_t nh = c->nh; const uint64_t* off = c->off;
  const uint32_t* vals = c->vals;
  uint64_t total = 0;
  uint32_t* s = NULL;
  uint64_t cap = 0;
  for (uint64_t ia = b; ia < e; ia++) {
    const uint32_t* na = vals + off[ia];
    const uint64_t da = off[ia + 1] - off[ia];
    if (da > cap) { free(s); cap = da; s = (uint32_t*)malloc(cap * sizeof(uint32_t)); }
    for (uint64_t j = 0; j < da; j++) {
      int64_t ib = head_find(head, nh, na[j]);
      if (ib < 0) continue;
      const uint64_t ns = eho_intersect(vals + off[ib], off[ib + 1] - off[ib], na, da, s);
      for (uint64_t q = 0; q < ns; q++) {
        int64_t ic = head_find(head, nh, s[q]);
        if (ic < 0) continue;
        total += eho_intersect(vals + off[ic], off[ic + 1] - off[ic], s, ns, NULL);
      }
    }
  }
  free(s);
  c->partial[tid * 8] += total;
}
uint64_t eho_clique4(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals) {
  q_ctx* c = (q_ctx*)calloc(1, sizeof(q_ctx));
  c->head = head; c->nh = nh; c->off = off; c->vals = vals;
  eho_parallel(nh, 16, c4_body, c);
  uint64_t t = 0;
  for (int i = 0; i < 256; i++) t += c->partial[i * 8];
  free(c);
  return t;
}

/* ---- equality selections (EHGenerator.scala:657-701) ----
 * A selected attribute x = v with one accessor is answered at the head of
 * its relation: get_next_block(key(v)) (ParTrieIterator::get_next_block,
 * TrieIterator.cpp:72-78) leaves the set of partners of v.  For Edge(a,x)
 * in order [x,a] that set is {a : (a,v) ∈ Edge}: the head entries whose
 * child set holds v.  mask[i] = 1 for those entries. */
static void select_in(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals, uint32_t v,
                      uint8_t* mask) {
  (void)head;
  for (uint32_t i = 0; i < nh; i++) {
    uint64_t lo = off[i], hi = off[i + 1];
    while (lo < hi) {
      const uint64_t mid = lo + (hi - lo) / 2;
      if (vals[mid] < v) lo = mid + 1; else hi = mid;
    }
    mask[i] = (lo < off[i + 1] && vals[lo] == v) ? 1 : 0;
  }
}

/* FliqueSelAgg(;z) :- 4-clique(a,b,c,d), Edge(a,x), x=v, COUNT(*)
 * (travis.py:385-401; plan QueryPlannerTest.scala:230-259): bag_1(a;z)
 * holds z(a) = 1 for every a with (a,v) ∈ Edge, and the 4-clique root bag
 * joins it at a, so only roots a of that set count. */
uint64_t eho_clique4_sel(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals, uint32_t v) {
  uint8_t* mask = (uint8_t*)malloc(nh ? nh : 1);
  select_in(head, nh, off, vals, v, mask);
  /* the FliqueAgg loop nest of eho_clique4, over the selected roots only */
  uint64_t total = 0;
  uint32_t* s = NULL;
  uint64_t cap = 0;
  for (uint32_t ia = 0; ia < nh; ia++) {
    if (!mask[ia]) continue;
    const uint32_t* na = vals + off[ia];
    const uint64_t da = off[ia + 1] - off[ia];
    if (da > cap) { free(s); cap = da; s = (uint32_t*)malloc(cap * sizeof(uint32_t)); }
    for (uint64_t j = 0; j < da; j++) {
      int64_t ib = head_find(head, nh, na[j]);
      if (ib < 0) continue;
      const uint64_t ns = eho_intersect(vals + off[ib], off[ib + 1] - off[ib], na, da, s);
      for (uint64_t q = 0; q < ns; q++) {
        int64_t ic = head_find(head, nh, s[q]);
        if (ic < 0) continue;
        total += eho_intersect(vals + off[ic], off[ic + 1] - off[ic], s, ns, NULL);
      }
    }
  }
  free(s);
  free(mask);
  return total;
}

/* BarbellSelAgg(;w) :- triangle(a,b,c), Edge(a,p), Edge(p,x),
 * triangle(x,y,z), p=v, COUNT(*) (travis.py:472-487; plan
 * QueryPlannerTest.scala:262-304): bag_1_p_a marks {a : (a,v) ∈ Edge},
 * bag_2_p_x marks N(v); the x,y,z bag reduces to the scalar
 * sum_{x ∈ N(v)} T(x) and the root bag to sum_{a : (a,v)} T(a) times it. */
uint64_t eho_barbell_sel(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals, uint32_t v) {
  uint64_t* T = (uint64_t*)malloc((nh ? nh : 1) * sizeof(uint64_t));
  uint8_t* mask = (uint8_t*)malloc(nh ? nh : 1);
  eho_triangle_per_vertex(head, nh, off, vals, T);
  select_in(head, nh, off, vals, v, mask);
  uint64_t s_in = 0, s_out = 0;
  for (uint32_t i = 0; i < nh; i++)
    if (mask[i]) s_in += T[i];
  const int64_t ip = head_find(head, nh, v);
  if (ip >= 0)
    for (uint64_t j = off[ip]; j < off[ip + 1]; j++) {
      const int64_t ix = head_find(head, nh, vals[j]);
      if (ix >= 0) s_out += T[ix];
    }
  free(mask);
  free(T);
  return s_in * s_out;
}

/* bag_1(a;z) of lollipop/barbell (QueryPlannerTest.scala:199-212):
 * T(a) = sum over b ∈ N(a) ∩ head of |N(a) ∩ N(b)|, annotated per a
 * (TrieBuilder::set_annotation, TrieBuilder.cpp:428-446). */
void eho_triangle_annot(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals,
                        uint64_t* T) {
  eho_triangle_per_vertex(head, nh, off, vals, T);
}
/* LollipopAgg root bag, order [a,d]: sum_a T(a) * |N(a)| */
uint64_t eho_lollipop(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals) {
  uint64_t* T = (uint64_t*)malloc((nh ? nh : 1) * sizeof(uint64_t));
  eho_triangle_annot(head, nh, off, vals, T);
  uint64_t t = 0;
  for (uint32_t i = 0; i < nh; i++) t += T[i] * (off[i + 1] - off[i]);
  free(T);
  return t;
}
/* BarbellAgg root bag, order [a,x]: sum over (a,x) in Edge of T(a) * T(x),
 * T read through TrieIterator::get_annotation (TrieIterator.cpp:45-59). */
static void barbell_body(void* p, uint64_t b, uint64_t e, int tid) {
  q_ctx* c = (q_ctx*)p;
  uint64_t t = 0;
  for (uint64_t ia = b; ia < e; ia++) {
    uint64_t s = 0;
    for (uint64_t j = c->off[ia]; j < c->off[ia + 1]; j++) {
      int64_t ix = head_find(c->head, c->nh, c->vals[j]);
      if (ix >= 0) s += c->T[ix];
    }
    t += c->T[ia] * s;
  }
  c->partial[tid * 8] += t;
}
uint64_t eho_barbell(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals) {
  uint64_t* T = (uint64_t*)malloc((nh ? nh : 1) * sizeof(uint64_t));
  eho_triangle_annot(head, nh, off, vals, T);
  q_ctx* c = (q_ctx*)calloc(1, sizeof(q_ctx));
  c->head = head; c->nh = nh; c->off = off; c->vals = vals; c->T = T;
  eho_parallel(nh, 64, barbell_body, c);
  uint64_t t = 0;
  for (int i = 0; i < 256; i++) t += c->partial[i * 8];
  free(c);
  free(T);
  return t;
}

/* ------------------------------------------------------------------- mlp */
double eho_mlp_loss_grad(int nlayers, const int* dims, const double* params, const double* x, const double* y,
                         int batch, double* grad) {
  int maxd = 0, total_act = 0;
  for (int l = 0; l <= nlayers; l++) { if (dims[l] > maxd) maxd = dims[l]; total_act += dims[l]; }
  int np = 0;
  for (int l = 0; l < nlayers; l++) np += dims[l + 1] * dims[l] + dims[l + 1];
  if (grad) memset(grad, 0, (size_t)np * sizeof(double));
  double* act = (double*)malloc((size_t)total_act * sizeof(double)); /* post-activation per layer */
  double* pre = (double*)malloc((size_t)total_act * sizeof(double));
  double* dcur = (double*)malloc((size_t)maxd * sizeof(double));
  double* dprev = (double*)malloc((size_t)maxd * sizeof(double));
  double loss = 0.0;
  for (int s = 0; s < batch; s++) {
    int ao = 0, po = 0;
    for (int i = 0; i < dims[0]; i++) act[i] = pre[i] = x[(size_t)s * dims[0] + i];
    for (int l = 0; l < nlayers; l++) {
      const double* W = params + po;
      const double* b = W + dims[l + 1] * dims[l];
      const int din = dims[l], dout = dims[l + 1];
      for (int o = 0; o < dout; o++) {
        double z = b[o];
        for (int i = 0; i < din; i++) z += W[o * din + i] * act[ao + i];
        pre[ao + din + o] = z;
        act[ao + din + o] = (l + 1 < nlayers && z < 0.0) ? 0.0 : z;
      }
      ao += din;
      po += dout * din + dout;
    }
    const int dL = dims[nlayers];
    for (int o = 0; o < dL; o++) {
      const double d = act[ao + o] - y[(size_t)s * dL + o];
      loss += 0.5 * d * d;
      dcur[o] = d / batch;
    }
    if (!grad) continue;
    for (int l = nlayers - 1; l >= 0; l--) {
      const int din = dims[l], dout = dims[l + 1];
      po -= dout * din + dout;
      ao -= din;
      const double* W = params + po;
      double* gW = grad + po;
      double* gb = gW + dout * din;
      for (int o = 0; o < dout; o++) {
        gb[o] += dcur[o];
        for (int i = 0; i < din; i++) gW[o * din + i] += dcur[o] * act[ao + i];
      }
      if (l > 0) {
        for (int i = 0; i < din; i++) {
          double g = 0.0;
          for (int o = 0; o < dout; o++) g += W[o * din + i] * dcur[o];
          dprev[i] = pre[ao + i] < 0.0 ? 0.0 : g;
        }
        for (int i = 0; i < din; i++) dcur[i] = dprev[i];
      }
    }
  }
  free(act); free(pre); free(dcur); free(dprev);
  return loss / batch;
}
