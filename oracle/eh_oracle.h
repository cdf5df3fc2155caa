/* CPU restatement of the EmptyHeaded storage-engine hot path.
 *
 * TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load this as the checker.  The product never links it.
 *
 * Parity is pinned: tests check this restatement against the reference's
 * own golden counts (test/graph/travis.py:29,70,212,253) and against the
 * reference engine itself compiled from its sources (oracle/_ref/eh_ref).
 *
 * All functions are plain C over caller-owned arrays.  Layout codes follow
 * storage_engine/include/utils/common.hpp:83-91:
 *   RANGE_BITSET = 0, UINTEGER = 1, BLOCK_BITSET = 3.
 */
#ifndef EH_ORACLE_H
#define EH_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- counter-based random numbers shared with the device generator ---- */
uint64_t eho_splitmix64(uint64_t x);
uint64_t eho_rand64(uint64_t seed, uint64_t index);

/* ---- raw edge samples ---- */
void eho_gen_er(uint64_t seed, uint32_t n, uint64_t m, uint32_t* u, uint32_t* v);
void eho_rmat_thresholds(double a, double b, double c, uint32_t t[3]);
void eho_gen_rmat(uint64_t seed, int scale, uint64_t m, const uint32_t t[3], uint32_t* u, uint32_t* v);
void eho_chunglu_cdf(uint32_t n, double gamma, uint64_t* cdf);
void eho_gen_chunglu(uint64_t seed, uint32_t n, uint64_t m, const uint64_t* cdf, uint32_t* u, uint32_t* v);

/* ---- preprocessing: symmetrise, drop self-loops, dedup, relabel by
 * (degree, id) ascending over nodes of degree > 0, then either keep
 * src < dst (symmetric == 0) or both directions (symmetric == 1).
 * Output is sorted by (src, dst).  Returns the number of output rows;
 * *nodes receives the number of relabelled nodes.  out arrays need
 * 2*m entries when symmetric, m otherwise. */
uint64_t eho_preprocess(const uint32_t* u, const uint32_t* v, uint64_t m, int symmetric,
                        uint32_t* out_src, uint32_t* out_dst, uint32_t* nodes);

/* ---- two-level trie from an encoded relation (Trie.cpp:380-510):
 * sort rows by (col0, col1), drop duplicate rows, head = distinct col0,
 * child set of head[i] = vals[off[i] .. off[i+1]).  head needs n entries,
 * off n+1, vals n.  Returns the number of distinct rows; *n_head is set. */
uint64_t eho_trie_build(const uint32_t* c0, const uint32_t* c1, uint64_t n, uint32_t* head, uint64_t* off,
                        uint32_t* vals, uint32_t* n_head);

/* ---- hybrid layout (layouts/hybrid.hpp:103-111, utils/common.hpp:60-66) ---- */
int eho_is_sparse(uint64_t length, uint64_t range);
int eho_hybrid_type(const uint32_t* data, uint64_t len);
/* bytes of the range_bitset encoding of a set (range_bitset.hpp:123-157) */
uint64_t eho_range_bitset_bytes(const uint32_t* data, uint64_t len);
/* writes [u64 start word][u64 words x W][u32 rank x W]; rank of an empty
 * word is the number of elements before it.  Returns bytes written. */
uint64_t eho_range_bitset_build(const uint32_t* data, uint64_t len, uint8_t* out);

/* ---- set intersection (ops/intersection/set.hpp:9-167): result elements
 * are the same for every layout pair; out may be NULL (count only). */
uint64_t eho_intersect(const uint32_t* a, uint64_t na, const uint32_t* b, uint64_t nb, uint32_t* out);

/* ---- generic-join COUNT queries over a two-level trie (CSR) ----
 * head[0..nh) sorted, child sets vals[off[i]..off[i+1]).  Counts are
 * accumulated modulo 2^64 (the reference accumulates in signed long). */
uint64_t eho_triangle(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals);
uint64_t eho_clique4(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals);
/* Triangle(a,b,c) tuples in (a,b,c) order; at most cap written, total returned */
uint64_t eho_triangle_list(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals, uint32_t* a,
                           uint32_t* b, uint32_t* c, uint64_t cap);
/* T(a) = number of ordered (b,c) closing a triangle at a; per head entry */
void eho_triangle_annot(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals,
                        uint64_t* T);
uint64_t eho_lollipop(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals);
uint64_t eho_barbell(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals);
/* equality-selection variants (travis.py:385-401, 472-487): only roots a
 * with (a,v) in the relation count; the barbell's second triangle starts
 * in N(v) */
uint64_t eho_clique4_sel(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals, uint32_t v);
uint64_t eho_barbell_sel(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals, uint32_t v);
/* per-head triangle contribution sum_{b in N(a)} |N(a) ∩ N(b)| */
void eho_triangle_per_vertex(const uint32_t* head, uint32_t nh, const uint64_t* off, const uint32_t* vals,
                             uint64_t* per);

/* ---- small fp32 MLP restated in double, for gradient checks ---- */
/* layer sizes d0 -> d1 -> ... -> dL, ReLU between layers, linear output.
 * W[l] row-major [d_{l+1} x d_l], b[l] [d_{l+1}], packed one after another
 * in params (W0,b0,W1,b1,...).  Loss = mean over batch of 0.5*(y_hat-y)^2
 * summed over outputs.  Writes the loss and, if grad != NULL, dLoss/dparams. */
double eho_mlp_loss_grad(int nlayers, const int* dims, const double* params, const double* x, const double* y,
                         int batch, double* grad);

#ifdef __cplusplus
}
#endif
#endif
