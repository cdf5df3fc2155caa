// Internal types shared by the engine's translation units.
#pragma once
#include <vector>

#include "eh_common.cuh"

// ------------------------------------------------------------------ context
struct eh_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // host-to-device copies overlapped with work on `stream`
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  // per-item timing records of the last recorded query (8 floats each)
  std::vector<float> timing_records;
  // the annotated triangle pass's per-head counters: a cudaMalloc'd buffer of
  // annot_cap entries kept across queries (see annot_buffer in eh_query.cu)
  unsigned long long* annot = nullptr;
  size_t annot_cap = 0;
};

namespace eh {

enum { DIR_GENERAL = 0, DIR_UP = 1, DIR_DOWN = 2, DIR_SYM = 3 };

// Per level-1 set side data for the bitset layouts.
//  RANGE_BITSET: off = first word in the word pool, start = first word
//                index (value >> 6 of the smallest element), n = words.
//  BLOCK_BITSET: off = first block in the block pools, n = blocks.
struct SetAux {
  uint64_t off;
  uint32_t start;
  uint32_t n;
};

// Raw device view of a two-level trie, passed to kernels by value.
struct TrieView {
  uint32_t n_head;
  uint32_t n_nodes;
  uint64_t rows;
  const uint32_t* head;       // [n_head] sorted first-column values
  const int32_t* head_index;  // [n_nodes] value -> head position, -1 if absent
  const uint64_t* off;        // [n_head + 1] child set i = vals[off[i] .. off[i+1])
  const uint32_t* vals;       // [rows] sorted within each set
  const uint8_t* layout;      // [n_head + 1] EH_LAYOUT_*; entry n_head is the head set
  const SetAux* aux;          // [n_head + 1]
  const uint64_t* bs_words;   // range-bitset words
  const uint32_t* bs_rank;    // per-word count of elements before the word
  const uint32_t* bb_id;      // block-bitset block ids (value >> 8)
  const uint32_t* bb_rank;    // index of the block's first element in its set
  const uint64_t* bb_words;   // 4 words per block
};

}  // namespace eh

struct eh_trie {
  eh_context* ctx = nullptr;
  uint64_t rows = 0;
  uint32_t n_head = 0, n_nodes = 0;
  eh::DevBuf<uint32_t> head;
  eh::DevBuf<int32_t> head_index;
  eh::DevBuf<uint64_t> off;
  eh::DevBuf<uint32_t> vals;
  eh::DevBuf<uint8_t> layout;
  eh::DevBuf<eh::SetAux> aux;
  eh::DevBuf<uint64_t> bs_words;
  eh::DevBuf<uint32_t> bs_rank;
  eh::DevBuf<uint32_t> bb_id;
  eh::DevBuf<uint32_t> bb_rank;
  eh::DevBuf<uint64_t> bb_words;
  // per head entry: sum over children v of d+(v) (wedge count), computed
  // once per trie for planning the generic-join loops
  eh::DevBuf<uint64_t> wedges;
  uint64_t total_wedges = 0;
  uint64_t sum_sq_deg = 0;  // sum over head entries of |N(a)|^2
  // Direction of the relation, decided at build: every row goes up
  // (col0 < col1), every row goes down, the relation is symmetric, or none.
  int dir = 0;
  // Reverse level (the relation in ordering [1,0], restricted to what the
  // triangle plans read): for head entry b, entries rev_off[b]..rev_off[b+1]
  // list rows a->b; entry k gives the range [rev_lo[k], rev_hi[k]) of vals
  // (inside N(a)) that can still meet N(b).  rev_work[k] = rev_hi - rev_lo.
  eh::DevBuf<uint64_t> rev_off;
  eh::DevBuf<uint32_t> rev_lo, rev_hi;
  eh::DevBuf<uint32_t> rev_src;   // head position of a for entry k
  eh::DevBuf<uint64_t> rev_wpre;  // exclusive prefix of entry work, rev_entries + 1 values
  uint64_t rev_entries = 0, rev_pairs = 0;
  // With learned layouts: the cost model's predicted SM cycles of every
  // staged set's work (0 for sets never staged), and their sum over the
  // probes; the planner cuts work items by predicted cycles instead of
  // probes, so items are uniform in time.
  eh::DevBuf<float> work_pred;
  double pred_per_probe = 0;
  eh_trie_info info{};

  eh::TrieView view() const {
    eh::TrieView v;
    v.n_head = n_head;
    v.n_nodes = n_nodes;
    v.rows = rows;
    v.head = head.p;
    v.head_index = head_index.p;
    v.off = off.p;
    v.vals = vals.p;
    v.layout = layout.p;
    v.aux = aux.p;
    v.bs_words = bs_words.p;
    v.bs_rank = bs_rank.p;
    v.bb_id = bb_id.p;
    v.bb_rank = bb_rank.p;
    v.bb_words = bb_words.p;
    return v;
  }
};

// Small fp32 MLP (eh_model.cu): widths dims[0..n_layers], parameters packed
// W0,b0,W1,b1,... with W row-major [d_{l+1} x d_l].
struct eh_model {
  eh_context* ctx = nullptr;
  int n_layers = 0;
  std::vector<int> dims;
  std::vector<size_t> w_off;  // offset of W_l in params; b_l follows W_l
  size_t n_params = 0;
  int max_dim = 0;
  eh::DevBuf<float> params, grads;
};

namespace eh {

// graph input pipeline (eh_graph.cu)
void gen_er(cudaStream_t s, uint64_t seed, uint32_t n, uint64_t m, uint32_t* u, uint32_t* v);
void gen_rmat(cudaStream_t s, uint64_t seed, int scale, uint64_t m, double a, double b, double c, uint32_t* u,
              uint32_t* v);
void gen_chunglu(cudaStream_t s, uint64_t seed, uint32_t n, uint64_t m, double gamma, uint32_t* u, uint32_t* v);
void preprocess(cudaStream_t s, const uint32_t* u, const uint32_t* v, uint64_t m, int symmetric, DevBuf<uint32_t>& src,
                DevBuf<uint32_t>& dst, uint64_t* rows, uint32_t* nodes);

// trie (eh_trie.cu)
void trie_build(eh_context* ctx, const uint32_t* col0, const uint32_t* col1, uint64_t n, const eh_layout_config* cfg,
                eh_trie* t);
void trie_build_from_csr(eh_context* ctx, eh_trie* t);  // head/off/vals already set
void trie_build_reverse(eh_context* ctx, eh_trie* t);   // dir + reverse level
// head/off/vals from host memory, the vals copy overlapped with the row work
void trie_build_from_host_csr(eh_context* ctx, eh_trie* t, const uint32_t* head, const uint64_t* off,
                              const uint32_t* vals, uint32_t n_nodes_hint);
void trie_layout(eh_context* ctx, eh_trie* t, const eh_layout_config* cfg);
void trie_set_bytes(const eh_trie* t, uint32_t set_index, std::vector<uint8_t>& out, uint8_t* layout);
// the reference's on-disk format (eh_disk.cu)
void trie_load_reference(eh_context* ctx, const char* dir, const eh_layout_config* cfg, eh_trie* t);
void trie_save_reference(eh_context* ctx, const eh_trie* t, const char* dir, uint32_t num_threads);

// set operations (eh_setops.cu)
void set_intersect_batch(eh_context* ctx, const uint32_t* elems, const uint64_t* set_off, uint32_t n_sets,
                         const uint8_t* layouts, const uint32_t* pair_a, const uint32_t* pair_b, uint32_t n_pairs,
                         uint64_t* counts, const uint64_t* out_off, uint32_t* out_elems);

// queries (eh_query.cu)
void query_count(eh_context* ctx, const eh_trie* t, int query, const eh_exec_config* cfg, uint64_t* result,
                 eh_query_stats* stats);
void query_count_batched(eh_context* ctx, const eh_trie* const* tries, uint32_t n, int query,
                         const eh_exec_config* cfg, uint64_t* results, eh_query_stats* stats);
void triangle_annotation(eh_context* ctx, const eh_trie* t, const eh_exec_config* cfg, uint64_t* annot_dev);
void query_weighted_root(eh_context* ctx, const eh_trie* t, int query, const uint64_t* z, uint32_t n_values,
                         uint64_t* result);
void query_count_select(eh_context* ctx, const eh_trie* t, int query, uint32_t value, const eh_exec_config* cfg,
                        uint64_t* result, eh_query_stats* stats);
eh_batch* batch_create(eh_context* ctx, const eh_trie* const* tries, uint32_t n, int query,
                       const eh_exec_config* cfg);
void batch_run(eh_context* ctx, eh_batch* b, uint64_t* results, eh_query_stats* stats);
void batch_free(eh_batch* b);
void query_count_in_scratch(eh_context* ctx, const eh_trie* t, int query, const eh_exec_config* cfg,
                            unsigned char* scratch, size_t bytes, uint64_t* result);
void query_materialize(eh_context* ctx, const eh_trie* t, int query, const eh_exec_config* cfg, int n_cols,
                       uint32_t* a, uint32_t* b, uint32_t* c, uint64_t cap, uint64_t* n_rows);

// rules (eh_rule.cu): the EH_QUERY_* of a rule body, and its relation
int rule_match(const eh_rule* rule, uint32_t* relation);

// dictionary encoding (eh_encode.cu)
eh_encoding* encoding_build(eh_context* ctx, const void* const* cols, const uint64_t* n_rows, uint32_t n_cols,
                            int type, int on_device);
void encoding_encode(eh_context* ctx, const eh_encoding* e, const void* col, uint64_t n, int on_device,
                     uint32_t* keys);
void encoding_decode(eh_context* ctx, const eh_encoding* e, const uint32_t* keys, uint64_t n, int on_device,
                     void* values);
void encoding_values(eh_context* ctx, const eh_encoding* e, void* values, uint64_t cap);
uint64_t encoding_size(const eh_encoding* e);
eh_context* encoding_ctx(const eh_encoding* e);
void encoding_free(eh_encoding* e);

// learned layout policy (eh_model.cu)
void model_choose_layouts(eh_context* ctx, const eh_model* m, const eh_trie* t, uint64_t max_bitset_bytes,
                          float min_gain, uint8_t* layout_dev, float* pred_dev);

}  // namespace eh
