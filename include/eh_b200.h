/* eh_b200.h -- C ABI of the B200 storage-engine hot path.
 *
 * Plain C: opaque handles, plain pointers and sizes, no torch or C++ types.
 * Every function returns eh_status (EH_OK == 0) and never aborts; the text
 * of the last failure on the calling thread is returned by eh_last_error().
 *
 * Each entry point names the reference interface it replaces (paths are
 * relative to the EmptyHeaded repository).  The reference is a C++ template
 * library driven by generated query code; include/eh/ holds a C++ layer with
 * the reference's Trie / TrieBuilder / TrieIterator / par::reducer names over
 * this ABI, so that such code compiles and links against it.
 */
#ifndef EH_B200_H
#define EH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int eh_status;
enum {
  EH_OK = 0,
  EH_ERR_INVALID = 1,     /* bad argument */
  EH_ERR_CUDA = 2,        /* CUDA runtime error */
  EH_ERR_OOM = 3,         /* device allocation failed */
  /* 4 is unused: no device loop here waits on another thread or device */
  EH_ERR_UNSUPPORTED = 5, /* request outside what the build supports */
  EH_ERR_IO = 6,          /* file read/write failed */
  EH_ERR_NO_DEVICE = 7    /* no CUDA device visible */
};

/* Set layouts; the codes are the reference's type::layout values
 * (storage_engine/include/utils/common.hpp:83-91). */
enum {
  EH_LAYOUT_RANGE_BITSET = 0,
  EH_LAYOUT_UINTEGER = 1,
  EH_LAYOUT_BLOCK_BITSET = 3
};

/* How a trie picks each level-1 set's layout.
 * HEURISTIC: the reference density rule, hybrid::get_type
 *   (layouts/hybrid.hpp:103-111, utils/common.hpp:60-66).
 * LEARNED: the cost model loaded with eh_trie_build (falls back to the
 *   heuristic where the model abstains).
 * FORCED: every set gets eh_layout_config.forced_layout.
 * EXPLICIT: level-1 set i gets eh_layout_config.layouts[i] (an assignment
 *   found elsewhere, e.g. the per-set exhaustive search that bounds every
 *   layout policy); the head set keeps the density rule. */
enum { EH_POLICY_HEURISTIC = 0, EH_POLICY_LEARNED = 1, EH_POLICY_FORCED = 2, EH_POLICY_EXPLICIT = 3 };

/* Named generic-join plans executed as one device bag each. */
enum {
  EH_QUERY_TRIANGLE = 0, /* TriangleAgg(;z) :- Edge(a,b),Edge(b,c),Edge(a,c),z:long<-[COUNT(*)] */
  EH_QUERY_CLIQUE4 = 1,  /* FliqueAgg(;z) :- 4-clique, COUNT(*) */
  EH_QUERY_LOLLIPOP = 2, /* LollipopAgg(;z) :- triangle + Edge(a,x), COUNT(*) (2 bags) */
  EH_QUERY_BARBELL = 3,  /* BarbellAgg(;w) :- two triangles + Edge(a,x), COUNT(*) (2 bags) */
  /* equality-selection plans, run by eh_query_count_select only */
  EH_QUERY_CLIQUE4_SEL = 4, /* FliqueSelAgg(;z) :- 4-clique(a,b,c,d),Edge(a,x),x=value */
  EH_QUERY_BARBELL_SEL = 5  /* BarbellSelAgg(;w) :- triangle(a,b,c),Edge(a,p),Edge(p,x),triangle(x,y,z),p=value */
};

typedef struct eh_context eh_context;
typedef struct eh_trie eh_trie;
typedef struct eh_model eh_model;

/* ------------------------------------------------------------- context */
const char* eh_last_error(void);
const char* eh_version(void);

/* Replaces thread_pool::initializeThreadPool / deleteThreadPool
 * (storage_engine/include/utils/thread_pool.hpp:16-41): owns the device,
 * a stream and scratch memory. */
eh_status eh_context_create(int device, eh_context** out);
eh_status eh_context_destroy(eh_context* ctx);
eh_status eh_context_sync(eh_context* ctx);
/* the cudaStream_t the context launches on */
eh_status eh_context_stream(eh_context* ctx, void** stream);
/* Engine memory pool of the context's device (no counterpart in the
 * reference, which allocates from the host heap per call): bytes the pool
 * holds, bytes in use, and the peak in use since the last reserve.  Not
 * counted: the lollipop / barbell COUNT's per-head counters (8 bytes per head
 * entry of the largest trie queried so), a separate device allocation the
 * context keeps until it is destroyed. */
eh_status eh_context_memory(eh_context* ctx, uint64_t* reserved, uint64_t* used, uint64_t* peak);
/* Returns the pool's unused memory to the driver and reserves `bytes` as one
 * block that later allocations are carved from, so that calls whose peak fits
 * never map new device memory (which costs milliseconds per call when the
 * pool's free blocks are too fragmented for a request).  Resets the peak. */
eh_status eh_context_reserve(eh_context* ctx, uint64_t bytes);

/* Plain device memory for callers without a CUDA runtime of their own. */
eh_status eh_device_alloc(eh_context* ctx, uint64_t bytes, void** out);
eh_status eh_device_free(eh_context* ctx, void* p);
eh_status eh_memcpy(eh_context* ctx, void* dst, const void* src, uint64_t bytes);

/* ------------------------------------------------------- input pipeline
 * Seeded edge-sample generators (device).  Outputs are device arrays of m
 * raw samples (u[i], v[i]) allocated with eh_device_alloc. */
eh_status eh_graph_er(eh_context* ctx, uint64_t seed, uint32_t n, uint64_t m, uint32_t** u, uint32_t** v);
eh_status eh_graph_rmat(eh_context* ctx, uint64_t seed, int scale, uint64_t m, double a, double b, double c,
                        uint32_t** u, uint32_t** v);
eh_status eh_graph_chunglu(eh_context* ctx, uint64_t seed, uint32_t n, uint64_t m, double gamma, uint32_t** u,
                           uint32_t** v);
/* Symmetrise, drop self-loops, dedup, relabel nodes of degree > 0 by
 * (degree, id) ascending, then keep src < dst (symmetric == 0) or both
 * directions (symmetric == 1).  Output rows sorted by (src, dst), device
 * arrays from eh_device_alloc.  Stands in for the reference's
 * loadAndEncode step (codegen/create/createDB.scala:16-39), whose
 * order-preserving dictionary encoding is the identity on these ids. */
eh_status eh_graph_preprocess(eh_context* ctx, const uint32_t* u, const uint32_t* v, uint64_t m, int symmetric,
                              uint32_t** src, uint32_t** dst, uint64_t* rows, uint32_t* nodes);

/* ------------------------------------------------------ dictionary encoding
 * Replaces Encoding<T> (storage_engine/include/Encoding.hpp,
 * storage_engine/src/Encoding.cpp:21-48) as the loader uses it
 * (query_compiler/.../codegen/create/createDB.scala:242-270).  Value types
 * are the reference's numeric instantiations: uint32_t, int, long, float
 * (strings stay with the host).  Keys are assigned in ascending value order
 * over the distinct values of every column given to eh_encoding_build
 * (Encoding::build over a std::set), so key 0 is the smallest value.
 * Columns and outputs are device pointers when on_device != 0, else host
 * pointers.  Encoding a value the dictionary lacks is EH_ERR_INVALID (the
 * reference's value_to_key.at throws); so is a NaN float. */
enum { EH_VALUE_UINT32 = 0, EH_VALUE_INT32 = 1, EH_VALUE_INT64 = 2, EH_VALUE_FLOAT32 = 3 };
typedef struct eh_encoding eh_encoding;
/* Encoding<T>::build over all values of n_cols columns */
eh_status eh_encoding_build(eh_context* ctx, const void* const* cols, const uint64_t* n_rows, uint32_t n_cols,
                            int value_type, int on_device, eh_encoding** out);
/* Encoding<T>::encode_column: keys[i] = value_to_key.at(col[i]) */
eh_status eh_encoding_encode(eh_context* ctx, const eh_encoding* enc, const void* col, uint64_t n, int on_device,
                             uint32_t* keys);
/* key_to_value: values[i] = key_to_value[keys[i]] (a key out of range is EH_ERR_INVALID) */
eh_status eh_encoding_decode(eh_context* ctx, const eh_encoding* enc, const uint32_t* keys, uint64_t n,
                             int on_device, void* values);
/* num_distinct, and the key_to_value table (first cap entries) on the host,
 * the values Encoding::to_binary writes (Encoding.cpp:114-124) */
eh_status eh_encoding_size(const eh_encoding* enc, uint64_t* n_distinct);
eh_status eh_encoding_values(eh_context* ctx, const eh_encoding* enc, void* values, uint64_t cap);
eh_status eh_encoding_free(eh_encoding* enc);

/* ------------------------------------------------------------------ trie */
typedef struct {
  int policy;          /* EH_POLICY_* */
  int forced_layout;   /* EH_LAYOUT_* when policy == EH_POLICY_FORCED */
  const eh_model* model; /* EH_POLICY_LEARNED */
  /* Per-set cap on range-bitset bytes (12 per word) for FORCED and LEARNED.
   * Nonzero: a set over it, or over 16 words per element plus 64, keeps the
   * heuristic layout.  0: no cap for FORCED; LEARNED always applies the
   * per-element bound. */
  uint64_t max_bitset_bytes;
  const uint8_t* layouts; /* EH_POLICY_EXPLICIT: host array, one EH_LAYOUT_* per level-1 set (n_head) */
  /* LEARNED: a set leaves the density rule's layout only when the model
   * predicts at least this fraction less cost for another (0: 0.1), so
   * that small prediction errors do not move sets for nothing. */
  float min_gain;
} eh_layout_config;

typedef struct {
  uint64_t rows;        /* distinct tuples */
  uint32_t n_head;      /* distinct first-column values */
  uint32_t n_nodes;     /* value domain: max value + 1 */
  uint32_t head_layout; /* layout of the head set */
  uint32_t n_uinteger, n_range_bitset, n_block_bitset; /* level-1 set layouts */
  uint64_t bitset_words, block_count;
  uint64_t device_bytes;
  uint32_t max_set;     /* largest level-1 set */
  float build_ms;       /* device time of the build */
} eh_trie_info;

/* Two-level trie from an encoded binary relation: rows (col0[i], col1[i]),
 * any order, duplicates allowed.  Replaces the constructor
 * Trie<A,M>::Trie(path, max_set_sizes, attr_in, annotations)
 * (storage_engine/src/Trie.cpp:380-510) for two uint32 columns.
 * cols_on_device != 0: col0/col1 are device pointers. */
eh_status eh_trie_build(eh_context* ctx, const uint32_t* col0, const uint32_t* col1, uint64_t n_rows,
                        int cols_on_device, const eh_layout_config* cfg, eh_trie** out);
/* Re-pick level-1 set layouts of an existing trie (same elements). */
eh_status eh_trie_relayout(eh_context* ctx, eh_trie* trie, const eh_layout_config* cfg);
/* Replaces Trie<A,M>::~Trie (storage_engine/include/Trie.hpp:58-60). */
eh_status eh_trie_free(eh_trie* trie);
eh_status eh_trie_info_get(const eh_trie* trie, eh_trie_info* out);
/* Host copy of the trie's sets, the content Trie::foreach walks
 * (storage_engine/src/Trie.cpp:130-160): head[n_head], off[n_head+1],
 * vals[rows], layout[n_head] (any pointer may be NULL). */
eh_status eh_trie_export(const eh_trie* trie, uint32_t* head, uint64_t* off, uint32_t* vals, uint8_t* layout);
/* Reference-format bytes of level-1 set i (Set<hybrid>::get_data and
 * number_of_bytes, trie/set/Set.hpp:18-24): uinteger = u32[n];
 * range_bitset = [u64 start word][u64 words][u32 rank]
 * (layouts/range_bitset.hpp:123-157); block_bitset = per block
 * [u32 block id][u32 start index][4 x u64] (layouts/block_bitset.hpp:112-131).
 * set_index == UINT32_MAX selects the head set.  *nbytes receives the size;
 * out may be NULL to query it. */
eh_status eh_trie_set_bytes(const eh_trie* trie, uint32_t set_index, uint8_t* out, uint64_t cap, uint64_t* nbytes,
                            uint8_t* layout);

/* Trie<void*,ParMemoryBuffer>::load (storage_engine/src/Trie.cpp:37-75) of a
 * two-level trie the reference saved with Trie::save: dir holds ram/trieinfo.bin,
 * ram/data_head.bin and ram/data_<i>.bin (ParMemoryBuffer.cpp:64-100,
 * MemoryBuffer.cpp:104-172).  The sets are decoded on the host in whatever
 * layout they were saved, and the device trie is built from them with cfg's
 * layout policy (NULL: the density rule).  Annotations are not read. */
eh_status eh_trie_load_reference(eh_context* ctx, const char* dir, const eh_layout_config* cfg, eh_trie** out);
/* Trie::save (Trie.cpp:15-35) of a device trie in the reference's format, so
 * that Trie<void*,ParMemoryBuffer>::load in an engine built with
 * NUM_THREADS == num_threads reads it (its head buffer is found at index
 * NUM_THREADS).  Sets are written in hybrid::build's layout (range bitset when
 * dense, else uint, layouts/hybrid.hpp:103-111) whatever the device layout;
 * child blocks go to the num_threads buffers in contiguous runs of head
 * entries.  Creates dir and dir/ram. */
eh_status eh_trie_save_reference(eh_context* ctx, const eh_trie* trie, const char* dir, uint32_t num_threads);

/* --------------------------------------------------------------- set ops
 * Pairwise intersection of sets given as sorted uint32 runs in one packed
 * host array: set k is elems[set_off[k] .. set_off[k+1]).  Each set is
 * laid out on the device with layouts[k] (EH_LAYOUT_*), then pair p
 * intersects sets pair_a[p] and pair_b[p] with the kernel for that layout
 * pair.  Replaces ops::set_intersect (trie/set/ops/intersection/set.hpp:9-167):
 * counts[p] is the aggregate result; when out_off != NULL the
 * materialized elements of pair p are written to
 * out_elems[out_off[p] .. out_off[p] + counts[p]) (out_off[p] must leave
 * room for min(|A|,|B|) elements). */
eh_status eh_set_intersect_batch(eh_context* ctx, const uint32_t* elems, const uint64_t* set_off, uint32_t n_sets,
                                 const uint8_t* layouts, const uint32_t* pair_a, const uint32_t* pair_b,
                                 uint32_t n_pairs, uint64_t* counts, const uint64_t* out_off, uint32_t* out_elems);

/* ------------------------------------------------------------- queries */
typedef struct {
  int warps_per_block;   /* 0 = tuned default */
  int chunk_pairs;       /* target (v,w) pairs per work item; 0 = tuned default */
  int long_row;          /* size-class boundary: rows with at least this many
                            candidates run warp-wide, shorter ones are
                            flattened over the lanes; 0 = default (32) */
  int smem_words;        /* per-warp shared staging capacity in u32 words; 0 = default */
  int record_timings;    /* 1: log per-item device time for the cost model */
  int shard_index;       /* run work items i with i % shard_count == shard_index */
  int shard_count;       /* 0 or 1: all items (multi-GPU ranks split the plan) */
  int no_block_items;    /* 1: stage every N(b) in one warp's region; 0: an N(b)
                            too large for a warp's region but not for the
                            block's is staged block-wide and all the block's
                            warps share its rows (triangle COUNT) */
} eh_exec_config;

typedef struct {
  float query_ms;        /* device time from first launch to result */
  float kernel_ms;       /* device time of the intersection kernel(s) */
  uint32_t launches;     /* kernels launched */
  uint64_t work_items;
  uint64_t wedges;       /* (v,w) pairs probed */
  uint64_t algorithmic_bytes; /* 4*sum over edges (d+(u)+d+(v)) for triangle */
} eh_query_stats;

/* Runs one named COUNT plan over `trie` (the Edge relation in ordering
 * [0,1]) on the device and returns the aggregate.  Replaces the generated
 * bag code run_<i> (query_compiler/.../codegen/query/EHGenerator.scala:728-838)
 * with its ParTrieBuilder::build_aggregated_set / par_foreach_aggregate
 * loop nest (storage_engine/include/TrieBuilder.hpp:117-165,
 * storage_engine/src/TrieBuilder.cpp:451-578) and par::reducer
 * (storage_engine/include/utils/parallel.hpp:8-34).  The result is the
 * count modulo 2^64 (the reference's signed long, bit for bit). */
eh_status eh_query_count(eh_context* ctx, const eh_trie* trie, int query, const eh_exec_config* cfg,
                         uint64_t* result, eh_query_stats* stats);

/* eh_query_count for callers that must not allocate device memory while
 * they query (an embedding host whose device memory belongs to another
 * allocator, where a library cudaMalloc could fail and a cudaFree would
 * synchronise the device under the host's own work).  No counterpart in
 * the reference.  Runs the triangle or 4-clique plan with all its scratch
 * (work plan, queue, result, and the 4-clique's per-warp S buffers) in one
 * fixed 64 MiB device array compiled into the library; calls no
 * cudaMalloc/cudaFree.  Limits: the trie's plan must fit, about 8 bytes per
 * head entry plus 16 per work item (an R-MAT scale-22 trie fits); for the
 * 4-clique, a largest set above what one block stages in shared memory
 * (96 KB for the staged set and S together) needs S buffers of
 * 4 x (largest set + 1) bytes per warp in what the plan leaves of the array
 * (with 8 warps per block, a largest set up to about 2M elements).  Larger
 * tries get EH_ERR_UNSUPPORTED, and the call returns with none of its GPU
 * work in flight (at most the planner's count has run).  The first call
 * on a device looks the array up (make it before any stream capture).  Calls
 * share the array: this entry serialises its own calls per device; other
 * GPU work touching the array concurrently would race. */
eh_status eh_query_count_noalloc(eh_context* ctx, const eh_trie* trie, int query, const eh_exec_config* cfg,
                                 uint64_t* result);

/* Equality-selection COUNT plans (test/graph/travis.py:385-401, 472-487;
 * plans query_compiler/src/test/scala/QueryPlannerTest.scala:230-304).
 * Replaces the generated selection bags: emitSelectionValues /
 * emitHeadContainsSelections (EHGenerator.scala:657-701) answer the selected
 * attribute at the head with get_next_block(value_to_key.at(value))
 * (TrieIterator.cpp:72-78), and the bag of the selected value's partners
 * joins the 4-clique or triangle bags.  query: EH_QUERY_CLIQUE4_SEL or
 * EH_QUERY_BARBELL_SEL; value: the selection literal, a value of the
 * relation's columns.  A value in neither column is EH_ERR_INVALID (the
 * reference's value_to_key.at throws).  A value without partners counts 0
 * (the reference's generated code reads a null or out-of-range block
 * there, TrieBlock.hpp:86-111).  Count modulo 2^64 as for eh_query_count. */
eh_status eh_query_count_select(eh_context* ctx, const eh_trie* trie, int query, uint32_t value,
                                const eh_exec_config* cfg, uint64_t* result, eh_query_stats* stats);

/* A COUNT rule given as data, the bag-level entry the generated code can
 * call instead of a named plan: the rule body's atoms over numbered
 * variables (relation index, first and second variable; rel(v0, v1) holds
 * for the rows (v0, v1) of relation `relation`) and an optional equality
 * selection (sel_var >= 0: that variable = sel_value).  Replaces the
 * query compiler's plan + emitted bag (QueryPlanner, EHGenerator.scala:
 * 728-838) for the bodies the device runs: a COUNT does not depend on the
 * attribute order or the bag decomposition, nor on the names of the
 * variables, so the body is matched up to renaming against the triangle,
 * 4-clique, lollipop and barbell bodies and the 4-clique / barbell
 * selections of test/graph/travis.py.  Other bodies, or atoms over more than
 * one relation, are EH_ERR_UNSUPPORTED. */
typedef struct {
  uint32_t relation;
  uint32_t v0, v1;
} eh_atom;
typedef struct {
  uint32_t n_vars;
  uint32_t n_atoms;
  const eh_atom* atoms;
  int32_t sel_var; /* -1: no selection */
  uint32_t sel_value;
} eh_rule;
/* the device plan (EH_QUERY_*) of a rule and the relation it reads; host only */
eh_status eh_rule_match(const eh_rule* rule, int* query, uint32_t* relation);
/* COUNT of a rule over relations[] (tries in ordering [0,1]); *query gets
 * the plan it ran (may be NULL) */
eh_status eh_rule_count(eh_context* ctx, const eh_trie* const* relations, uint32_t n_relations, const eh_rule* rule,
                        const eh_exec_config* cfg, uint64_t* result, int* query, eh_query_stats* stats);

/* Materialized output of the triangle plan, rows sorted lexicographically
 * (the order Trie::foreach, storage_engine/src/Trie.cpp:130-160, walks the
 * reference's output trie).  Replaces the materializing bag of
 * Triangle(a,b,c) :- Edge(a,b),Edge(b,c),Edge(a,c) (TrieBuilder::build_set /
 * allocate_next / set_level, storage_engine/src/TrieBuilder.cpp:44-221,
 * 376-410).  n_cols == 3: rows (a,b,c) in a, b, c; n_cols == 2: the
 * projection TriangleProj(a,b) as the reference plans it -- attributes
 * neither materialized, selected nor aggregated are dropped
 * (query_compiler/.../codegen/query/QueryPlan.scala:245), so the rows are
 * (a,b) with b in N(a) ∩ head (c unused).  Host columns of cap rows; with
 * a == NULL only *n_rows is returned. */
eh_status eh_query_materialize(eh_context* ctx, const eh_trie* trie, int query, const eh_exec_config* cfg,
                               int n_cols, uint32_t* a, uint32_t* b, uint32_t* c, uint64_t cap, uint64_t* n_rows);

/* Same plan over many tries in one persistent launch; results[g] per
 * trie. */
eh_status eh_query_count_batched(eh_context* ctx, const eh_trie* const* tries, uint32_t n_tries, int query,
                                 const eh_exec_config* cfg, uint64_t* results, eh_query_stats* stats);

/* A prepared batch: the work plans of n tries (triangle or 4-clique)
 * concatenated once into one queue, and the step (zero the results and the
 * queue, the persistent kernel over every trie's items, the results to
 * host) captured in a CUDA graph.  eh_batch_run replays the graph: one
 * launch for the whole batch.  Same results as eh_query_count per trie.
 * The tries must outlive the batch and not be re-laid-out while it exists. */
typedef struct eh_batch eh_batch;
eh_status eh_batch_create(eh_context* ctx, const eh_trie* const* tries, uint32_t n_tries, int query,
                          const eh_exec_config* cfg, eh_batch** out);
eh_status eh_batch_run(eh_context* ctx, eh_batch* batch, uint64_t* results, eh_query_stats* stats);
eh_status eh_batch_free(eh_batch* batch);

/* Per-head-entry triangle annotation T(a) (the annotated bag of
 * lollipop/barbell, TrieBuilder::set_annotation, TrieBuilder.cpp:428-446),
 * copied to host annot[n_head]. */
eh_status eh_triangle_annotation(eh_context* ctx, const eh_trie* trie, const eh_exec_config* cfg, uint64_t* annot);

/* The root bag of the lollipop / barbell plans joined with an annotated
 * unary relation Z(v; z) (the intermediate bag the reference materialises
 * with TrieBuilder::set_annotation and reads back with
 * TrieIterator::get_annotation, TrieIterator.cpp:45-59; the root bags of
 * QueryPlannerTest.scala:199-230 as EHGenerator.scala:399-480 emits them):
 *   EH_QUERY_LOLLIPOP: sum over head values a of z(a) * |{d : (a,d)}|
 *   EH_QUERY_BARBELL:  sum over rows (a,x) of z(a) * z(x)
 * z is given by value on the host: z[v] for v < n_values; values beyond
 * and values without an annotation count 0.  Result modulo 2^64 (the
 * reference's signed long, bit for bit). */
eh_status eh_query_weighted_root(eh_context* ctx, const eh_trie* trie, int query, const uint64_t* z,
                                 uint32_t n_values, uint64_t* result);

/* Host-buffer convenience: copy a CSR trie (head, off, vals) from host
 * memory, lay it out with cfg, count, and return; the reference-facing
 * call with host inputs. */
eh_status eh_query_count_host_csr(eh_context* ctx, const uint32_t* head, uint32_t n_head, const uint64_t* off,
                                  const uint32_t* vals, uint32_t n_nodes, const eh_layout_config* cfg, int query,
                                  const eh_exec_config* ecfg, uint64_t* result, eh_query_stats* stats);

/* Records of per-item intersection timings from the last query run with
 * record_timings, for the cost model.  One record per work item, 8 floats:
 * [|N(b)|, pairs probed, density of N(b), range of N(b), layout of N(b),
 * probe mode, b (uint32 bit pattern), SM cycles].  rec must hold cap
 * records; *n receives the count. */
eh_status eh_timing_records(eh_context* ctx, float* rec, uint64_t cap, uint64_t* n);

/* --------------------------------------------------------- cost model
 * A small fp32 MLP trained on the device by hand-written kernels.  dims:
 * layer widths d0..dL.  Parameters packed (W0,b0,W1,b1,...) with W row-major
 * [d_{l+1} x d_l]. */
eh_status eh_model_create(eh_context* ctx, int n_layers, const int* dims, uint64_t seed, eh_model** out);
eh_status eh_model_free(eh_model* m);
eh_status eh_model_params(eh_model* m, float* host_params, uint64_t cap, uint64_t* n, int set);
/* one SGD step on a batch (host arrays x[batch*d0], y[batch*dL]); returns the loss */
eh_status eh_model_train(eh_context* ctx, eh_model* m, const float* x, const float* y, uint32_t batch, float lr,
                         uint32_t steps, float* loss);
/* loss and gradient without updating (host arrays); grad has n_params entries */
eh_status eh_model_loss_grad(eh_context* ctx, eh_model* m, const float* x, const float* y, uint32_t batch,
                             float* loss, float* grad);
eh_status eh_model_predict(eh_context* ctx, eh_model* m, const float* x, uint32_t batch, float* y);

#ifdef __cplusplus
}
#endif
#endif /* EH_B200_H */
