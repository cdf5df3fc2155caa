// C ABI entry points (declared in include/eh_b200.h).  Every call catches
// its own failures and returns a status; nothing here aborts the process.
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "eh_internal.cuh"

namespace eh {
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

namespace {
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxPoolDevices] = {};
}  // namespace

cudaMemPool_t device_pool() {
  int dev = 0;
  EH_CUDA(cudaGetDevice(&dev));
  EH_REQUIRE(dev >= 0 && dev < kMaxPoolDevices, EH_ERR_UNSUPPORTED, "device index too large");
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    EH_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = ~0ull;  // keep freed blocks for reuse until trimmed
    EH_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pools[dev] = pool;
  }
  return g_pools[dev];
}

int trace_mode() {
  static const int mode = [] {
    const char* e = getenv("EH_TRACE");
    if (!e || !*e || strcmp(e, "0") == 0) return 0;
    return strcmp(e, "2") == 0 ? 2 : 1;
  }();
  return mode;
}

bool trace_enabled() { return trace_mode() != 0; }

static double wall_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static double pool_reserved_gb() {
  int dev = 0;
  uint64_t reserved = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kMaxPoolDevices && g_pools[dev])
    cudaMemPoolGetAttribute(g_pools[dev], cudaMemPoolAttrReservedMemCurrent, &reserved);
  return reserved / 1e9;
}

namespace {
// event-timed phases of the current thread's outermost traced call
struct EventPhase {
  const char* name;
  int depth;
  cudaEvent_t a, b;
  double host_ms;
};
thread_local std::vector<EventPhase> t_phases;
thread_local int t_depth = 0;
}  // namespace

TracePhase::TracePhase(const char* n, cudaStream_t st) : name(n), s(st), mode(trace_mode()), on(mode != 0) {
  if (!on) return;
  if (mode == 2) {
    cudaEvent_t a = nullptr;
    cudaEventCreate(&a);
    cudaEventRecord(a, s);
    idx = (int)t_phases.size();
    t_phases.push_back({n, t_depth++, a, nullptr, 0});
    t0 = wall_ms();
    return;
  }
  cudaStreamSynchronize(s);
  t0 = wall_ms();
}

void TracePhase::end() {
  if (!on) return;
  on = false;
  if (mode == 2) {
    // no synchronisation until the outermost phase ends: the stream runs as
    // it does untraced, and the events give each phase's device time
    cudaEvent_t b = nullptr;
    cudaEventCreate(&b);
    cudaEventRecord(b, s);
    t_phases[idx].b = b;
    t_phases[idx].host_ms = wall_ms() - t0;
    if (--t_depth == 0) {
      cudaEventSynchronize(b);
      for (const EventPhase& p : t_phases) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        fprintf(stderr, "eh-trace %*s%-*s %9.3f ms device %9.3f ms host\n", 2 * p.depth, "", 24 - 2 * p.depth,
                p.name, ms, p.host_ms);
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
      }
      fprintf(stderr, "eh-trace pool %.3f GB\n", pool_reserved_gb());
      t_phases.clear();
    }
    return;
  }
  cudaStreamSynchronize(s);
  // the engine pool's reserved bytes: a phase that grew it paid for new pages
  fprintf(stderr, "eh-trace %-24s %9.3f ms  pool %.3f GB\n", name, wall_ms() - t0, pool_reserved_gb());
}

void trim_device_pool(int device) {
  if (device < 0 || device >= kMaxPoolDevices) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (g_pools[device]) cudaMemPoolTrimTo(g_pools[device], 0);
}

eh_model* model_create(eh_context* ctx, int n_layers, const int* dims, uint64_t seed);
float model_train(eh_model* m, const float* x, const float* y, uint32_t batch, float lr, uint32_t steps);
float model_loss_grad_host(eh_model* m, const float* x, const float* y, uint32_t batch, float* grad);
void model_predict(eh_model* m, const float* x, uint32_t batch, float* y);
}  // namespace eh

using namespace eh;

template <typename F>
static eh_status guarded(F&& f) {
  try {
    f();
    return EH_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return EH_ERR_OOM;
  } catch (const std::exception& e) {
    set_error(e.what());
    return EH_ERR_INVALID;
  } catch (...) {
    set_error("unknown failure");
    return EH_ERR_INVALID;
  }
}

static void need(bool c, const char* msg) {
  if (!c) throw Error{EH_ERR_INVALID, msg};
}

static void set_device(eh_context* ctx) { EH_CUDA(cudaSetDevice(ctx->device)); }

extern "C" {

const char* eh_last_error(void) { return g_last_error.c_str(); }
const char* eh_version(void) { return "emptyheaded_b200 0.1 (sm_100a)"; }

eh_status eh_context_create(int device, eh_context** out) {
  return guarded([&] {
    need(out != nullptr, "out is null");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
      cudaGetLastError();
      throw Error{EH_ERR_NO_DEVICE, "no CUDA device visible"};
    }
    need(device >= 0 && device < n, "device index out of range");
    EH_CUDA(cudaSetDevice(device));
    auto* c = new eh_context();
    c->device = device;
    try {
      EH_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      EH_CUDA(cudaEventCreate(&c->ev0));
      EH_CUDA(cudaEventCreate(&c->ev1));
      EH_CUDA(cudaEventCreate(&c->ev2));
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
  });
}

eh_status eh_context_destroy(eh_context* ctx) {
  return guarded([&] {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->annot) cudaFree(ctx->annot);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->ev2) cudaEventDestroy(ctx->ev2);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->copy_stream) {
      cudaStreamSynchronize(ctx->copy_stream);
      cudaStreamDestroy(ctx->copy_stream);
    }
    trim_device_pool(ctx->device);  // return the pool's unused blocks to the driver
    delete ctx;
  });
}

eh_status eh_context_memory(eh_context* ctx, uint64_t* reserved, uint64_t* used, uint64_t* peak) {
  return guarded([&] {
    need(ctx, "ctx is null");
    set_device(ctx);
    cudaMemPool_t pool = device_pool();
    uint64_t r = 0, u = 0, h = 0;
    EH_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r));
    EH_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
    EH_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &h));
    if (reserved) *reserved = r;
    if (used) *used = u;
    if (peak) *peak = h;
  });
}

eh_status eh_context_reserve(eh_context* ctx, uint64_t bytes) {
  return guarded([&] {
    need(ctx, "ctx is null");
    set_device(ctx);
    cudaMemPool_t pool = device_pool();
    EH_CUDA(cudaStreamSynchronize(ctx->stream));
    // unused blocks go back to the driver, then one block of the requested
    // size is taken and freed: the pool keeps it (release threshold is
    // unbounded) and carves later allocations out of it
    EH_CUDA(cudaMemPoolTrimTo(pool, 0));
    if (bytes) {
      void* p = nullptr;
      cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, ctx->stream);
      if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error{EH_ERR_OOM, "reserving " + std::to_string(bytes) + " bytes failed"};
      }
      EH_CUDA(cudaFreeAsync(p, ctx->stream));
      EH_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    uint64_t zero = 0;
    EH_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero));
  });
}

eh_status eh_context_sync(eh_context* ctx) {
  return guarded([&] {
    need(ctx, "ctx is null");
    EH_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

eh_status eh_context_stream(eh_context* ctx, void** stream) {
  return guarded([&] {
    need(ctx && stream, "null argument");
    *stream = (void*)ctx->stream;
  });
}

eh_status eh_device_alloc(eh_context* ctx, uint64_t bytes, void** out) {
  return guarded([&] {
    need(ctx && out, "null argument");
    set_device(ctx);
    *out = nullptr;
    if (!bytes) return;
    cudaError_t e = cudaMallocFromPoolAsync(out, bytes, device_pool(), ctx->stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      *out = nullptr;
      throw Error{EH_ERR_OOM, "device allocation failed"};
    }
    EH_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

eh_status eh_device_free(eh_context* ctx, void* p) {
  return guarded([&] {
    need(ctx, "ctx is null");
    if (p) {
      EH_CUDA(cudaFreeAsync(p, ctx->stream));
      EH_CUDA(cudaStreamSynchronize(ctx->stream));
    }
  });
}

eh_status eh_memcpy(eh_context* ctx, void* dst, const void* src, uint64_t bytes) {
  return guarded([&] {
    need(ctx && (bytes == 0 || (dst && src)), "null argument");
    if (!bytes) return;
    EH_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
    EH_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

// --------------------------------------------------------------- graphs
static void alloc_pair(eh_context* ctx, uint64_t m, uint32_t** u, uint32_t** v) {
  need(u && v, "null output");
  *u = *v = nullptr;
  if (!m) return;
  if (cudaMallocFromPoolAsync((void**)u, m * 4, device_pool(), ctx->stream) != cudaSuccess ||
      cudaMallocFromPoolAsync((void**)v, m * 4, device_pool(), ctx->stream) != cudaSuccess) {
    cudaGetLastError();
    if (*u) cudaFreeAsync(*u, ctx->stream);
    *u = *v = nullptr;
    throw Error{EH_ERR_OOM, "device allocation of edge samples failed"};
  }
}

eh_status eh_graph_er(eh_context* ctx, uint64_t seed, uint32_t n, uint64_t m, uint32_t** u, uint32_t** v) {
  return guarded([&] {
    need(ctx, "ctx is null");
    set_device(ctx);
    alloc_pair(ctx, m, u, v);
    gen_er(ctx->stream, seed, n, m, *u, *v);
    EH_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

eh_status eh_graph_rmat(eh_context* ctx, uint64_t seed, int scale, uint64_t m, double a, double b, double c,
                        uint32_t** u, uint32_t** v) {
  return guarded([&] {
    need(ctx, "ctx is null");
    set_device(ctx);
    alloc_pair(ctx, m, u, v);
    gen_rmat(ctx->stream, seed, scale, m, a, b, c, *u, *v);
    EH_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

eh_status eh_graph_chunglu(eh_context* ctx, uint64_t seed, uint32_t n, uint64_t m, double gamma, uint32_t** u,
                           uint32_t** v) {
  return guarded([&] {
    need(ctx, "ctx is null");
    set_device(ctx);
    alloc_pair(ctx, m, u, v);
    gen_chunglu(ctx->stream, seed, n, m, gamma, *u, *v);
    EH_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

eh_status eh_graph_preprocess(eh_context* ctx, const uint32_t* u, const uint32_t* v, uint64_t m, int symmetric,
                              uint32_t** src, uint32_t** dst, uint64_t* rows, uint32_t* nodes) {
  return guarded([&] {
    need(ctx && src && dst && rows && nodes, "null argument");
    need(m == 0 || (u && v), "null input");
    set_device(ctx);
    DevBuf<uint32_t> s, d;
    preprocess(ctx->stream, u, v, m, symmetric ? 1 : 0, s, d, rows, nodes);
    *src = s.p;
    *dst = d.p;
    s.p = nullptr;  // ownership passes to the caller (eh_device_free)
    d.p = nullptr;
  });
}

// ----------------------------------------------------------------- tries
eh_status eh_trie_build(eh_context* ctx, const uint32_t* col0, const uint32_t* col1, uint64_t n_rows,
                        int cols_on_device, const eh_layout_config* cfg, eh_trie** out) {
  return guarded([&] {
    need(ctx && out, "null argument");
    need(n_rows == 0 || (col0 && col1), "null columns");
    need(n_rows < (1ull << 32), "tries hold fewer than 2^32 rows");
    set_device(ctx);
    *out = nullptr;
    auto* t = new eh_trie();
    t->ctx = ctx;
    try {
      if (cols_on_device || n_rows == 0) {
        trie_build(ctx, col0, col1, n_rows, cfg, t);
      } else {
        DevBuf<uint32_t> d0(n_rows, ctx->stream), d1(n_rows, ctx->stream);
        EH_CUDA(cudaMemcpyAsync(d0.p, col0, n_rows * 4, cudaMemcpyHostToDevice, ctx->stream));
        EH_CUDA(cudaMemcpyAsync(d1.p, col1, n_rows * 4, cudaMemcpyHostToDevice, ctx->stream));
        trie_build(ctx, d0.p, d1.p, n_rows, cfg, t);
        EH_CUDA(cudaStreamSynchronize(ctx->stream));
      }
    } catch (...) {
      delete t;
      throw;
    }
    *out = t;
  });
}

eh_status eh_trie_relayout(eh_context* ctx, eh_trie* trie, const eh_layout_config* cfg) {
  return guarded([&] {
    need(ctx && trie, "null argument");
    need(trie->ctx == ctx, "trie belongs to another context");
    set_device(ctx);
    trie_layout(ctx, trie, cfg);
  });
}

eh_status eh_trie_free(eh_trie* trie) {
  return guarded([&] {
    if (!trie) return;
    cudaSetDevice(trie->ctx->device);
    cudaStream_t s = trie->ctx->stream;
    delete trie;
    cudaStreamSynchronize(s);
  });
}

eh_status eh_trie_load_reference(eh_context* ctx, const char* dir, const eh_layout_config* cfg, eh_trie** out) {
  return guarded([&] {
    need(ctx && dir && out, "null argument");
    *out = nullptr;
    set_device(ctx);
    auto* t = new eh_trie();
    try {
      trie_load_reference(ctx, dir, cfg, t);
    } catch (...) {
      delete t;
      throw;
    }
    *out = t;
  });
}

eh_status eh_trie_save_reference(eh_context* ctx, const eh_trie* trie, const char* dir, uint32_t num_threads) {
  return guarded([&] {
    need(ctx && trie && dir, "null argument");
    need(trie->ctx == ctx, "trie belongs to another context");
    set_device(ctx);
    trie_save_reference(ctx, trie, dir, num_threads);
  });
}

eh_status eh_trie_info_get(const eh_trie* trie, eh_trie_info* out) {
  return guarded([&] {
    need(trie && out, "null argument");
    *out = trie->info;
  });
}

eh_status eh_trie_export(const eh_trie* trie, uint32_t* head, uint64_t* off, uint32_t* vals, uint8_t* layout) {
  return guarded([&] {
    need(trie, "trie is null");
    set_device(trie->ctx);
    cudaStream_t s = trie->ctx->stream;
    if (head && trie->n_head) EH_CUDA(cudaMemcpyAsync(head, trie->head.p, trie->n_head * 4, cudaMemcpyDeviceToHost, s));
    if (off) EH_CUDA(cudaMemcpyAsync(off, trie->off.p, (trie->n_head + 1) * 8, cudaMemcpyDeviceToHost, s));
    if (vals && trie->rows) EH_CUDA(cudaMemcpyAsync(vals, trie->vals.p, trie->rows * 4, cudaMemcpyDeviceToHost, s));
    if (layout && trie->n_head) EH_CUDA(cudaMemcpyAsync(layout, trie->layout.p, trie->n_head, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
  });
}

eh_status eh_trie_set_bytes(const eh_trie* trie, uint32_t set_index, uint8_t* out, uint64_t cap, uint64_t* nbytes,
                            uint8_t* layout) {
  return guarded([&] {
    need(trie && nbytes, "null argument");
    set_device(trie->ctx);
    std::vector<uint8_t> b;
    trie_set_bytes(trie, set_index, b, layout);
    *nbytes = b.size();
    if (out) {
      need(cap >= b.size(), "output buffer too small");
      if (!b.empty()) memcpy(out, b.data(), b.size());
    }
  });
}

// --------------------------------------------------------------- set ops
eh_status eh_set_intersect_batch(eh_context* ctx, const uint32_t* elems, const uint64_t* set_off, uint32_t n_sets,
                                 const uint8_t* layouts, const uint32_t* pair_a, const uint32_t* pair_b,
                                 uint32_t n_pairs, uint64_t* counts, const uint64_t* out_off, uint32_t* out_elems) {
  return guarded([&] {
    need(ctx && set_off && layouts && (n_pairs == 0 || (pair_a && pair_b && counts)), "null argument");
    need(set_off[n_sets] == 0 || elems, "null elements");
    need(!out_off || out_elems, "out_off given without out_elems");
    set_device(ctx);
    set_intersect_batch(ctx, elems, set_off, n_sets, layouts, pair_a, pair_b, n_pairs, counts, out_off, out_elems);
  });
}

// --------------------------------------------------------------- queries
eh_status eh_query_count(eh_context* ctx, const eh_trie* trie, int query, const eh_exec_config* cfg,
                         uint64_t* result, eh_query_stats* stats) {
  return guarded([&] {
    need(ctx && trie && result, "null argument");
    set_device(ctx);
    query_count(ctx, trie, query, cfg, result, stats);
  });
}

eh_status eh_encoding_build(eh_context* ctx, const void* const* cols, const uint64_t* n_rows, uint32_t n_cols,
                            int value_type, int on_device, eh_encoding** out) {
  return guarded([&] {
    need(ctx && out && (n_cols == 0 || (cols && n_rows)), "null argument");
    *out = nullptr;
    set_device(ctx);
    *out = encoding_build(ctx, cols, n_rows, n_cols, value_type, on_device);
  });
}

eh_status eh_encoding_encode(eh_context* ctx, const eh_encoding* enc, const void* col, uint64_t n, int on_device,
                             uint32_t* keys) {
  return guarded([&] {
    need(ctx && enc && (n == 0 || (col && keys)), "null argument");
    need(encoding_ctx(enc) == ctx, "encoding belongs to another context");
    set_device(ctx);
    encoding_encode(ctx, enc, col, n, on_device, keys);
  });
}

eh_status eh_encoding_decode(eh_context* ctx, const eh_encoding* enc, const uint32_t* keys, uint64_t n,
                             int on_device, void* values) {
  return guarded([&] {
    need(ctx && enc && (n == 0 || (keys && values)), "null argument");
    need(encoding_ctx(enc) == ctx, "encoding belongs to another context");
    set_device(ctx);
    encoding_decode(ctx, enc, keys, n, on_device, values);
  });
}

eh_status eh_encoding_size(const eh_encoding* enc, uint64_t* n_distinct) {
  return guarded([&] {
    need(enc && n_distinct, "null argument");
    *n_distinct = encoding_size(enc);
  });
}

eh_status eh_encoding_values(eh_context* ctx, const eh_encoding* enc, void* values, uint64_t cap) {
  return guarded([&] {
    need(ctx && enc && (cap == 0 || values), "null argument");
    need(encoding_ctx(enc) == ctx, "encoding belongs to another context");
    set_device(ctx);
    encoding_values(ctx, enc, values, cap);
  });
}

eh_status eh_encoding_free(eh_encoding* enc) {
  return guarded([&] {
    if (!enc) return;
    encoding_free(enc);
  });
}

eh_status eh_rule_match(const eh_rule* rule, int* query, uint32_t* relation) {
  return guarded([&] {
    need(rule && query, "null argument");
    *query = rule_match(rule, relation);
  });
}

eh_status eh_rule_count(eh_context* ctx, const eh_trie* const* relations, uint32_t n_relations, const eh_rule* rule,
                        const eh_exec_config* cfg, uint64_t* result, int* query, eh_query_stats* stats) {
  return guarded([&] {
    need(ctx && relations && rule && result, "null argument");
    uint32_t rel = 0;
    const int q = rule_match(rule, &rel);
    need(rel < n_relations && relations[rel], "rule names a relation that was not given");
    set_device(ctx);
    if (q == EH_QUERY_CLIQUE4_SEL || q == EH_QUERY_BARBELL_SEL)
      query_count_select(ctx, relations[rel], q, rule->sel_value, cfg, result, stats);
    else
      query_count(ctx, relations[rel], q, cfg, result, stats);
    if (query) *query = q;
  });
}

eh_status eh_query_count_select(eh_context* ctx, const eh_trie* trie, int query, uint32_t value,
                                const eh_exec_config* cfg, uint64_t* result, eh_query_stats* stats) {
  return guarded([&] {
    need(ctx && trie && result, "null argument");
    set_device(ctx);
    query_count_select(ctx, trie, query, value, cfg, result, stats);
  });
}

eh_status eh_query_count_batched(eh_context* ctx, const eh_trie* const* tries, uint32_t n_tries, int query,
                                 const eh_exec_config* cfg, uint64_t* results, eh_query_stats* stats) {
  return guarded([&] {
    need(ctx && tries && results, "null argument");
    set_device(ctx);
    query_count_batched(ctx, tries, n_tries, query, cfg, results, stats);
  });
}

eh_status eh_query_materialize(eh_context* ctx, const eh_trie* trie, int query, const eh_exec_config* cfg,
                               int n_cols, uint32_t* a, uint32_t* b, uint32_t* c, uint64_t cap, uint64_t* n_rows) {
  return guarded([&] {
    need(ctx && trie && n_rows, "null argument");
    set_device(ctx);
    query_materialize(ctx, trie, query, cfg, n_cols, a, b, c, cap, n_rows);
  });
}

eh_status eh_batch_create(eh_context* ctx, const eh_trie* const* tries, uint32_t n_tries, int query,
                          const eh_exec_config* cfg, eh_batch** out) {
  return guarded([&] {
    need(ctx && tries && out, "null argument");
    set_device(ctx);
    *out = nullptr;
    *out = batch_create(ctx, tries, n_tries, query, cfg);
  });
}

eh_status eh_batch_run(eh_context* ctx, eh_batch* batch, uint64_t* results, eh_query_stats* stats) {
  return guarded([&] {
    need(ctx && batch && results, "null argument");
    set_device(ctx);
    batch_run(ctx, batch, results, stats);
  });
}

eh_status eh_batch_free(eh_batch* batch) {
  return guarded([&] {
    if (batch) batch_free(batch);
  });
}

eh_status eh_triangle_annotation(eh_context* ctx, const eh_trie* trie, const eh_exec_config* cfg, uint64_t* annot) {
  return guarded([&] {
    need(ctx && trie && annot, "null argument");
    set_device(ctx);
    DevBuf<uint64_t> d(trie->n_head ? trie->n_head : 1, ctx->stream);
    triangle_annotation(ctx, trie, cfg, d.p);
    if (trie->n_head)
      EH_CUDA(cudaMemcpyAsync(annot, d.p, trie->n_head * 8, cudaMemcpyDeviceToHost, ctx->stream));
    EH_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

eh_status eh_query_weighted_root(eh_context* ctx, const eh_trie* trie, int query, const uint64_t* z,
                                 uint32_t n_values, uint64_t* result) {
  return guarded([&] {
    need(ctx && trie && result, "null argument");
    set_device(ctx);
    query_weighted_root(ctx, trie, query, z, n_values, result);
  });
}

eh_status eh_query_count_host_csr(eh_context* ctx, const uint32_t* head, uint32_t n_head, const uint64_t* off,
                                  const uint32_t* vals, uint32_t n_nodes, const eh_layout_config* cfg, int query,
                                  const eh_exec_config* ecfg, uint64_t* result, eh_query_stats* stats) {
  return guarded([&] {
    need(ctx && off && result, "null argument");
    need(n_head == 0 || (head && vals), "null arrays");
    set_device(ctx);
    cudaStream_t s = ctx->stream;
    eh_trie t;
    t.ctx = ctx;
    t.n_head = n_head;
    t.rows = off[n_head];
    need(t.rows < (1ull << 32), "tries hold fewer than 2^32 rows");
    need(off[0] == 0, "off[0] must be 0");
    TracePhase all("host_csr.total", s);
    trie_build_from_host_csr(ctx, &t, head, off, vals, n_nodes);
    trie_layout(ctx, &t, cfg);
    TracePhase ph("host_csr.query", s);
    query_count(ctx, &t, query, ecfg, result, stats);
  });
}

eh_status eh_timing_records(eh_context* ctx, float* rec, uint64_t cap, uint64_t* n) {
  return guarded([&] {
    need(ctx && n, "null argument");
    const uint64_t have = ctx->timing_records.size() / 8;
    *n = have;
    if (rec) {
      const uint64_t k = std::min(have, cap);
      if (k) memcpy(rec, ctx->timing_records.data(), k * 8 * sizeof(float));
    }
  });
}

// ------------------------------------------------------------------ model
eh_status eh_model_create(eh_context* ctx, int n_layers, const int* dims, uint64_t seed, eh_model** out) {
  return guarded([&] {
    need(ctx && dims && out, "null argument");
    set_device(ctx);
    *out = model_create(ctx, n_layers, dims, seed);
  });
}

eh_status eh_model_free(eh_model* m) {
  return guarded([&] {
    if (!m) return;
    cudaStream_t s = m->ctx->stream;
    delete m;
    cudaStreamSynchronize(s);
  });
}

eh_status eh_model_params(eh_model* m, float* host_params, uint64_t cap, uint64_t* n, int set) {
  return guarded([&] {
    need(m && n, "null argument");
    *n = m->n_params;
    if (!host_params) return;
    need(cap >= m->n_params, "buffer too small");
    cudaStream_t s = m->ctx->stream;
    if (set)
      EH_CUDA(cudaMemcpyAsync(m->params.p, host_params, m->n_params * 4, cudaMemcpyHostToDevice, s));
    else
      EH_CUDA(cudaMemcpyAsync(host_params, m->params.p, m->n_params * 4, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
  });
}

eh_status eh_model_train(eh_context* ctx, eh_model* m, const float* x, const float* y, uint32_t batch, float lr,
                         uint32_t steps, float* loss) {
  return guarded([&] {
    need(ctx && m && x && y && batch > 0, "bad argument");
    set_device(ctx);
    const float l = model_train(m, x, y, batch, lr, steps);
    if (loss) *loss = l;
  });
}

eh_status eh_model_loss_grad(eh_context* ctx, eh_model* m, const float* x, const float* y, uint32_t batch,
                             float* loss, float* grad) {
  return guarded([&] {
    need(ctx && m && x && y && batch > 0, "bad argument");
    set_device(ctx);
    const float l = model_loss_grad_host(m, x, y, batch, grad);
    if (loss) *loss = l;
  });
}

eh_status eh_model_predict(eh_context* ctx, eh_model* m, const float* x, uint32_t batch, float* y) {
  return guarded([&] {
    need(ctx && m && x && y, "null argument");
    set_device(ctx);
    if (batch) model_predict(m, x, batch, y);
  });
}

}  // extern "C"
