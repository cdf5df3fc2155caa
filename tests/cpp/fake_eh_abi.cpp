/* TEST DOUBLE of the C ABI (include/eh_b200.h) for the C++ layer's host logic.
 *
 * Never linked into the product.  tests/test_dropin_cpu.py links
 * tests/cpp/dropin_bags.cpp against this file instead of libeh_b200.so, so
 * that the layer's symbolic pass, plan matching and replay run on a machine
 * without a GPU.  Every call computes by brute force on the host (small
 * graphs only) and appends its name to the file named by $EH_FAKE_LOG, which
 * tells the test which entry each bag was dispatched to.  The counts it
 * returns are checked against the reference's goldens by the test, so a
 * wrong dispatch or a wrong replay shows as a wrong count.
 */
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "eh_b200.h"

struct eh_context {
  int device;
};
struct eh_trie {
  std::vector<uint32_t> head;
  std::vector<uint64_t> off;
  std::vector<uint32_t> vals;
  uint32_t n_nodes = 0;
  bool has(uint32_t a, uint32_t b) const {
    auto h = std::lower_bound(head.begin(), head.end(), a);
    if (h == head.end() || *h != a) return false;
    const size_t i = h - head.begin();
    return std::binary_search(vals.begin() + off[i], vals.begin() + off[i + 1], b);
  }
};

static std::string g_err;
static void log_call(const char* name) {
  const char* p = getenv("EH_FAKE_LOG");
  if (!p) return;
  FILE* f = fopen(p, "a");
  if (!f) return;
  fprintf(f, "%s\n", name);
  fclose(f);
}

extern "C" {

const char* eh_last_error(void) { return g_err.c_str(); }

eh_status eh_context_create(int device, eh_context** out) {
  *out = new eh_context{device};
  return EH_OK;
}
eh_status eh_context_destroy(eh_context* ctx) {
  delete ctx;
  return EH_OK;
}

eh_status eh_trie_build(eh_context*, const uint32_t* c0, const uint32_t* c1, uint64_t n, int, const eh_layout_config*,
                        eh_trie** out) {
  std::vector<std::pair<uint32_t, uint32_t>> r(n);
  for (uint64_t i = 0; i < n; i++) r[i] = {c0[i], c1[i]};
  std::sort(r.begin(), r.end());
  r.erase(std::unique(r.begin(), r.end()), r.end());
  eh_trie* t = new eh_trie();
  for (auto& e : r) {
    if (t->head.empty() || t->head.back() != e.first) {
      t->head.push_back(e.first);
      t->off.push_back(t->vals.size());
    }
    t->vals.push_back(e.second);
    t->n_nodes = std::max(t->n_nodes, std::max(e.first, e.second) + 1);
  }
  t->off.push_back(t->vals.size());
  *out = t;
  return EH_OK;
}
eh_status eh_trie_free(eh_trie* t) {
  delete t;
  return EH_OK;
}
eh_status eh_trie_info_get(const eh_trie* t, eh_trie_info* o) {
  memset(o, 0, sizeof(*o));
  o->rows = t->vals.size();
  o->n_head = (uint32_t)t->head.size();
  o->n_nodes = t->n_nodes;
  return EH_OK;
}
eh_status eh_trie_export(const eh_trie* t, uint32_t* head, uint64_t* off, uint32_t* vals, uint8_t* layout) {
  if (head) std::copy(t->head.begin(), t->head.end(), head);
  if (off) std::copy(t->off.begin(), t->off.end(), off);
  if (vals) std::copy(t->vals.begin(), t->vals.end(), vals);
  if (layout) memset(layout, EH_LAYOUT_UINTEGER, t->head.size());
  return EH_OK;
}
eh_status eh_trie_save_reference(eh_context*, const eh_trie*, const char*, uint32_t) {
  g_err = "not in the test double";
  return EH_ERR_UNSUPPORTED;
}
eh_status eh_trie_load_reference(eh_context*, const char*, const eh_layout_config*, eh_trie**) {
  g_err = "not in the test double";
  return EH_ERR_UNSUPPORTED;
}

eh_status eh_set_intersect_batch(eh_context*, const uint32_t* elems, const uint64_t* set_off, uint32_t,
                                 const uint8_t*, const uint32_t* pa, const uint32_t* pb, uint32_t n_pairs,
                                 uint64_t* counts, const uint64_t* out_off, uint32_t* out_elems) {
  log_call("eh_set_intersect_batch");
  for (uint32_t p = 0; p < n_pairs; p++) {
    const uint32_t* a = elems + set_off[pa[p]];
    const uint32_t* b = elems + set_off[pb[p]];
    std::vector<uint32_t> r;
    std::set_intersection(a, elems + set_off[pa[p] + 1], b, elems + set_off[pb[p] + 1], std::back_inserter(r));
    counts[p] = r.size();
    if (out_off) std::copy(r.begin(), r.end(), out_elems + out_off[p]);
  }
  return EH_OK;
}

// COUNT of a conjunctive body over one binary relation by backtracking
// over the variables in order (test sizes only); bodies the device has no
// plan for are refused like the real entry refuses them
static void count_rec(const eh_trie* t, const eh_rule* r, std::vector<uint32_t>& val, uint32_t k, uint64_t* acc) {
  if (k == r->n_vars) {
    (*acc)++;
    return;
  }
  // candidates: the set of an atom (bound, k), else every value
  const uint32_t* lo = nullptr;
  const uint32_t* hi = nullptr;
  for (uint32_t i = 0; i < r->n_atoms && !lo; i++) {
    const eh_atom& a = r->atoms[i];
    if (a.v1 == k && a.v0 < k) {
      auto h = std::lower_bound(t->head.begin(), t->head.end(), val[a.v0]);
      if (h == t->head.end() || *h != val[a.v0]) return;
      const size_t j = h - t->head.begin();
      lo = t->vals.data() + t->off[j];
      hi = t->vals.data() + t->off[j + 1];
    }
  }
  std::vector<uint32_t> all;
  if (!lo) {
    all.resize(t->n_nodes);
    for (uint32_t v = 0; v < t->n_nodes; v++) all[v] = v;
    lo = all.data();
    hi = all.data() + all.size();
  }
  for (const uint32_t* c = lo; c < hi; c++) {
    val[k] = *c;
    bool ok = true;
    for (uint32_t i = 0; i < r->n_atoms && ok; i++) {
      const eh_atom& a = r->atoms[i];
      if (a.v0 <= k && a.v1 <= k && (a.v0 == k || a.v1 == k)) ok = t->has(val[a.v0], val[a.v1]);
    }
    if (ok) count_rec(t, r, val, k + 1, acc);
  }
}
eh_status eh_rule_count(eh_context*, const eh_trie* const* rel, uint32_t, const eh_rule* r, const eh_exec_config*,
                        uint64_t* result, int* query, eh_query_stats*) {
  // the device plans: 3 variables / 3 atoms (triangle) or 4 / 6 (4-clique)
  const bool plan = (r->n_vars == 3 && r->n_atoms == 3) || (r->n_vars == 4 && r->n_atoms == 6);
  if (!plan) {
    log_call("eh_rule_count:unsupported");
    g_err = "no device plan for this body";
    return EH_ERR_UNSUPPORTED;
  }
  log_call("eh_rule_count");
  std::vector<uint32_t> val(r->n_vars);
  uint64_t acc = 0;
  count_rec(rel[0], r, val, 0, &acc);
  *result = acc;
  if (query) *query = r->n_vars == 3 ? EH_QUERY_TRIANGLE : EH_QUERY_CLIQUE4;
  return EH_OK;
}

eh_status eh_triangle_annotation(eh_context*, const eh_trie* t, const eh_exec_config*, uint64_t* annot) {
  log_call("eh_triangle_annotation");
  for (size_t i = 0; i < t->head.size(); i++) {
    uint64_t c = 0;
    const uint32_t a = t->head[i];
    for (uint64_t e = t->off[i]; e < t->off[i + 1]; e++)
      for (uint64_t f = t->off[i]; f < t->off[i + 1]; f++)
        if (t->has(t->vals[e], t->vals[f])) c++;
    (void)a;
    annot[i] = c;
  }
  return EH_OK;
}

eh_status eh_query_weighted_root(eh_context*, const eh_trie* t, int query, const uint64_t* z, uint32_t n_values,
                                 uint64_t* result) {
  log_call(query == EH_QUERY_LOLLIPOP ? "eh_query_weighted_root:lollipop" : "eh_query_weighted_root:barbell");
  auto zv = [&](uint32_t v) { return v < n_values ? z[v] : 0ull; };
  uint64_t acc = 0;
  for (size_t i = 0; i < t->head.size(); i++) {
    const uint64_t za = zv(t->head[i]);
    if (query == EH_QUERY_LOLLIPOP) {
      acc += za * (t->off[i + 1] - t->off[i]);
    } else {
      uint64_t s = 0;
      for (uint64_t e = t->off[i]; e < t->off[i + 1]; e++) s += zv(t->vals[e]);
      acc += za * s;
    }
  }
  *result = acc;
  return EH_OK;
}

}  // extern "C"
