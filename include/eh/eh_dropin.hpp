// eh_dropin.hpp -- the reference storage engine's C++ API over the B200 C ABI.
//
// Generated query code (the run_<i> bags EHGenerator.scala:728-838 emits)
// is written against the reference's templates: Trie<A,M>
// (storage_engine/include/Trie.hpp:22-67), ParTrieIterator / TrieIterator
// (include/TrieIterator.hpp:24-59), ParTrieBuilder / TrieBuilder
// (include/TrieBuilder.hpp:28-165), TrieBlock / Set (trie/TrieBlock.hpp,
// trie/set/Set.hpp:18-159), par::reducer (utils/parallel.hpp:8-34),
// thread_pool and timer.  This header gives those names, signatures and
// ownership rules, so such code compiles unchanged and links against
// libeh_b200.so.  The named headers beside it (Trie.hpp, TrieBuilder.hpp,
// ...) include this file.
//
// How a bag runs.  The reference executes the bag's host lambdas over its
// CPU sets.  Here:
//  1. Tries live on the device (eh_trie_build / eh_trie_load_reference);
//     a host copy of their sets is fetched only when a host loop needs it.
//  2. ParTrieBuilder::par_foreach_aggregate / par_foreach_builder first
//     call the lambda once in a symbolic pass: no set is read, every build
//     returns 0 and every loop runs one placeholder value, and the layer
//     records which accessor (relation, level) each build reads at which
//     attribute.  That gives the bag's rule body: one atom per accessor
//     over numbered attributes.
//  3. A body the device runs as one plan is dispatched:
//       - an aggregate bag over one binary relation -> eh_rule_count
//         (matched up to renaming against the triangle / 4-clique plans);
//       - the lollipop / barbell root bag: one relation atom joined with an
//         annotated unary relation -> eh_query_weighted_root;
//       - the annotated triangle bag bag(a;z) that materialises a with
//         z = number of (b,c) closing a triangle -> eh_triangle_annotation.
//     The device's aggregate is then handed to the generated code through
//     its own arithmetic: the lambda runs again (once for an aggregate,
//     once per output element for the annotated bag) with every loop over
//     one placeholder element, every count and annotation read equal to 1,
//     except one -- the last value the symbolic pass saw read that is not a
//     loop's set -- which returns the device's value.  For the COUNT bags
//     EHGenerator emits (annotation += count * 1 and products of
//     annotations, EHGenerator.scala:399-520) the lambda's reducer then
//     holds exactly the device's aggregate.
//  4. Any other bag runs the generated code's own loops on the host, with
//     every set intersection done on the device (eh_set_intersect_batch):
//     correct, and launch-bound.
// The layer's host loop runs on one thread (tid 0); NUM_THREADS is 1.
// The NUM ROWS a dispatched bag reports counts the replayed rows, not the
// reference's intermediate rows; annotations and aggregates are exact.
//
// Errors: the reference asserts or prints and continues; this layer throws
// std::runtime_error carrying eh_last_error().
#ifndef EH_DROPIN_HPP
#define EH_DROPIN_HPP

#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../eh_b200.h"

// The layer's host loop is one thread; the reference's is NUM_THREADS_IN.
static const size_t NUM_THREADS = 1;
#define PADDING 300

// Memory-buffer template arguments of the reference (ParMemoryBuffer,
// ParMMapBuffer, utils/ParMemoryBuffer.hpp): here only tags, tries live on
// the device.
struct ParMemoryBuffer {};
struct ParMMapBuffer {};
struct MemoryBuffer {};
struct hybrid {};
typedef hybrid layout;

namespace type {
enum layout : uint8_t { RANGE_BITSET = 0, UINTEGER = 1, HYBRID = 2, BLOCK_BITSET = 3, BLOCK = 4, NOT_VALID = 8 };
}

namespace common {
static size_t bitset_length = 2;
static double bitset_req = 128.0;
// the reference's density rule (utils/common.hpp:60-66)
inline bool is_sparse(size_t length, size_t range) {
  if (length > bitset_length) return ((double)range / length) > bitset_req;
  return true;
}
}  // namespace common

namespace timer {
static inline std::chrono::time_point<std::chrono::system_clock> start_clock() {
  return std::chrono::system_clock::now();
}
static inline double stop_clock(std::chrono::time_point<std::chrono::system_clock> t_in) {
  std::chrono::duration<double> s = std::chrono::system_clock::now() - t_in;
  return s.count();
}
static inline double stop_clock(std::string in, std::chrono::time_point<std::chrono::system_clock> t_in) {
  const double t = stop_clock(t_in);
  std::cout << "Time[" + in + "]: " << t << " s" << std::endl;
  return t;
}
}  // namespace timer

// -------------------------------------------------------------- Encoding
// A relation's dictionary (storage_engine/include/Encoding.hpp:21-37): key i
// stands for key_to_value[i]; value_to_key maps back.  build() gives keys in
// the order the values come (a std::set: ascending, Encoding.cpp:21-37); a
// value given twice keeps its first key and still takes a key number, as
// there.  encode_column maps a column through value_to_key and throws on a
// value the dictionary lacks (the reference's .at).  to_binary / from_binary
// write and read <path>encoding.bin: the uint32 count, then every value in key
// order as its bytes (strings: a size_t length, then the characters), the
// reference's file (Encoding.cpp:52-130), so dictionaries pass between the
// engines.  Host code: the device dictionary of eh_encoding_* builds the same
// keys for uint32/uint64 columns (ascending values).
template <class T>
struct Encoding {
  uint32_t num_distinct = 0;
  std::vector<T> key_to_value;
  std::unordered_map<T, uint32_t> value_to_key;

  void build(std::set<T>* values) {
    for (const T& v : *values) add(v);
  }
  void build(std::vector<T>* values) {
    for (const T& v : *values) add(v);
  }
  std::vector<uint32_t>* encode_column(T* column, const size_t length) {
    std::unique_ptr<std::vector<uint32_t>> out(new std::vector<uint32_t>(length));
    for (size_t i = 0; i < length; i++) (*out)[i] = value_to_key.at(column[i]);
    return out.release();
  }
  void to_binary(const std::string path) {
    std::ofstream f(path + "encoding.bin", std::ios::binary | std::ios::out);
    if (!f) throw std::runtime_error("cannot write " + path + "encoding.bin");
    f.write(reinterpret_cast<const char*>(&num_distinct), sizeof(num_distinct));
    for (uint32_t k = 0; k < num_distinct; k++) write_value(f, key_to_value.at(k));
    if (!f) throw std::runtime_error("write of " + path + "encoding.bin failed");
  }
  static Encoding<T>* from_binary(const std::string path) {
    std::ifstream f(path + "encoding.bin", std::ios::binary | std::ios::in);
    if (!f) throw std::runtime_error("cannot read " + path + "encoding.bin");
    std::unique_ptr<Encoding<T>> e(new Encoding<T>());
    uint32_t n = 0;
    f.read(reinterpret_cast<char*>(&n), sizeof(n));
    if (!f) throw std::runtime_error(path + "encoding.bin is truncated");
    e->key_to_value.reserve(n);
    e->value_to_key.reserve(n);
    for (uint32_t k = 0; k < n; k++) {
      T v;
      read_value(f, v);
      if (!f) throw std::runtime_error(path + "encoding.bin is truncated");
      e->add(v);
    }
    return e.release();
  }

 private:
  void add(const T& v) {
    value_to_key.insert(std::make_pair(v, num_distinct++));
    key_to_value.push_back(v);
  }
  static void write_value(std::ofstream& f, const T& v) {
    if constexpr (std::is_same<T, std::string>::value) {
      const size_t len = v.size();
      f.write(reinterpret_cast<const char*>(&len), sizeof(len));
      f.write(v.data(), (std::streamsize)len);
    } else {
      f.write(reinterpret_cast<const char*>(&v), sizeof(T));
    }
  }
  static void read_value(std::ifstream& f, T& v) {
    if constexpr (std::is_same<T, std::string>::value) {
      size_t len = 0;
      f.read(reinterpret_cast<char*>(&len), sizeof(len));
      if (!f) return;
      v.assign(len, '\0');
      f.read(&v[0], (std::streamsize)len);
    } else {
      f.read(reinterpret_cast<char*>(&v), sizeof(T));
    }
  }
};

// ------------------------------------------------------------------ engine
namespace ehd {

inline void check(eh_status st, const char* what) {
  if (st != EH_OK) throw std::runtime_error(std::string(what) + ": " + eh_last_error());
}

// The process's engine context: device $EH_DEVICE (default 0), created on
// first use, destroyed by thread_pool::deleteThreadPool or at exit.
struct Engine {
  eh_context* ctx = nullptr;
  ~Engine() {
    if (ctx) eh_context_destroy(ctx);
  }
};
inline Engine& engine() {
  static Engine e;
  return e;
}
inline eh_context* context() {
  Engine& e = engine();
  if (!e.ctx) {
    const char* d = getenv("EH_DEVICE");
    check(eh_context_create(d ? atoi(d) : 0, &e.ctx), "eh_context_create");
  }
  return e.ctx;
}

// A binary relation resident on the device, with a host copy of its sets
// made when a host loop first needs one.
struct Relation {
  eh_trie* trie = nullptr;
  uint32_t n_head = 0;
  uint64_t rows = 0;
  bool mirrored = false;
  std::vector<uint32_t> head;
  std::vector<uint64_t> off;
  std::vector<uint32_t> vals;
  explicit Relation(eh_trie* t) : trie(t) {
    eh_trie_info info;
    check(eh_trie_info_get(t, &info), "eh_trie_info_get");
    n_head = info.n_head;
    rows = info.rows;
  }
  ~Relation() {
    if (trie) eh_trie_free(trie);
  }
  Relation(const Relation&) = delete;
  Relation& operator=(const Relation&) = delete;
  void mirror() {
    if (mirrored) return;
    head.resize(n_head ? n_head : 1);
    off.resize(n_head + 1);
    vals.resize(rows ? rows : 1);
    check(eh_trie_export(trie, head.data(), off.data(), vals.data(), nullptr), "eh_trie_export");
    head.resize(n_head);
    vals.resize(rows);
    mirrored = true;
  }
  long find_head(uint32_t v) {
    mirror();
    auto it = std::lower_bound(head.begin(), head.end(), v);
    return (it != head.end() && *it == v) ? (long)(it - head.begin()) : -1;
  }
};

// the layout hybrid::build would pick (layouts/hybrid.hpp:103-111)
inline uint8_t hybrid_layout(const uint32_t* p, size_t n) {
  const size_t range = n > 1 ? (size_t)(p[n - 1] - p[0]) : 0;
  return common::is_sparse(n, range) ? (uint8_t)EH_LAYOUT_UINTEGER : (uint8_t)EH_LAYOUT_RANGE_BITSET;
}

// |A ∩ B| and its elements, on the device (ops::set_intersect,
// trie/set/ops/intersection/set.hpp:9-167)
inline void intersect(const uint32_t* a, size_t na, const uint32_t* b, size_t nb, std::vector<uint32_t>& out) {
  out.clear();
  if (!na || !nb) return;
  std::vector<uint32_t> elems(na + nb);
  std::copy(a, a + na, elems.begin());
  std::copy(b, b + nb, elems.begin() + na);
  const uint64_t set_off[3] = {0, na, na + nb};
  const uint8_t lay[2] = {hybrid_layout(a, na), hybrid_layout(b, nb)};
  const uint32_t pa = 0, pb = 1;
  uint64_t count = 0, out_off = 0;
  out.resize(std::min(na, nb));
  check(eh_set_intersect_batch(context(), elems.data(), set_off, 2, lay, &pa, &pb, 1, &count, &out_off, out.data()),
        "eh_set_intersect_batch");
  out.resize(count);
}

// ------------------------------------------------- accessors and the trace
// One accessor per ParTrieIterator (an atom of the bag's rule body).
struct Accessor {
  Relation* rel = nullptr;  // binary relation on the device, or null
  // unary annotated relation: its annotation by value (uint64 bit patterns)
  std::function<void(std::vector<uint64_t>&)> z_by_value;
  const void* unary_key = nullptr;  // identity of the unary relation
};
inline std::vector<Accessor>& accessors() {
  static std::vector<Accessor> a;
  return a;
}

enum Mode { REAL = 0, TRACE = 1, REPLAY = 2 };
// placeholder values the symbolic pass hands to loops: attribute k gets kPlaceholder + k
constexpr uint32_t kPlaceholder = 0xFFFFFF00u;
inline bool is_placeholder(uint32_t v) { return v >= kPlaceholder; }

struct Use {
  int l0 = -1, l1 = -1;    // attribute whose build read level 0 / level 1
  int desc = -1;           // attribute of get_next_block(0, .)
  std::vector<int> annot;  // attributes of get_annotation(0, .)
};

struct State {
  Mode mode = REAL;
  // TRACE
  int attr = 0;              // attribute the current builds produce
  std::map<int, Use> use;    // per accessor
  struct Value {
    bool build;
    bool looped;
  };
  std::vector<Value> values;  // value reads in call order
  bool ok = true;
  std::string why;
  bool wrote_annotation = false;
  bool inner_materialize = false;
  // REPLAY
  int carrier = -1;
  int seen = 0;
  uint64_t carried = 0;
};
inline State& state() {
  static State s;
  return s;
}
inline void fail_trace(const std::string& why) {
  State& s = state();
  if (s.ok) s.why = why;
  s.ok = false;
}

// a value read in TRACE / REPLAY: returns what the generated code sees
inline uint64_t value_read(bool build) {
  State& s = state();
  if (s.mode == TRACE) {
    s.values.push_back({build, false});
    return 0;
  }
  const int k = s.seen++;
  return k == s.carrier ? s.carried : 1;
}

}  // namespace ehd

// ------------------------------------------------------------------- Set
template <class T>
class Set {
 public:
  uint32_t cardinality = 0;
  uint32_t range = 0;
  size_t number_of_bytes = 0;
  type::layout type = type::NOT_VALID;
  const uint32_t* elems = nullptr;  // sorted elements (host)
  std::shared_ptr<std::vector<uint32_t>> store;  // owned elements of a set ops:: produced

  Set() {}
  void view(const uint32_t* p, size_t n) {
    elems = p;
    cardinality = (uint32_t)n;
    range = n ? p[n - 1] : 0;  // Set::from_array (Set.hpp:164-172)
    const bool dense = !common::is_sparse(n, n > 1 ? (size_t)(p[n - 1] - p[0]) : 0);
    type = dense ? type::RANGE_BITSET : type::UINTEGER;
    number_of_bytes = dense ? (size_t)((p[n - 1] >> 6) - (p[0] >> 6) + 1) * 12 + 8 : 4 * n;
  }
  uint8_t* get_data() const { return (uint8_t*)elems; }
  long find(uint32_t key) const {
    const uint32_t* e = std::lower_bound(elems, elems + cardinality, key);
    return (e != elems + cardinality && *e == key) ? (long)(e - elems) : -1;
  }
  template <typename F>
  void foreach (F f) const {
    for (uint32_t i = 0; i < cardinality; i++) f(elems[i]);
  }
  template <typename F>
  void foreach_index(F f) const {
    for (uint32_t i = 0; i < cardinality; i++) f(i, elems[i]);
  }
  template <typename F>
  size_t par_foreach(F f) const {
    for (uint32_t i = 0; i < cardinality; i++) f((size_t)0, elems[i]);
    return cardinality;
  }
  template <typename F>
  size_t par_foreach_index(F f) const {
    for (uint32_t i = 0; i < cardinality; i++) f((size_t)0, i, elems[i]);
    return cardinality;
  }
};

// ------------------------------------------------------------------- ops
// ops::set_intersect (trie/set/ops/intersection/set.hpp:9-167), all four
// forms with the reference's overload shapes (the plain forms are not
// templates, so a call with three set pointers picks the materialising one),
// over the layer's host set views: A ∩ B is computed on the device
// (eh_set_intersect_batch, whatever the sets' layouts); the materialising
// forms give C its own storage of the result (sorted, its layout by the
// density rule, as hybrid::build picks it), and the callback forms call
// f(x, index of x in A, index of x in B) for every element in order, as the
// reference's do.  For host code over sets already read (a Trie's foreach,
// the blocks an iterator returns); inside a bag's lambda the builders'
// build_aggregated_set is the entry the generated code uses.
namespace ops {
namespace detail {
template <class T>
inline std::vector<uint32_t> intersect(const Set<T>* A, const Set<T>* B) {
  std::vector<uint32_t> out;
  ehd::intersect(A->elems, A->cardinality, B->elems, B->cardinality, out);
  return out;
}
template <class T, typename F>
inline void each(const Set<T>* A, const Set<T>* B, const std::vector<uint32_t>& r, F& f) {
  uint32_t ia = 0, ib = 0;
  for (const uint32_t x : r) {  // both sets are sorted and x is in both
    while (A->elems[ia] < x) ia++;
    while (B->elems[ib] < x) ib++;
    f(x, ia, ib);
  }
}
template <class T>
inline Set<T>* own(Set<T>* C, std::vector<uint32_t>&& r) {
  C->store = std::make_shared<std::vector<uint32_t>>(std::move(r));
  C->view(C->store->data(), C->store->size());
  if (!C->cardinality) {
    C->type = type::UINTEGER;
    C->number_of_bytes = 0;
  }
  return C;
}
}  // namespace detail

template <typename F>
inline Set<hybrid>* set_intersect(Set<hybrid>* C, const Set<hybrid>* A, const Set<hybrid>* B, F f) {
  std::vector<uint32_t> r = detail::intersect(A, B);
  detail::each(A, B, r, f);
  return detail::own(C, std::move(r));
}
inline Set<hybrid>* set_intersect(Set<hybrid>* C, const Set<hybrid>* A, const Set<hybrid>* B) {
  return detail::own(C, detail::intersect(A, B));
}
template <typename F>
inline size_t set_intersect(const Set<hybrid>* A, const Set<hybrid>* B, F f) {
  const std::vector<uint32_t> r = detail::intersect(A, B);
  detail::each(A, B, r, f);
  return r.size();
}
inline size_t set_intersect(const Set<hybrid>* A, const Set<hybrid>* B) {
  return detail::intersect(A, B).size();
}
}  // namespace ops

// --------------------------------------------------------------- TrieBlock
// A set of a trie level as the generated code sees it, tagged with the
// accessor and level it was reached through (the symbolic pass reads the
// tags, not the set).
template <class T, class M>
struct TrieBlock {
  bool is_sparse = true;
  Set<T> set;
  int acc = -1;
  int level = 0;
  TrieBlock() {}
  const Set<T>* get_const_set() const { return &set; }
  Set<T>* get_set() const { return const_cast<Set<T>*>(&set); }
  bool contains(uint32_t data) const { return set.find(data) != -1; }
};

namespace ehd {

// Host node of a trie the layer holds on the host: outputs of bags
// (TrieBuilder::build_set / set_level / set_annotation) and annotated
// one-column inputs.
template <class A>
struct Node {
  std::vector<uint32_t> set;
  std::vector<A> annot;
  std::vector<std::unique_ptr<Node>> child;
};

template <class A>
inline uint64_t bits_of(A v) {
  uint64_t u = 0;
  std::memcpy(&u, &v, sizeof(A) < 8 ? sizeof(A) : 8);
  if (sizeof(A) < 8 && (A)(-1) < (A)0) {  // sign-extend narrower signed integers
    int64_t s = (int64_t)v;
    std::memcpy(&u, &s, 8);
  }
  return u;
}
template <>
inline uint64_t bits_of<void*>(void*) {
  return 0;
}

// A value of the annotation type from the device's uint64 bit pattern
template <class A>
inline A from_bits(uint64_t u) {
  int64_t s;
  std::memcpy(&s, &u, 8);
  return (A)s;
}
template <>
inline void* from_bits<void*>(uint64_t) {
  return nullptr;
}

}  // namespace ehd

// -------------------------------------------------------------------- Trie
template <class A, class M>
struct Trie {
  bool annotated = false;
  size_t num_rows = 0;
  size_t num_columns = 0;
  M* memoryBuffers = nullptr;
  std::vector<void*> encodings;
  A annotation = A();
  std::string path;
  // a relation on the device (two columns), or a host trie (outputs, one
  // annotated column)
  std::shared_ptr<ehd::Relation> rel;
  std::unique_ptr<ehd::Node<A>> root;
  TrieBlock<hybrid, M> head_block;

  Trie() {}
  Trie(bool annotated_in, A annotation_in, size_t num_rows_in, size_t num_columns_in, M* buf_in)
      : annotated(annotated_in), num_rows(num_rows_in), num_columns(num_columns_in), memoryBuffers(buf_in) {
    (void)annotation_in;
    annotation = (A)0;
    root.reset(new ehd::Node<A>());
  }
  // an output trie of a bag (EHGenerator.scala:246-271)
  Trie(std::string path_in, size_t num_columns_in, bool annotated_in)
      : annotated(annotated_in), num_columns(num_columns_in), path(path_in) {
    root.reset(new ehd::Node<A>());
  }
  // Trie<A,M>::Trie(path, max_set_sizes, attr_in, annotations)
  // (storage_engine/src/Trie.cpp:380-510): two columns build a device trie;
  // one column (with or without annotations) a host one-level trie.
  Trie(std::string path_in, std::vector<uint32_t>* max_set_sizes, std::vector<std::vector<uint32_t>>* attr_in,
       std::vector<A>* annotation_in)
      : path(path_in) {
    (void)max_set_sizes;
    num_columns = attr_in->size();
    if (num_columns == 2) {
      if (annotation_in && !annotation_in->empty())
        throw std::runtime_error("annotated binary relations are not supported by the B200 layer");
      const std::vector<uint32_t>& c0 = attr_in->at(0);
      const std::vector<uint32_t>& c1 = attr_in->at(1);
      if (c0.size() != c1.size()) throw std::runtime_error("columns differ in length");
      eh_trie* t = nullptr;
      ehd::check(eh_trie_build(ehd::context(), c0.data(), c1.data(), c0.size(), 0, nullptr, &t), "eh_trie_build");
      rel = std::make_shared<ehd::Relation>(t);
      num_rows = rel->rows;
      annotated = false;
    } else if (num_columns == 1) {
      const std::vector<uint32_t>& c0 = attr_in->at(0);
      std::vector<size_t> order(c0.size());
      for (size_t i = 0; i < order.size(); i++) order[i] = i;
      std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return c0[x] < c0[y]; });
      root.reset(new ehd::Node<A>());
      annotated = annotation_in && !annotation_in->empty();
      for (size_t k = 0; k < order.size(); k++) {
        const uint32_t v = c0[order[k]];
        if (!root->set.empty() && root->set.back() == v) continue;
        root->set.push_back(v);
        if (annotated) root->annot.push_back(annotation_in->at(order[k]));
      }
      num_rows = root->set.size();
    } else {
      throw std::runtime_error("the B200 layer builds tries of one or two columns");
    }
  }
  ~Trie() {}
  Trie(const Trie&) = delete;
  Trie& operator=(const Trie&) = delete;

  TrieBlock<hybrid, M>* getHead() {
    if (rel) {
      rel->mirror();
      head_block.set.view(rel->head.data(), rel->head.size());
    } else {
      head_block.set.view(root->set.data(), root->set.size());
    }
    head_block.is_sparse = common::is_sparse(head_block.set.cardinality, head_block.set.range);
    return &head_block;
  }

  // Trie::foreach (Trie.cpp:130-160): every tuple in order, with its annotation
  void foreach (const std::function<void(std::vector<uint32_t>*, A)> body) {
    std::vector<uint32_t> tuple;
    if (rel) {
      rel->mirror();
      tuple.resize(2);
      for (uint32_t i = 0; i < rel->n_head; i++)
        for (uint64_t e = rel->off[i]; e < rel->off[i + 1]; e++) {
          tuple[0] = rel->head[i];
          tuple[1] = rel->vals[e];
          body(&tuple, annotation);
        }
      return;
    }
    walk(root.get(), tuple, body);
  }

  // Trie::save (Trie.cpp:15-35) for device relations, in the reference's
  // on-disk format with one buffer per thread of the loading engine
  void save() {
    if (!rel) throw std::runtime_error("the B200 layer saves device relations only");
    mkdir(path.c_str(), 0755);
    ehd::check(eh_trie_save_reference(ehd::context(), rel->trie, path.c_str(), (uint32_t)NUM_THREADS),
               "eh_trie_save_reference");
  }

  // Trie<A,M>::load (Trie.cpp:37-75) of a two-level relation the reference saved
  static Trie<A, M>* load(std::string path_in) {
    eh_trie* t = nullptr;
    ehd::check(eh_trie_load_reference(ehd::context(), path_in.c_str(), nullptr, &t), "eh_trie_load_reference");
    Trie<A, M>* out = new Trie<A, M>();
    out->path = path_in;
    out->num_columns = 2;
    out->rel = std::make_shared<ehd::Relation>(t);
    out->num_rows = out->rel->rows;
    return out;
  }

 private:
  void walk(const ehd::Node<A>* n, std::vector<uint32_t>& tuple,
            const std::function<void(std::vector<uint32_t>*, A)>& body) {
    if (!n) return;
    for (size_t i = 0; i < n->set.size(); i++) {
      tuple.push_back(n->set[i]);
      const bool leaf = i >= n->child.size() || !n->child[i];
      if (leaf) body(&tuple, i < n->annot.size() ? n->annot[i] : annotation);
      else walk(n->child[i].get(), tuple, body);
      tuple.pop_back();
    }
  }
};

// ------------------------------------------------------------ TrieIterator
template <class A, class M>
struct TrieIterator {
  Trie<A, M>* trie;
  std::vector<const TrieBlock<layout, M>*> levels;
  size_t num_rows = 0;
  int a[300];  // padding, as in the reference
  // the layer's own copies of the blocks it points at, tagged with the accessor
  std::vector<TrieBlock<hybrid, M>> slots;
  std::vector<const ehd::Node<A>*> nodes;  // host tries: the node of each level
  int acc = -1;

  explicit TrieIterator(Trie<A, M>* t_in, int acc_in = -1) : trie(t_in), acc(acc_in) {
    const size_t n = std::max<size_t>(trie->num_columns, 1);
    levels.assign(n, nullptr);
    slots.resize(n);
    nodes.assign(n, nullptr);
    for (size_t l = 0; l < n; l++) {
      slots[l].acc = acc;
      slots[l].level = (int)l;
    }
    if (trie->num_columns > 0) reset_head(trie->getHead());
    (void)a;
  }
  void reset_head(const TrieBlock<hybrid, M>* h) {
    if (!h) {
      levels[0] = nullptr;
      return;
    }
    slots[0].set = h->set;
    slots[0].is_sparse = h->is_sparse;
    slots[0].acc = acc;
    slots[0].level = h->level;
    levels[0] = &slots[0];
    nodes[0] = trie->rel ? nullptr : trie->root.get();
  }

  // TrieIterator::get_next_block(level, data) (TrieIterator.cpp:24-28)
  void get_next_block(const size_t level, const uint32_t data) {
    ehd::State& st = ehd::state();
    if (level + 1 >= levels.size()) throw std::runtime_error("get_next_block past the trie's last level");
    if (st.mode == ehd::TRACE) {
      if (!ehd::is_placeholder(data)) ehd::fail_trace("descent by a value that is not a loop variable");
      else if (level != 0) ehd::fail_trace("descent below level 1");
      else st.use[acc].desc = (int)(data - ehd::kPlaceholder);
      slots[level + 1].acc = acc;
      slots[level + 1].level = (int)level + 1;
      slots[level + 1].set = Set<hybrid>();
      levels[level + 1] = &slots[level + 1];
      return;
    }
    if (st.mode == ehd::REPLAY) {
      levels[level + 1] = &slots[level + 1];
      return;
    }
    levels[level + 1] = nullptr;
    const TrieBlock<hybrid, M>* cur = levels[level];
    if (!cur) return;
    const long i = cur->set.find(data);
    if (i < 0) return;
    TrieBlock<hybrid, M>& nb = slots[level + 1];
    nb.acc = acc;
    nb.level = (int)level + 1;
    if (trie->rel) {
      if (level != 0 || cur->level != 0) throw std::runtime_error("a binary relation has two levels");
      ehd::Relation& r = *trie->rel;
      r.mirror();
      nb.set.view(r.vals.data() + r.off[i], r.off[i + 1] - r.off[i]);
    } else {
      const ehd::Node<A>* n = nodes[level];
      if (!n || (size_t)i >= n->child.size() || !n->child[i]) return;
      nodes[level + 1] = n->child[i].get();
      nb.set.view(nodes[level + 1]->set.data(), nodes[level + 1]->set.size());
    }
    nb.is_sparse = common::is_sparse(nb.set.cardinality, nb.set.range);
    levels[level + 1] = &nb;
  }
  void get_next_block(const size_t level, const uint32_t index, const uint32_t data) {
    (void)index;
    get_next_block(level, data);
  }

  // TrieIterator::get_annotation (TrieIterator.cpp:45-59): 0 when absent
  A get_annotation(const size_t level, const uint32_t data) {
    ehd::State& st = ehd::state();
    if (st.mode == ehd::TRACE) {
      if (level != 0 || !ehd::is_placeholder(data)) ehd::fail_trace("annotation read below the head");
      else st.use[acc].annot.push_back((int)(data - ehd::kPlaceholder));
      ehd::value_read(false);
      return (A)0;
    }
    if (st.mode == ehd::REPLAY) return ehd::from_bits<A>(ehd::value_read(false));
    const TrieBlock<hybrid, M>* b = levels[level];
    const ehd::Node<A>* n = nodes[level];
    if (!b || !n) return (A)0;
    const long i = b->set.find(data);
    if (i < 0 || (size_t)i >= n->annot.size()) return (A)0;
    return n->annot[i];
  }

  const TrieBlock<hybrid, M>* get_block(const size_t level) const { return levels.at(level); }
};

template <class A, class M>
struct ParTrieIterator {
  A annotation;
  TrieBlock<hybrid, M>* head;
  Trie<A, M>* trie;
  std::vector<TrieIterator<A, M>*> iterators;
  TrieBlock<hybrid, M> head_slot;
  int acc;

  explicit ParTrieIterator(Trie<A, M>* t_in) : annotation(t_in->annotation), trie(t_in) {
    // register the accessor (one atom of the bag)
    ehd::Accessor info;
    if (t_in->rel) {
      info.rel = t_in->rel.get();
    } else if (t_in->annotated && t_in->num_columns == 1) {
      Trie<A, M>* tp = t_in;
      info.unary_key = tp;
      info.z_by_value = [tp](std::vector<uint64_t>& z) {
        const ehd::Node<A>* r = tp->root.get();
        const uint32_t n = r->set.empty() ? 0 : r->set.back() + 1;
        z.assign(n, 0);
        for (size_t i = 0; i < r->set.size() && i < r->annot.size(); i++) z[r->set[i]] = ehd::bits_of<A>(r->annot[i]);
      };
    }
    ehd::accessors().push_back(info);
    acc = (int)ehd::accessors().size() - 1;
    head_slot = *t_in->getHead();
    head_slot.acc = acc;
    head_slot.level = 0;
    head = &head_slot;
    for (size_t i = 0; i < NUM_THREADS; i++) iterators.push_back(new TrieIterator<A, M>(t_in, acc));
  }
  ~ParTrieIterator() {
    for (auto* it : iterators) delete it;
  }
  ParTrieIterator(const ParTrieIterator&) = delete;
  ParTrieIterator& operator=(const ParTrieIterator&) = delete;

  // ParTrieIterator::get_next_block(data) (TrieIterator.cpp:72-78): the head
  // moves to data's child set (NULL when data heads none)
  void get_next_block(const uint32_t data) {
    if (!head) return;
    const long i = head->set.find(data);
    if (i < 0 || !trie->rel || head->level != 0) {
      head = nullptr;
    } else {
      ehd::Relation& r = *trie->rel;
      r.mirror();
      head_slot.set.view(r.vals.data() + r.off[i], r.off[i + 1] - r.off[i]);
      head_slot.level = 1;
      head_slot.is_sparse = common::is_sparse(head_slot.set.cardinality, head_slot.set.range);
      head = &head_slot;
    }
    for (auto* it : iterators) it->reset_head(head);
  }
};

// ---------------------------------------------------------------- par
namespace par {
// par::reducer (utils/parallel.hpp:8-34): one padded slot per thread,
// starting at zero like the reference's (it memsets after storing init)
template <class T>
class reducer {
 public:
  T* elem;
  std::function<T(T, T)> f;
  reducer(T init_in, std::function<T(T, T)> f_in) : f(f_in) {
    (void)init_in;
    elem = new T[NUM_THREADS * PADDING]();
  }
  ~reducer() { delete[] elem; }
  reducer(const reducer&) = delete;
  reducer& operator=(const reducer&) = delete;
  inline void update(size_t tid, T new_val) { elem[tid * PADDING] = f(elem[tid * PADDING], new_val); }
  inline void clear() {
    for (size_t i = 0; i < NUM_THREADS; i++) elem[i * PADDING] = T();
  }
  inline T evaluate(T init) {
    for (size_t i = 0; i < NUM_THREADS; i++) init = f(init, elem[i * PADDING]);
    return init;
  }
};
}  // namespace par

// ---------------------------------------------------------------- builders
template <class A, class M>
struct TrieBuilder {
  Trie<A, M>* trie;
  uint32_t cur_level = 1;
  uint32_t tmp_level = 0;
  std::vector<std::vector<uint32_t>> tmp;       // aggregate set per attribute level
  std::vector<const Set<hybrid>*> aggregate_sets;
  std::vector<Set<hybrid>> tmp_sets;
  std::vector<int> tmp_value;                   // TRACE: the value read of each level's last build
  // output levels: node[l] is the node whose set is being built at level l
  std::vector<ehd::Node<A>*> node;
  std::vector<std::unique_ptr<ehd::Node<A>>> pending;  // sets built by build_set, not yet linked

  TrieBuilder(Trie<A, M>* t_in, const size_t num_attributes) : trie(t_in) {
    const size_t n = std::max<size_t>(num_attributes, 1) + 1;
    tmp.resize(n);
    tmp_sets.resize(n);
    aggregate_sets.assign(n, nullptr);
    tmp_value.assign(n, -1);
    node.assign(std::max<size_t>(t_in->num_columns, 1) + 1, nullptr);
    pending.resize(node.size());
    node[0] = t_in->root.get();
  }

  // ---- aggregated sets (TrieBuilder.cpp:223-348)
  size_t build_aggregated_set(const TrieBlock<hybrid, M>* s1) {
    std::vector<const TrieBlock<hybrid, M>*> v{s1};
    return aggregate(v);
  }
  size_t build_aggregated_set(const TrieBlock<hybrid, M>* s1, const TrieBlock<hybrid, M>* s2) {
    std::vector<const TrieBlock<hybrid, M>*> v{s1, s2};
    return aggregate(v);
  }
  size_t build_aggregated_set(std::vector<const TrieBlock<hybrid, M>*>* isets) { return aggregate(*isets); }
  size_t build_aggregated_equality_selection_set(const TrieBlock<hybrid, M>* s1) { return build_aggregated_set(s1); }

  size_t count_set(const TrieBlock<hybrid, M>* s1) {
    if (ehd::state().mode != ehd::REAL) ehd::fail_trace("count_set inside a traced bag");
    if (!s1) return 0;
    return s1->set.cardinality;
  }
  size_t count_set(const TrieBlock<hybrid, M>* s1, const TrieBlock<hybrid, M>* s2) {
    if (ehd::state().mode != ehd::REAL) ehd::fail_trace("count_set inside a traced bag");
    if (!s1 || !s2) return 0;
    std::vector<uint32_t> r;
    ehd::intersect(s1->set.elems, s1->set.cardinality, s2->set.elems, s2->set.cardinality, r);
    return r.size();
  }

  template <typename F>
  inline void foreach_aggregate(F f) {
    ehd::State& st = ehd::state();
    if (st.mode == ehd::TRACE) {
      if (tmp_value[tmp_level] >= 0) st.values[tmp_value[tmp_level]].looped = true;
      const int a = st.attr;
      tmp_level++;
      st.attr = a + 1;
      f(ehd::kPlaceholder + (uint32_t)a);
      st.attr = a;
      tmp_level--;
      return;
    }
    if (st.mode == ehd::REPLAY) {
      tmp_level++;
      f(ehd::kPlaceholder);
      tmp_level--;
      return;
    }
    const std::vector<uint32_t> s = tmp.at(tmp_level);  // a copy: nested builds reuse deeper levels only
    tmp_level++;
    for (uint32_t x : s) f(x);
    tmp_level--;
  }

  // ---- materialized sets (TrieBuilder.cpp:44-221, 376-446)
  size_t build_set(const size_t tid, const TrieBlock<hybrid, M>* s1) {
    std::vector<const TrieBlock<hybrid, M>*> v{s1};
    return materialize(tid, v);
  }
  size_t build_set(const size_t tid, const TrieBlock<hybrid, M>* s1, const TrieBlock<hybrid, M>* s2) {
    std::vector<const TrieBlock<hybrid, M>*> v{s1, s2};
    return materialize(tid, v);
  }
  size_t build_set(const size_t tid, std::vector<const TrieBlock<hybrid, M>*>* isets) {
    return materialize(tid, *isets);
  }
  void allocate_next(const size_t tid) {
    (void)tid;
    if (ehd::state().mode != ehd::REAL) return;
    ehd::Node<A>* n = pending.at(cur_level).get();
    if (n) n->child.resize(n->set.size());
  }
  void allocate_annotation(const size_t tid) {
    (void)tid;
    if (ehd::state().mode != ehd::REAL) return;
    ehd::Node<A>* n = pending.at(cur_level).get();
    if (n) n->annot.assign(n->set.size(), A());
  }
  // links the set built at this level under element index of the level above
  void set_level(const uint32_t index, const uint32_t data) {
    (void)data;
    if (ehd::state().mode != ehd::REAL) return;
    ehd::Node<A>* parent = node.at(cur_level - 1);
    if (!parent || index >= parent->child.size()) return;
    parent->child[index] = std::move(pending.at(cur_level));
  }
  void set_annotation(const A value, const uint32_t index, const uint32_t data) {
    (void)data;
    ehd::State& st = ehd::state();
    if (st.mode == ehd::TRACE) {
      st.wrote_annotation = true;
      return;
    }
    ehd::Node<A>* n = node.at(cur_level - 1);
    if (n && index < n->annot.size()) n->annot[index] = value;
  }

  template <typename F>
  inline void foreach_builder(F f) {
    ehd::State& st = ehd::state();
    if (st.mode == ehd::TRACE) {
      if (tmp_value[tmp_level] >= 0) st.values[tmp_value[tmp_level]].looped = true;
      const int a = st.attr;
      cur_level++;
      st.attr = a + 1;
      f((uint32_t)0, ehd::kPlaceholder + (uint32_t)a);
      st.attr = a;
      cur_level--;
      return;
    }
    if (st.mode == ehd::REPLAY) throw std::runtime_error("a replayed bag materialises below its head");
    // iterate the set built at this level; sets built inside go one level down
    ehd::Node<A>* n = pending.at(cur_level).get();
    if (!n) return;
    node.at(cur_level) = n;
    cur_level++;
    for (uint32_t i = 0; i < n->set.size(); i++) f(i, n->set[i]);
    cur_level--;
  }

 private:
  // N-way intersection, smallest set first (TrieBuilder.cpp:276-348); the
  // result is the same set whatever the order
  static void intersect_all(std::vector<const TrieBlock<hybrid, M>*>& v, std::vector<uint32_t>& out) {
    out.clear();
    for (auto* b : v)
      if (!b) return;
    std::sort(v.begin(), v.end(), [](const TrieBlock<hybrid, M>* x, const TrieBlock<hybrid, M>* y) {
      return x->set.cardinality < y->set.cardinality;
    });
    out.assign(v[0]->set.elems, v[0]->set.elems + v[0]->set.cardinality);
    std::vector<uint32_t> nxt;
    for (size_t i = 1; i < v.size() && !out.empty(); i++) {
      ehd::intersect(out.data(), out.size(), v[i]->set.elems, v[i]->set.cardinality, nxt);
      out.swap(nxt);
    }
  }
  void trace_operands(const std::vector<const TrieBlock<hybrid, M>*>& v) {
    ehd::State& st = ehd::state();
    for (auto* b : v) {
      if (!b || b->acc < 0) {
        ehd::fail_trace("a build reads a set the layer cannot attribute to an accessor");
        continue;
      }
      ehd::Use& u = st.use[b->acc];
      int& slot = b->level == 0 ? u.l0 : u.l1;
      if (b->level > 1 || (slot >= 0 && slot != st.attr)) ehd::fail_trace("an accessor level is read at two attributes");
      slot = st.attr;
    }
  }
  size_t aggregate(std::vector<const TrieBlock<hybrid, M>*>& v) {
    ehd::State& st = ehd::state();
    if (st.mode == ehd::TRACE) {
      trace_operands(v);
      tmp_value[tmp_level] = (int)st.values.size();
      ehd::value_read(true);
      tmp[tmp_level].assign(1, ehd::kPlaceholder);
      return 0;
    }
    if (st.mode == ehd::REPLAY) {
      tmp[tmp_level].assign(1, ehd::kPlaceholder);
      return (size_t)ehd::value_read(true);
    }
    intersect_all(v, tmp[tmp_level]);
    tmp_sets[tmp_level].view(tmp[tmp_level].data(), tmp[tmp_level].size());
    aggregate_sets[tmp_level] = &tmp_sets[tmp_level];
    return tmp[tmp_level].size();
  }
  size_t materialize(size_t tid, std::vector<const TrieBlock<hybrid, M>*>& v) {
    (void)tid;
    ehd::State& st = ehd::state();
    if (st.mode == ehd::TRACE) {
      trace_operands(v);
      st.inner_materialize = true;
      tmp_value[tmp_level] = (int)st.values.size();
      ehd::value_read(true);
      return 0;
    }
    if (st.mode == ehd::REPLAY) return (size_t)ehd::value_read(true);
    std::unique_ptr<ehd::Node<A>> n(new ehd::Node<A>());
    intersect_all(v, n->set);
    const size_t c = n->set.size();
    pending.at(cur_level) = std::move(n);
    return c;
  }
};

template <class A, class M>
struct ParTrieBuilder {
  Trie<A, M>* trie;
  std::vector<TrieBuilder<A, M>*> builders;
  const TrieBlock<hybrid, M>* tmp_head = nullptr;
  size_t num_attributes;
  // the set the outer loop runs over and the accessors its build read
  std::vector<uint32_t> head_set;
  TrieBlock<hybrid, M> head_block;
  std::vector<std::pair<int, int>> head_reads;  // (accessor, level)

  ParTrieBuilder(Trie<A, M>* t_in, const size_t num_attributes_in) : trie(t_in), num_attributes(num_attributes_in) {
    for (size_t i = 0; i < NUM_THREADS; i++) builders.push_back(new TrieBuilder<A, M>(t_in, num_attributes));
  }
  ~ParTrieBuilder() {
    for (auto* b : builders) delete b;
  }
  ParTrieBuilder(const ParTrieBuilder&) = delete;
  ParTrieBuilder& operator=(const ParTrieBuilder&) = delete;

  size_t build_aggregated_set(const TrieBlock<hybrid, M>* s1) {
    std::vector<const TrieBlock<hybrid, M>*> v{s1};
    return head_build(v, false);
  }
  size_t build_aggregated_set(const TrieBlock<hybrid, M>* s1, const TrieBlock<hybrid, M>* s2) {
    std::vector<const TrieBlock<hybrid, M>*> v{s1, s2};
    return head_build(v, false);
  }
  size_t build_aggregated_set(std::vector<const TrieBlock<hybrid, M>*>* isets) { return head_build(*isets, false); }
  size_t build_aggregated_equality_selection_set(const uint32_t data, const TrieBlock<hybrid, M>* s1) {
    return s1 ? (size_t)s1->set.find(data) : (size_t)-1;
  }
  size_t build_set(const TrieBlock<hybrid, M>* s1) {
    std::vector<const TrieBlock<hybrid, M>*> v{s1};
    return head_build(v, true);
  }
  size_t build_set(const TrieBlock<hybrid, M>* s1, const TrieBlock<hybrid, M>* s2) {
    std::vector<const TrieBlock<hybrid, M>*> v{s1, s2};
    return head_build(v, true);
  }
  size_t build_set(std::vector<const TrieBlock<hybrid, M>*>* isets) { return head_build(*isets, true); }

  void allocate_next() { trie->root->child.resize(trie->root->set.size()); }
  void allocate_annotation() { trie->root->annot.assign(trie->root->set.size(), A()); }

  // the outer loop of an aggregating bag (TrieBuilder.hpp:152-157)
  template <typename F>
  void par_foreach_aggregate(F f) {
    uint64_t value = 0;
    if (dispatch(false, [&] { f((size_t)0, ehd::kPlaceholder); }, &value, nullptr)) {
      replay_once(value, [&] { f((size_t)0, ehd::kPlaceholder); });
      return;
    }
    for (uint32_t x : head_set) f((size_t)0, x);
  }

  // the outer loop of a materialising bag over the output's head (TrieBuilder.hpp:159-164)
  template <typename F>
  void par_foreach_builder(F f) {
    std::vector<uint64_t> per;
    ehd::Node<A>* out = trie->root.get();
    for (auto* b : builders) b->node[0] = out;
    if (dispatch(true, [&] { f((size_t)0, (uint32_t)0, ehd::kPlaceholder); }, nullptr, &per)) {
      for (uint32_t i = 0; i < out->set.size(); i++) replay_once(per[i], [&] { f((size_t)0, i, out->set[i]); });
      return;
    }
    for (uint32_t i = 0; i < out->set.size(); i++) f((size_t)0, i, out->set[i]);
  }

 private:
  size_t head_build(std::vector<const TrieBlock<hybrid, M>*>& v, bool materialize) {
    head_reads.clear();
    for (auto* b : v)
      if (b) head_reads.push_back({b->acc, b->level});
    head_set.clear();
    bool null_in = false;
    for (auto* b : v) null_in = null_in || !b;
    if (!null_in) {
      std::sort(v.begin(), v.end(), [](const TrieBlock<hybrid, M>* x, const TrieBlock<hybrid, M>* y) {
        return x->set.cardinality < y->set.cardinality;
      });
      head_set.assign(v[0]->set.elems, v[0]->set.elems + v[0]->set.cardinality);
      std::vector<uint32_t> nxt;
      for (size_t i = 1; i < v.size() && !head_set.empty(); i++) {
        ehd::intersect(head_set.data(), head_set.size(), v[i]->set.elems, v[i]->set.cardinality, nxt);
        head_set.swap(nxt);
      }
    }
    head_block.set.view(head_set.data(), head_set.size());
    tmp_head = &head_block;
    if (materialize) {
      trie->root->set = head_set;
      trie->root->child.clear();
      trie->root->annot.clear();
    }
    return head_set.size();
  }

  template <typename G>
  void replay_once(uint64_t value, G g) {
    ehd::State& st = ehd::state();
    st.mode = ehd::REPLAY;
    st.seen = 0;
    st.carried = value;
    builders.at(0)->tmp_level = 0;
    builders.at(0)->cur_level = 1;
    try {
      g();
    } catch (...) {
      st.mode = ehd::REAL;
      throw;
    }
    st.mode = ehd::REAL;
  }

  // The symbolic pass (trace_call runs the lambda once on placeholders)
  // and the match against the device plans; true when the device computed
  // the bag (value: the aggregate; per: per element of the output head of
  // a materialising bag).
  bool dispatch(bool materializing, const std::function<void()>& trace_call, uint64_t* value,
                std::vector<uint64_t>* per);
};

// ----------------------------------------------------------- the dispatch
namespace ehd {

struct Atom {
  int acc, v0, v1;
};

// the body a trace describes: binary atoms over one device relation, and
// annotated unary atoms; false when the trace has a shape no plan takes
inline bool trace_body(const State& st, size_t n_attrs, Relation** rel, std::vector<Atom>& bin,
                       std::vector<Atom>& un) {
  if (!st.ok) return false;
  *rel = nullptr;
  for (const auto& kv : st.use) {
    const Accessor& a = accessors().at(kv.first);
    const Use& u = kv.second;
    if (a.rel) {
      if (u.l0 < 0 || u.l1 < 0 || !u.annot.empty()) return false;
      if (u.desc != u.l0) return false;
      if (*rel && *rel != a.rel) return false;
      *rel = a.rel;
      bin.push_back({kv.first, u.l0, u.l1});
    } else if (a.z_by_value) {
      if (u.l0 < 0 || u.l1 >= 0 || u.annot.empty()) return false;
      for (int x : u.annot)
        if (x != u.l0) return false;
      un.push_back({kv.first, u.l0, -1});
    } else {
      return false;
    }
  }
  for (const auto& x : bin)
    if (x.v0 >= (int)n_attrs || x.v1 >= (int)n_attrs) return false;
  return *rel != nullptr;
}

// the value read that carries the device's aggregate in the replay: the
// last one that is not a loop's set
inline int carrier_of(const State& st) {
  for (int i = (int)st.values.size() - 1; i >= 0; i--)
    if (!(st.values[i].build && st.values[i].looped)) return i;
  return -1;
}

}  // namespace ehd

template <class A, class M>
bool ParTrieBuilder<A, M>::dispatch(bool materializing, const std::function<void()>& trace_call, uint64_t* value,
                                    std::vector<uint64_t>* per) {
  if (getenv("EH_DROPIN_HOST_LOOP")) return false;  // the host loop for every bag (tests compare both)
  ehd::State& st = ehd::state();
  st = ehd::State();
  st.mode = ehd::TRACE;
  for (const auto& r : head_reads) {
    if (r.first < 0 || r.second > 1) {
      ehd::fail_trace("the outer build reads a set of no accessor");
      continue;
    }
    ehd::Use& u = st.use[r.first];
    (r.second == 0 ? u.l0 : u.l1) = 0;
  }
  TrieBuilder<A, M>* b = builders.at(0);
  b->tmp_level = 0;
  b->cur_level = 1;
  st.attr = 1;
  try {
    trace_call();
  } catch (const std::exception& e) {
    ehd::fail_trace(e.what());
  }
  st.mode = ehd::REAL;
  b->tmp_level = 0;
  b->cur_level = 1;
  std::fill(b->tmp_value.begin(), b->tmp_value.end(), -1);

  ehd::Relation* rel = nullptr;
  std::vector<ehd::Atom> bin, un;
  if (!ehd::trace_body(st, num_attributes, &rel, bin, un)) return false;
  st.carrier = ehd::carrier_of(st);
  if (st.carrier < 0 || st.inner_materialize) return false;
  eh_context* ctx = ehd::context();
  if (!materializing) {
    if (st.wrote_annotation) return false;
    uint64_t result = 0;
    if (un.empty()) {
      // one binary relation: a COUNT rule body the device matches up to renaming
      std::vector<eh_atom> atoms;
      for (const auto& x : bin) atoms.push_back(eh_atom{0u, (uint32_t)x.v0, (uint32_t)x.v1});
      eh_rule rule{(uint32_t)num_attributes, (uint32_t)atoms.size(), atoms.data(), -1, 0u};
      const eh_trie* tries[1] = {rel->trie};
      int q = -1;
      const eh_status s = eh_rule_count(ctx, tries, 1, &rule, nullptr, &result, &q, nullptr);
      if (s == EH_ERR_UNSUPPORTED) return false;
      ehd::check(s, "eh_rule_count");
    } else {
      // the lollipop / barbell root: Edge(a,x) joined with annotated unary bags
      if (num_attributes != 2 || bin.size() != 1 || bin[0].v0 != 0 || bin[0].v1 != 1) return false;
      int query = -1;
      if (un.size() == 1 && un[0].v0 == 0) query = EH_QUERY_LOLLIPOP;
      if (un.size() == 2 && std::min(un[0].v0, un[1].v0) == 0 && std::max(un[0].v0, un[1].v0) == 1 &&
          ehd::accessors()[un[0].acc].unary_key == ehd::accessors()[un[1].acc].unary_key)
        query = EH_QUERY_BARBELL;
      if (query < 0) return false;
      std::vector<uint64_t> z;
      ehd::accessors()[un[0].acc].z_by_value(z);
      ehd::check(eh_query_weighted_root(ctx, rel->trie, query, z.empty() ? nullptr : z.data(), (uint32_t)z.size(),
                                        &result),
                 "eh_query_weighted_root");
    }
    *value = result;
    return true;
  }
  // bag(a; z) :- E(a,p), E(a,q), E(p,q): z(a) is the triangle annotation
  if (!st.wrote_annotation || !un.empty() || bin.size() != 3 || num_attributes != 3) return false;
  int from0 = 0, pq = 0;
  for (const auto& x : bin) {
    if (x.v0 == 0 && x.v1 != 0) from0++;
    else if (x.v0 != 0 && x.v1 != 0 && x.v0 != x.v1) pq++;
  }
  if (from0 != 2 || pq != 1) return false;
  {
    int p = -1, q = -1;
    for (const auto& x : bin)
      if (x.v0 == 0) (p < 0 ? p : q) = x.v1;
    if (p == q) return false;
    for (const auto& x : bin)
      if (x.v0 != 0 && !((x.v0 == p && x.v1 == q) || (x.v0 == q && x.v1 == p))) return false;
  }
  std::vector<uint64_t> T(rel->n_head ? rel->n_head : 1);
  ehd::check(eh_triangle_annotation(ctx, rel->trie, nullptr, T.data()), "eh_triangle_annotation");
  const ehd::Node<A>* out = trie->root.get();
  per->assign(out->set.size(), 0);
  for (size_t i = 0; i < out->set.size(); i++) {
    const long h = rel->find_head(out->set[i]);
    (*per)[i] = h >= 0 ? T[h] : 0;
  }
  return true;
}

// ------------------------------------------------------------ thread_pool
struct thread_pool {
  // the reference's pinned pthread pool (utils/thread_pool.hpp:16-41); the
  // device does the parallel work here, so these open and close the engine
  static void initializeThreadPool() { (void)ehd::context(); }
  static void deleteThreadPool() {}
};

#endif  // EH_DROPIN_HPP
