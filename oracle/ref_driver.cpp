/* Reference-engine driver for the CPU oracle and the timed CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled (by oracle/Makefile)
 * against the reference storage engine's own sources, which stay where they
 * lie; nothing here ships in the product.
 *
 * The Scala query compiler cannot run in this image (no JVM), so the
 * per-query C++ it would emit is written out here by hand, statement by
 * statement in the shape EHGenerator.scala emits for the plans pinned by
 * QueryPlannerTest.scala:
 *   - emitHeadParForeach  query_compiler/.../codegen/query/EHGenerator.scala:273-300
 *   - emitBuildCode       EHGenerator.scala:302-354
 *   - emitForeach         EHGenerator.scala:384-397
 *   - annotation code     EHGenerator.scala:399-480
 *   - bag wrapper         EHGenerator.scala:728-838
 * Plans: triangle / 4-clique one bag, order [a,b,(c),(d)]
 * (QueryPlannerTest.scala:78-96); lollipop / barbell two bags with an
 * annotated bag (QueryPlannerTest.scala:199-230, IROptimizerTest.scala:189).
 *
 * The bags themselves (the generated code) are in generated_bags.hpp, which
 * the B200 layer's test compiles too.
 *
 * Modes (all print one JSON line on stdout):
 *   eh_ref triangle|clique4|lollipop|barbell|path2 <edges> [repeats]
 *   eh_ref clique4_sel|barbell_sel <edges> <repeats> <value>
 *                                         the travis.py selection queries
 *                                         (x = value, p = value)
 *   eh_ref trie_dump <edges> <out.bin>      dump the reference trie
 *   eh_ref setops <pairs.bin> <out.bin>     per-pair ops::set_intersect
 *   eh_ref encode <cols.bin> <out.bin>      Encoding<T> build + encode_column
 *   eh_ref save <edges> <dir>               Trie::save of the Edge trie (dir/ram/)
 *   eh_ref load_triangle <dir>              Trie::load, then the TriangleAgg bag
 * <edges> is a .tsv (two uint32 columns) or an edge file written by the
 * project's graph generator ("EHEDGE01" header, u64 n, u32 src[n], u32 dst[n]).
 *
 * Values are dictionary-encoded before the trie build the way the
 * reference's loader does it: one order-preserving code per distinct value
 * over both columns (storage_engine/src/Encoding.cpp:21-48 assigns keys in
 * sorted value order).  The encoding here is a sort-unique + lower_bound
 * with the same result.
 */
#include <sys/stat.h>
#include <sys/time.h>
#include <sched.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <string>
#include <vector>

#include "Trie.hpp"
#include "TrieBuilder.hpp"
#include "TrieIterator.hpp"
#include "trie/TrieBlock.hpp"
#include "utils/thread_pool.hpp"
#include "utils/timer.hpp"

typedef ParMemoryBuffer MB;

std::size_t eh_ref_num_threads() {
  const char* e = getenv("EH_REF_THREADS");
  if (e && atoi(e) > 0) return (std::size_t)atoi(e);
  cpu_set_t set;
  CPU_ZERO(&set);
  if (sched_getaffinity(0, sizeof(set), &set) == 0) {
    int c = CPU_COUNT(&set);
    if (c > 0) return (std::size_t)std::min(c, 500);
  }
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (std::size_t)std::min(n, 500L) : 1;
}

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

/* ---------------------------------------------------------------- input */
static bool read_edges(const std::string& path, std::vector<uint32_t>& s, std::vector<uint32_t>& d) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  char magic[8] = {0};
  if (fread(magic, 1, 8, f) == 8 && memcmp(magic, "EHEDGE01", 8) == 0) {
    uint64_t n = 0;
    if (fread(&n, 8, 1, f) != 1) { fclose(f); return false; }
    s.resize(n); d.resize(n);
    if (n && (fread(s.data(), 4, n, f) != n || fread(d.data(), 4, n, f) != n)) { fclose(f); return false; }
    fclose(f);
    return true;
  }
  fseek(f, 0, SEEK_SET);
  unsigned long a, b;
  while (fscanf(f, "%lu %lu", &a, &b) == 2) { s.push_back((uint32_t)a); d.push_back((uint32_t)b); }
  fclose(f);
  return true;
}

/* order-preserving dictionary encoding over both columns; key_to_value
 * receives the distinct values in key order */
static uint32_t encode(std::vector<uint32_t>& s, std::vector<uint32_t>& d, std::vector<uint32_t>& key_to_value) {
  std::vector<uint32_t>& vals = key_to_value;
  vals = s;
  vals.insert(vals.end(), d.begin(), d.end());
  std::sort(vals.begin(), vals.end());
  vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
  bool identity = vals.empty() || (vals.front() == 0 && vals.back() + 1 == vals.size());
  if (!identity) {
    for (auto* col : {&s, &d})
      for (auto& x : *col) x = (uint32_t)(std::lower_bound(vals.begin(), vals.end(), x) - vals.begin());
  }
  return (uint32_t)vals.size();
}

/* Encoding::value_to_key.at(v) (EHGenerator.scala:657-667): the key of a
 * selection literal; a value absent from the relation is an error there
 * (std::map::at throws) and here */
static bool value_to_key(const std::vector<uint32_t>& key_to_value, uint32_t v, uint32_t* key) {
  auto it = std::lower_bound(key_to_value.begin(), key_to_value.end(), v);
  if (it == key_to_value.end() || *it != v) return false;
  *key = (uint32_t)(it - key_to_value.begin());
  return true;
}

static Trie<void*, MB>* build_edge_trie(const std::string& dir, std::vector<uint32_t>& s,
                                        std::vector<uint32_t>& d, uint32_t ndistinct) {
  mkdir(dir.c_str(), 0755);
  mkdir((dir + "/ram").c_str(), 0755);
  std::vector<std::vector<uint32_t>> cols(2);
  cols[0] = s;
  cols[1] = d;
  std::vector<uint32_t> max_set_size(2, ndistinct);
  std::vector<void*> annotation;  // Edge is not annotated
  return new Trie<void*, MB>(dir, &max_set_size, &cols, &annotation);
}

#include "generated_bags.hpp"

static void put(FILE* f, const void* p, size_t n) { fwrite(p, 1, n, f); }

/* Writes, for the head and for each child set: type, cardinality, range,
 * number_of_bytes and the layout bytes.  Layout bytes are the reference's
 * own: uinteger = sorted u32; range_bitset = [u64 start word][u64 words][u32
 * per-word rank] (layouts/range_bitset.hpp:123-157). */
static int trie_dump(Trie<void*, MB>* t, const char* outp) {
  FILE* f = fopen(outp, "wb");
  if (!f) return 1;
  TrieBlock<hybrid, MB>* head = t->getHead();
  const Set<hybrid>* hs = head->get_set();
  auto dump_set = [&](const Set<hybrid>* s) {
    uint8_t ty = (uint8_t)s->type;
    uint32_t card = s->cardinality, range = s->range;
    uint64_t nb = s->number_of_bytes;
    put(f, &ty, 1); put(f, &card, 4); put(f, &range, 4); put(f, &nb, 8);
    put(f, s->get_data(), nb);
  };
  dump_set(hs);
  hs->foreach_index([&](uint32_t a_i, uint32_t a_d) {
    TrieBlock<hybrid, MB>* nb = head->get_next_block(a_i, a_d, t->memoryBuffers);
    uint32_t v = a_d;
    uint8_t present = nb != NULL;
    put(f, &v, 4); put(f, &present, 1);
    if (nb) dump_set(nb->get_set());
  });
  fclose(f);
  return 0;
}

/* pairs file: u64 npairs, then per pair u32 na, u32 A[na], u32 nb, u32 B[nb].
 * out file, per pair: u8 typeA, u8 typeB, u64 bytesA, bytesA of layout A,
 * u64 count (aggregate mode), u8 result type, u32 n, u32 elems[n]
 * (materialize mode, elements via Set::foreach). */
static int setops(const char* inp, const char* outp) {
  FILE* f = fopen(inp, "rb");
  if (!f) return 1;
  uint64_t np = 0;
  if (fread(&np, 8, 1, f) != 1) { fclose(f); return 1; }
  FILE* o = fopen(outp, "wb");
  if (!o) { fclose(f); return 1; }
  std::vector<uint32_t> A, B;
  for (uint64_t p = 0; p < np; p++) {
    uint32_t na, nb;
    if (fread(&na, 4, 1, f) != 1) return 1;
    A.resize(na);
    if (na && fread(A.data(), 4, na, f) != na) return 1;
    if (fread(&nb, 4, 1, f) != 1) return 1;
    B.resize(nb);
    if (nb && fread(B.data(), 4, nb, f) != nb) return 1;
    const uint32_t ra = na ? A.back() - A.front() : 0, rb = nb ? B.back() - B.front() : 0;
    const size_t ba = hybrid::get_number_of_bytes(na, ra) + 64, bb = hybrid::get_number_of_bytes(nb, rb) + 64;
    std::vector<uint8_t> bufA(sizeof(Set<hybrid>) + ba, 0), bufB(sizeof(Set<hybrid>) + bb, 0);
    Set<hybrid>* sA = new (bufA.data()) Set<hybrid>();
    Set<hybrid>* sB = new (bufB.data()) Set<hybrid>();
    sA->from_array(sA->get_data(), A.data(), na);
    sB->from_array(sB->get_data(), B.data(), nb);
    /* result buffer sized the way TrieBuilder does it (TrieBuilder.cpp:15-24),
       with slack for the bitset result that starts at max(start words) */
    const size_t rbytes = std::max(ba, bb) * 2 + 256;
    std::vector<uint8_t> bufC(sizeof(Set<hybrid>) + rbytes, 0);
    Set<hybrid>* sC = new (bufC.data()) Set<hybrid>();
    const Set<hybrid>* cA = sA;
    const Set<hybrid>* cB = sB;
    const uint64_t cnt = ops::set_intersect(cA, cB);
    sC = ops::set_intersect(sC, cA, cB);
    std::vector<uint32_t> out;
    sC->foreach([&](uint32_t x) { out.push_back(x); });
    uint8_t ta = sA->type, tb = sB->type, tc = sC->type;
    uint64_t nba = sA->number_of_bytes;
    uint32_t nout = (uint32_t)out.size();
    put(o, &ta, 1); put(o, &tb, 1); put(o, &nba, 8); put(o, sA->get_data(), nba);
    put(o, &cnt, 8); put(o, &tc, 1); put(o, &nout, 4);
    if (nout) put(o, out.data(), 4 * (size_t)nout);
  }
  fclose(f);
  fclose(o);
  printf("{\"mode\": \"setops\", \"pairs\": %llu}\n", (unsigned long long)np);
  return 0;
}

/* ---- dictionary encoding with the reference's Encoding<T>
 * (Encoding.cpp:21-48): build over a std::set of every column's values,
 * then encode_column per column.  Input: u32 type (0 uint32, 1 int,
 * 2 long, 3 float), u32 n_cols, per column u64 n and n values.  Output:
 * u32 num_distinct, key_to_value[num_distinct], then u32 keys per column. */
#include "Encoding.hpp"
template <class T>
static int encode_typed(FILE* f, FILE* o, uint32_t n_cols) {
  std::vector<std::vector<T>> cols(n_cols);
  std::set<T> values;
  for (uint32_t c = 0; c < n_cols; c++) {
    uint64_t n = 0;
    if (fread(&n, 8, 1, f) != 1) return 1;
    cols[c].resize(n);
    if (n && fread(cols[c].data(), sizeof(T), n, f) != n) return 1;
    values.insert(cols[c].begin(), cols[c].end());
  }
  Encoding<T> enc;
  enc.build(&values);
  put(o, &enc.num_distinct, 4);
  for (uint32_t k = 0; k < enc.num_distinct; k++) put(o, &enc.key_to_value.at(k), sizeof(T));
  for (uint32_t c = 0; c < n_cols; c++) {
    std::vector<uint32_t>* keys = enc.encode_column(cols[c].data(), cols[c].size());
    if (!keys->empty()) put(o, keys->data(), 4 * keys->size());
    delete keys;
  }
  return 0;
}

static int encode_mode(const char* inp, const char* outp) {
  FILE* f = fopen(inp, "rb");
  if (!f) return 1;
  uint32_t hdr[2];
  if (fread(hdr, 4, 2, f) != 2) { fclose(f); return 1; }
  FILE* o = fopen(outp, "wb");
  if (!o) { fclose(f); return 1; }
  thread_pool::initializeThreadPool();
  int rc = 2;
  switch (hdr[0]) {
    case 0: rc = encode_typed<uint32_t>(f, o, hdr[1]); break;
    case 1: rc = encode_typed<int>(f, o, hdr[1]); break;
    case 2: rc = encode_typed<long>(f, o, hdr[1]); break;
    case 3: rc = encode_typed<float>(f, o, hdr[1]); break;
  }
  fclose(f);
  fclose(o);
  printf("{\"mode\": \"encode\", \"rc\": %d}\n", rc);
  fflush(stdout);
  _exit(rc);
}

static std::string scratch_dir() {
  const char* t = getenv("TMPDIR");
  std::string base = t ? t : "/tmp";
  char buf[64];
  snprintf(buf, sizeof buf, "/eh_ref_%d", (int)getpid());
  std::string d = base + buf;
  mkdir(d.c_str(), 0755);
  return d;
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: eh_ref triangle|clique4|lollipop|barbell <edges> [repeats]\n"
                    "       eh_ref clique4_sel|barbell_sel <edges> <repeats> <value>\n"
                    "       eh_ref trie_dump <edges> <out>\n       eh_ref setops <pairs> <out>\n");
    return 2;
  }
  const std::string mode = argv[1];
  if (mode == "setops") return argc > 3 ? setops(argv[2], argv[3]) : 2;
  if (mode == "encode") return argc > 3 ? encode_mode(argv[2], argv[3]) : 2;
  if (mode == "load_triangle") {
    /* Trie::load (Trie.cpp:37-75) of a saved Edge trie, then the TriangleAgg bag */
    thread_pool::initializeThreadPool();
    Trie<void*, MB>* loaded = Trie<void*, MB>::load(argv[2]);
    const std::string dir = scratch_dir();
    const long count = bag_triangle(loaded, dir + "/TriangleAgg");
    printf("{\"mode\": \"load_triangle\", \"count\": %ld, \"count_u64\": %llu, \"rows\": %zu, "
           "\"threads\": %zu}\n",
           count, (unsigned long long)(uint64_t)count, loaded->num_rows, NUM_THREADS);
    fflush(stdout);
    _exit(0);
  }

  std::vector<uint32_t> s, d;
  if (!read_edges(argv[2], s, d) || s.empty()) {
    fprintf(stderr, "cannot read edges from %s\n", argv[2]);
    return 1;
  }
  std::vector<uint32_t> key_to_value;
  const uint32_t nd = encode(s, d, key_to_value);
  const std::string dir = scratch_dir();
  thread_pool::initializeThreadPool();
  const double tb0 = now_s();
  Trie<void*, MB>* Trie_Edge_0_1 = build_edge_trie(dir + "/Edge_0_1", s, d, nd);
  /* selection plans read Edge(a,x) in order [x,a]: the relation's second
   * trie, columns swapped (createDB.scala builds one per attribute order) */
  const bool sel_mode = mode == "clique4_sel" || mode == "barbell_sel";
  Trie<void*, MB>* Trie_Edge_1_0 = sel_mode ? build_edge_trie(dir + "/Edge_1_0", d, s, nd) : nullptr;
  const double build_s = now_s() - tb0;
  uint32_t sel_key = 0;
  if (sel_mode) {
    const uint32_t sel_value = argc > 4 ? (uint32_t)strtoul(argv[4], nullptr, 10) : 0u;
    if (!value_to_key(key_to_value, sel_value, &sel_key)) {
      fprintf(stderr, "selection value %u is not in the relation\n", sel_value);
      return 1;
    }
  }

  if (mode == "save") {
    /* Trie::save (Trie.cpp:15-35) of the Edge trie into <dir>/ram/ */
    if (argc < 4) return 2;
    const std::string out = argv[3];
    Trie<void*, MB>* saved = build_edge_trie(out, s, d, nd);
    saved->save();
    printf("{\"mode\": \"save\", \"rows\": %zu, \"threads\": %zu}\n", s.size(), NUM_THREADS);
    fflush(stdout);
    _exit(0);
  }

  if (mode == "trie_dump") {
    int rc = argc > 3 ? trie_dump(Trie_Edge_0_1, argv[3]) : 2;
    printf("{\"mode\": \"trie_dump\", \"rows\": %zu, \"build_s\": %.6f}\n", s.size(), build_s);
    thread_pool::deleteThreadPool();
    return rc;
  }

  const int repeats = argc > 3 ? std::max(1, atoi(argv[3])) : 1;
  std::vector<double> times;
  long count = 0;
  for (int r = 0; r < repeats; r++) {
    auto query_timer = timer::start_clock();
    if (mode == "triangle") {
      count = bag_triangle(Trie_Edge_0_1, dir + "/TriangleAgg");
    } else if (mode == "clique4") {
      count = bag_clique4(Trie_Edge_0_1, dir + "/FliqueAgg");
    } else if (mode == "path2") {
      count = bag_path2(Trie_Edge_0_1, dir + "/PathAgg");
    } else if (mode == "lollipop" || mode == "barbell") {
      Trie<long, MB>* bag1 = bag_triangle_annot(Trie_Edge_0_1, dir + "/bag_1_a_b_c");
      count = mode == "lollipop" ? bag_lollipop_root(Trie_Edge_0_1, bag1, dir + "/LollipopAgg")
                                 : bag_barbell_root(Trie_Edge_0_1, bag1, dir + "/BarbellAgg");
      delete bag1;
    } else if (mode == "clique4_sel") {
      Trie<long, MB>* bag1 = bag_selected_partners(Trie_Edge_1_0, sel_key, dir + "/bag_1_x_a_FliqueSelAgg");
      count = bag1 ? bag_clique4_sel_root(Trie_Edge_0_1, bag1, dir + "/FliqueSelAgg") : 0;
      delete bag1;
    } else if (mode == "barbell_sel") {
      Trie<long, MB>* bag1 = bag_selected_partners(Trie_Edge_1_0, sel_key, dir + "/bag_1_p_a_BarbellSelAgg");
      Trie<long, MB>* bag2 = bag_selected_partners(Trie_Edge_0_1, sel_key, dir + "/bag_2_p_x_BarbellSelAgg");
      if (bag1 && bag2) {
        const long scalar = bag_triangle_sel_scalar(Trie_Edge_0_1, bag2, dir + "/bag_1_x_y_z_BarbellSelAgg");
        count = bag_barbell_sel_root(Trie_Edge_0_1, bag1, scalar, dir + "/BarbellSelAgg");
      } else {
        count = 0;
      }
      delete bag1;
      delete bag2;
    } else {
      fprintf(stderr, "unknown mode %s\n", mode.c_str());
      return 2;
    }
    times.push_back(timer::stop_clock(query_timer));
  }
  thread_pool::deleteThreadPool();
  std::vector<double> sorted(times);
  std::sort(sorted.begin(), sorted.end());
  printf("{\"mode\": \"%s\", \"count\": %ld, \"count_u64\": %llu, \"rows\": %zu, \"distinct\": %u, "
         "\"threads\": %zu, \"build_s\": %.6f, \"query_s_median\": %.9f, \"query_s\": [",
         mode.c_str(), count, (unsigned long long)(uint64_t)count, s.size(), nd, NUM_THREADS, build_s,
         sorted[sorted.size() / 2]);
  for (size_t i = 0; i < times.size(); i++) printf("%s%.9f", i ? ", " : "", times[i]);
  printf("]}\n");
  fflush(stdout);
  _exit(0); /* the reference's pool threads are parked; skip their teardown */
}
