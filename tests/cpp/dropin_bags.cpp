/* The reference's generated bag code compiled against the B200 layer.
 *
 * TEST PROGRAM.  It includes the drop-in headers of include/eh/ (Trie.hpp,
 * TrieBuilder.hpp, TrieIterator.hpp, trie/TrieBlock.hpp, ... under the
 * reference's names) and then oracle/generated_bags.hpp, the same
 * generated-shape bags oracle/ref_driver.cpp compiles against the reference
 * storage engine; it links against libeh_b200.so only.
 *
 *   dropin_bags <query> <edges.tsv> [value]
 *     query: triangle | clique4 | lollipop | barbell | path2, or
 *            clique4_sel | barbell_sel with the selection literal value
 *            (x = value, p = value; test/graph/travis.py:385-401, 472-487)
 *
 * The edge file is loaded the way the reference's loader does it: values
 * dictionary-encoded in ascending order (Encoding.cpp:21-48; the identity on
 * dense ids), then the Edge trie is built with
 * Trie<void*,MB>(path, max_set_sizes, attr_in, annotations)
 * (Trie.cpp:380-510).  Prints one JSON line: the count as the generated code
 * computed it (signed long) and its uint64 bit pattern.
 */
#include <sys/stat.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <cstring>
#include <string>
#include <vector>

#include "Trie.hpp"
#include "TrieBuilder.hpp"
#include "TrieIterator.hpp"
#include "trie/TrieBlock.hpp"
#include "utils/thread_pool.hpp"
#include "utils/timer.hpp"

typedef ParMemoryBuffer MB;

#include "generated_bags.hpp"

static bool read_tsv(const char* path, std::vector<uint32_t>& s, std::vector<uint32_t>& d) {
  FILE* f = fopen(path, "r");
  if (!f) return false;
  unsigned long a, b;
  while (fscanf(f, "%lu %lu", &a, &b) == 2) {
    s.push_back((uint32_t)a);
    d.push_back((uint32_t)b);
  }
  fclose(f);
  return true;
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: dropin_bags <query> <edges.tsv> [value]\n");
    return 2;
  }
  const std::string mode = argv[1];
  std::vector<uint32_t> s, d;
  if (!read_tsv(argv[2], s, d)) {
    fprintf(stderr, "cannot read %s\n", argv[2]);
    return 2;
  }
  // order-preserving dictionary encoding over both columns
  std::vector<uint32_t> key_to_value(s);
  key_to_value.insert(key_to_value.end(), d.begin(), d.end());
  std::sort(key_to_value.begin(), key_to_value.end());
  key_to_value.erase(std::unique(key_to_value.begin(), key_to_value.end()), key_to_value.end());
  for (auto* col : {&s, &d})
    for (auto& x : *col)
      x = (uint32_t)(std::lower_bound(key_to_value.begin(), key_to_value.end(), x) - key_to_value.begin());

  char tmpl[] = "/tmp/eh_dropin_XXXXXX";
  const std::string dir = mkdtemp(tmpl) ? std::string(tmpl) : std::string("/tmp");
  try {
    thread_pool::initializeThreadPool();
    std::vector<std::vector<uint32_t>> cols(2);
    cols[0] = s;
    cols[1] = d;
    std::vector<uint32_t> max_set_size(2, (uint32_t)key_to_value.size());
    std::vector<void*> annotation;
    auto t0 = timer::start_clock();
    Trie<void*, MB>* Trie_Edge_0_1 = new Trie<void*, MB>(dir + "/Edge_0_1", &max_set_size, &cols, &annotation);
    const double build_s = timer::stop_clock(t0);
    long count = 0;
    auto query_timer = timer::start_clock();
    if (mode == "triangle") {
      count = bag_triangle(Trie_Edge_0_1, dir + "/TriangleAgg");
    } else if (mode == "clique4") {
      count = bag_clique4(Trie_Edge_0_1, dir + "/FliqueAgg");
    } else if (mode == "path2") {
      count = bag_path2(Trie_Edge_0_1, dir + "/PathAgg");
    } else if (mode == "clique4_sel" || mode == "barbell_sel") {
      // the selection literal's key (Encoding::value_to_key.at, EHGenerator.scala:657-667)
      const uint32_t v = argc > 3 ? (uint32_t)strtoul(argv[3], nullptr, 10) : 0;
      auto it = std::lower_bound(key_to_value.begin(), key_to_value.end(), v);
      if (it == key_to_value.end() || *it != v) throw std::runtime_error("selection value not in the relation");
      const uint32_t sel = (uint32_t)(it - key_to_value.begin());
      std::vector<std::vector<uint32_t>> rcols(2);
      rcols[0] = d;
      rcols[1] = s;
      Trie<void*, MB>* Trie_Edge_1_0 = new Trie<void*, MB>(dir + "/Edge_1_0", &max_set_size, &rcols, &annotation);
      if (mode == "clique4_sel") {
        Trie<long, MB>* bag1 = bag_selected_partners(Trie_Edge_1_0, sel, dir + "/bag_1_x_a_FliqueSelAgg");
        count = bag1 ? bag_clique4_sel_root(Trie_Edge_0_1, bag1, dir + "/FliqueSelAgg") : 0;
        delete bag1;
      } else {
        Trie<long, MB>* bag1 = bag_selected_partners(Trie_Edge_1_0, sel, dir + "/bag_1_p_a_BarbellSelAgg");
        Trie<long, MB>* bag2 = bag_selected_partners(Trie_Edge_0_1, sel, dir + "/bag_2_p_x_BarbellSelAgg");
        if (bag1 && bag2) {
          const long scalar = bag_triangle_sel_scalar(Trie_Edge_0_1, bag2, dir + "/bag_1_x_y_z_BarbellSelAgg");
          count = bag_barbell_sel_root(Trie_Edge_0_1, bag1, scalar, dir + "/BarbellSelAgg");
        }
        delete bag1;
        delete bag2;
      }
      delete Trie_Edge_1_0;
    } else if (mode == "lollipop" || mode == "barbell") {
      Trie<long, MB>* bag1 = bag_triangle_annot(Trie_Edge_0_1, dir + "/bag_1_a_b_c");
      count = mode == "lollipop" ? bag_lollipop_root(Trie_Edge_0_1, bag1, dir + "/LollipopAgg")
                                 : bag_barbell_root(Trie_Edge_0_1, bag1, dir + "/BarbellAgg");
      delete bag1;
    } else {
      fprintf(stderr, "unknown query %s\n", mode.c_str());
      return 2;
    }
    const double query_s = timer::stop_clock(query_timer);
    delete Trie_Edge_0_1;
    thread_pool::deleteThreadPool();
    printf("{\"mode\": \"%s\", \"count\": %ld, \"count_u64\": %llu, \"rows\": %zu, \"build_s\": %.6f, "
           "\"query_s\": %.6f}\n",
           mode.c_str(), count, (unsigned long long)(uint64_t)count, s.size(), build_s, query_s);
  } catch (const std::exception& e) {
    printf("{\"mode\": \"%s\", \"error\": \"%s\"}\n", mode.c_str(), e.what());
    return 1;
  }
  return 0;
}
