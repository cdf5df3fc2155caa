/* ops::set_intersect of the drop-in layer (include/eh/eh_dropin.hpp).
 *
 * TEST PROGRAM.  dropin_setops: intersects fixed sorted sets with the four
 * forms of ops::set_intersect (materialise into C with and without a
 * callback; count with and without one) and prints one JSON line with the
 * results, the callback's (x, index in A, index in B) triples and C's
 * layout, for the test to compare against a restatement.
 */
#include <cstdio>
#include <string>
#include <vector>

#include "trie/set/Set.hpp"

static std::string list(const uint32_t* p, size_t n) {
  std::string s = "[";
  for (size_t i = 0; i < n; i++) s += (i ? ", " : "") + std::to_string(p[i]);
  return s + "]";
}

int main() {
  // a sparse list and a dense run: 300 elements over 256 values and a gap
  std::vector<uint32_t> a = {1, 5, 9, 64, 65, 300, 1000, 5000, 70000};
  std::vector<uint32_t> b;
  for (uint32_t v = 0; v < 256; v++) b.push_back(v);
  for (uint32_t v = 990; v < 1010; v++) b.push_back(v);
  b.push_back(70000);
  Set<hybrid> A, B, E, C1, C2;
  A.view(a.data(), a.size());
  B.view(b.data(), b.size());
  E.view(nullptr, 0);
  // inputs as const sets, as the reference's callers pass them
  // (TrieBuilder.cpp:108, 194, 268, 326): with three non-const pointers the
  // materialising and the callback-counting forms tie, there as here
  const Set<hybrid>* pa = &A;
  const Set<hybrid>* pb = &B;
  const Set<hybrid>* pe = &E;
  std::string triples = "[";
  bool first = true;
  auto f = [&](uint32_t x, uint32_t ia, uint32_t ib) {
    triples += std::string(first ? "" : ", ") + "[" + std::to_string(x) + ", " + std::to_string(ia) + ", " +
               std::to_string(ib) + "]";
    first = false;
  };
  ops::set_intersect(&C1, pa, pb, f);
  triples += "]";
  ops::set_intersect(&C2, pb, pa);
  size_t calls = 0;
  const size_t n_f = ops::set_intersect(pa, pb, [&](uint32_t, uint32_t, uint32_t) { calls++; });
  const size_t n = ops::set_intersect(pa, pb);
  const size_t n_empty = ops::set_intersect(pa, pe);
  Set<hybrid> C3;
  ops::set_intersect(&C3, pe, pb);
  printf("{\"c1\": %s, \"c2\": %s, \"triples\": %s, \"count_f\": %zu, \"calls\": %zu, \"count\": %zu, "
         "\"count_empty\": %zu, \"c3_cardinality\": %u, \"c1_type\": %d, \"b_type\": %d, \"c1_range\": %u}\n",
         list(C1.elems, C1.cardinality).c_str(), list(C2.elems, C2.cardinality).c_str(), triples.c_str(), n_f, calls, n,
         n_empty, C3.cardinality, (int)C1.type, (int)B.type, C1.range);
  return 0;
}
