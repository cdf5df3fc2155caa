/* Encoding<T> of the drop-in layer (include/eh/Encoding.hpp).
 *
 * TEST PROGRAM.  dropin_encoding <dir>: builds dictionaries of uint32_t,
 * long and std::string values, writes them with to_binary under <dir>/<type>/,
 * reads them back with from_binary and encodes a column through each; prints
 * one JSON line with the keys, the read-back dictionaries and the encoded
 * columns for the test to compare against the reference's file format
 * (storage_engine/src/Encoding.cpp:52-130).
 */
#include <sys/stat.h>

#include <cstdio>
#include <set>
#include <string>
#include <vector>

#include "Encoding.hpp"

template <class T>
static std::string show(const T& v) {
  return std::to_string(v);
}
template <>
std::string show<std::string>(const std::string& v) {
  return "\"" + v + "\"";
}

template <class T>
static std::string list(const std::vector<T>& xs) {
  std::string s = "[";
  for (size_t i = 0; i < xs.size(); i++) s += (i ? ", " : "") + show(xs[i]);
  return s + "]";
}

template <class T>
static std::string round_trip(const std::string& dir, std::set<T> values, std::vector<T> column) {
  mkdir(dir.c_str(), 0755);
  Encoding<T> e;
  e.build(&values);
  e.to_binary(dir + "/");
  Encoding<T>* back = Encoding<T>::from_binary(dir + "/");
  std::vector<uint32_t>* keys = back->encode_column(column.data(), column.size());
  std::vector<uint32_t> lookups;
  for (const T& v : column) lookups.push_back(back->value_to_key.at(v));
  std::string out = "{\"num_distinct\": " + std::to_string(back->num_distinct) +
                    ", \"key_to_value\": " + list(back->key_to_value) + ", \"encoded\": " + list(*keys) +
                    ", \"lookups\": " + list(lookups) + "}";
  delete keys;
  delete back;
  return out;
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string dir = argv[1];
  const std::string u = round_trip<uint32_t>(dir + "/u32", {900u, 5u, 3u, 7u}, {7u, 3u, 900u, 3u});
  const std::string l = round_trip<long>(dir + "/long", {-2L, 1L << 40, 0L}, {0L, 1L << 40, -2L});
  const std::string s =
      round_trip<std::string>(dir + "/str", {"b", "", "alpha"}, {std::string("alpha"), std::string(""), std::string("b")});
  // build() from a vector keeps the order given; a repeated value keeps its
  // first key and still takes a key number
  Encoding<uint32_t> v;
  std::vector<uint32_t> given = {40, 10, 40, 20};
  v.build(&given);
  bool unknown_throws = false;
  try {
    uint32_t missing = 99;
    delete v.encode_column(&missing, 1);
  } catch (const std::out_of_range&) {
    unknown_throws = true;
  }
  printf("{\"u32\": %s, \"long\": %s, \"str\": %s, \"vector_num_distinct\": %u, \"vector_key_of_40\": %u, "
         "\"vector_key_to_value\": %s, \"unknown_throws\": %s}\n",
         u.c_str(), l.c_str(), s.c_str(), v.num_distinct, v.value_to_key.at(40), list(v.key_to_value).c_str(),
         unknown_throws ? "true" : "false");
  return 0;
}
