/* Reference-engine dictionary writer for the encoding-format test.
 *
 * TEST INFRASTRUCTURE ONLY: compiled against the reference's own
 * Encoding<T> (storage_engine/include/Encoding.hpp, src/Encoding.cpp) by
 * `make -C oracle ref_encoding`; the product never links it.
 *
 *   eh_ref_encoding <dir>
 *
 * builds the dictionaries of three value sets with Encoding<T>::build over a
 * std::set and writes each with to_binary under <dir>/u32/, <dir>/long/ and
 * <dir>/str/ (the values match tests/cpp/dropin_encoding.cpp).
 */
#include <sys/stat.h>

#include <set>
#include <string>

#include "Encoding.hpp"

// the thread count the recipe's NUM_THREADS_IN calls (tbb_shim/eh_ref_threads.h);
// writing a dictionary runs on one thread
std::size_t eh_ref_num_threads() { return 1; }

template <class T>
static void write(const std::string& dir, std::set<T> values) {
  mkdir(dir.c_str(), 0755);
  Encoding<T> e;
  e.build(&values);
  e.to_binary(dir + "/");
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string dir = argv[1];
  write<uint32_t>(dir + "/u32", {900u, 5u, 3u, 7u});
  write<long>(dir + "/long", {-2L, 1L << 40, 0L});
  write<std::string>(dir + "/str", {"b", "", "alpha"});
  return 0;
}
