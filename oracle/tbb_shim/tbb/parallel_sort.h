/* Stand-in for TBB's parallel_sort, used only to compile the reference
 * storage engine for the CPU oracle.  TBB is not installed in this image.
 * The reference calls tbb::parallel_sort(first, last, comp) once per trie
 * build (storage_engine/src/Trie.cpp:403-404) and once in the encoder.
 * This stand-in sorts with std::sort on the calling thread, so trie-build
 * time of the reference is serial; query time is unaffected.  The result is
 * identical to a parallel sort because the comparator used there
 * (SortColumns, Trie.cpp:173-186) is a strict weak order whose ties are
 * rows with identical column values. */
#ifndef EH_SHIM_TBB_PARALLEL_SORT_H
#define EH_SHIM_TBB_PARALLEL_SORT_H
#include <algorithm>
namespace tbb {
template <typename It, typename Cmp>
inline void parallel_sort(It first, It last, const Cmp& cmp) { std::sort(first, last, cmp); }
template <typename It>
inline void parallel_sort(It first, It last) { std::sort(first, last); }
}  // namespace tbb
#endif
