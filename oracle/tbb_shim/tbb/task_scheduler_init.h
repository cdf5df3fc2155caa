/* Stand-in for TBB's task_scheduler_init (constructed at
 * storage_engine/src/Trie.cpp:403).  It only sized TBB's worker pool, which
 * the sort stand-in in parallel_sort.h does not use. */
#ifndef EH_SHIM_TBB_TASK_SCHEDULER_INIT_H
#define EH_SHIM_TBB_TASK_SCHEDULER_INIT_H
#include <cstddef>
namespace tbb {
struct task_scheduler_init {
  explicit task_scheduler_init(std::size_t = 0) {}
};
}  // namespace tbb
#endif
