/* Forced-include for the reference build.  The reference sizes its thread
 * pool with a per-translation-unit `static size_t NUM_THREADS =
 * NUM_THREADS_IN;` (storage_engine/include/utils/common.hpp:32-34).  The
 * oracle recipe defines NUM_THREADS_IN as a call to eh_ref_num_threads(), so
 * every translation unit initialises its copy from the same run-time value:
 * $EH_REF_THREADS if set, else the number of CPUs this process may use. */
#ifndef EH_REF_THREADS_H
#define EH_REF_THREADS_H
#include <cstddef>
std::size_t eh_ref_num_threads();
#endif
