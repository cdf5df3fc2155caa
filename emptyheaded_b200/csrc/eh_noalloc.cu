// Allocation-free variant of the COUNT query (eh_query_count_noalloc).
//
// Who needs it: callers that must not allocate device memory while they
// run queries.  A host that embeds this engine next to another memory owner
// (a framework with its own caching allocator, a database with a fixed
// device-memory budget) cannot have a library call cudaMalloc behind its
// back: the allocation can fail when that owner holds or has fragmented
// the memory, and cudaFree synchronises the whole device in the middle of
// the host's other work.  eh_query_count allocates its work plan, queue and
// result on every call; this entry point uses instead one fixed array that
// is part of the library image.
//
// The array: g_noalloc_scratch below, EH_NOALLOC_SCRATCH_BYTES (64 MiB),
// file-scope __device__.  Every GPU that loads the library holds it until
// the process exits.  Host code never uses the symbol itself as an address
// (on the host it only names the variable); the first call on each device
// asks the runtime for the device address with cudaGetSymbolAddress, with
// that device current, and passes that pointer to the kernels.  Do that
// first call before any stream capture on the device.  Every call reuses
// the array and finds the previous call's contents in it; the query clears
// the parts that must start at zero.  Two calls whose GPU work overlapped
// would race on the array: calls through this entry point in one process
// take a per-device lock and return only after their result is back, so
// they never overlap each other.
#include <mutex>

#include "eh_internal.cuh"

#define EH_NOALLOC_SCRATCH_BYTES (64ull << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[EH_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_dev[kMaxDevices] = {};
std::mutex g_device_mu[kMaxDevices];

// device address of g_noalloc_scratch on the current device (set up once)
unsigned char* scratch_for(int dev) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      throw eh::Error{EH_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                                       cudaGetErrorString(e)};
    }
    g_scratch_dev[dev] = p;
  }
  return static_cast<unsigned char*>(g_scratch_dev[dev]);
}
}  // namespace

extern "C" eh_status eh_query_count_noalloc(eh_context* ctx, const eh_trie* trie, int query,
                                            const eh_exec_config* cfg, uint64_t* result) {
  try {
    if (!ctx || !trie || !result) throw eh::Error{EH_ERR_INVALID, "null argument"};
    if (ctx->device < 0 || ctx->device >= kMaxDevices) throw eh::Error{EH_ERR_UNSUPPORTED, "device index too large"};
    EH_CUDA(cudaSetDevice(ctx->device));
    std::lock_guard<std::mutex> lk(g_device_mu[ctx->device]);
    try {
      unsigned char* scratch = scratch_for(ctx->device);
      eh::query_count_in_scratch(ctx, trie, query, cfg, scratch, EH_NOALLOC_SCRATCH_BYTES, result);
    } catch (...) {
      // a failed call releases the lock only once its own GPU work is done
      cudaStreamSynchronize(ctx->stream);
      throw;
    }
    return EH_OK;
  } catch (const eh::Error& e) {
    eh::set_error(e.msg);
    return e.code;
  } catch (const std::exception& e) {
    eh::set_error(e.what());
    return EH_ERR_INVALID;
  }
}
