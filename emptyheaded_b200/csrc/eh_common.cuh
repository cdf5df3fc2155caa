// Shared definitions for the B200 storage-engine kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "eh_b200.h"

namespace eh {

constexpr int kWarp = 32;
constexpr uint32_t kFull = 0xffffffffu;

// ---------------------------------------------------------------- errors
// Every entry point returns an eh_status; the message of the last failure
// on the calling thread is kept for eh_last_error().
void set_error(const std::string& msg);

struct Error {
  int code;
  std::string msg;
};

#define EH_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      throw ::eh::Error{EH_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

#define EH_CHECK_LAUNCH() EH_CUDA(cudaGetLastError())

#define EH_REQUIRE(cond, code, msg)                           \
  do {                                                        \
    if (!(cond)) throw ::eh::Error{(code), std::string(msg)}; \
  } while (0)

inline int ceil_div(uint64_t a, uint64_t b) { return (int)((a + b - 1) / b); }

inline int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

// ---------------------------------------------------------------- tracing
// Phase timings on stderr when the environment variable EH_TRACE is set,
// like the reference's timer::start_clock / stop_clock prints
// (storage_engine/include/utils/timer.hpp:11-20).  EH_TRACE=1: a traced phase
// synchronises its stream when it begins and ends and reports the wall time
// between.  EH_TRACE=2: phases record CUDA events instead, nothing
// synchronises, and the outermost phase prints every phase's device time (and
// the host time spent inside it) when it ends.  With EH_TRACE unset it costs
// one branch.
bool trace_enabled();
struct TracePhase {
  const char* name;
  cudaStream_t s;
  double t0 = 0;
  int mode;
  int idx = -1;
  bool on;
  TracePhase(const char* n, cudaStream_t st);
  ~TracePhase() { end(); }
  void end();  // report now (once)
  TracePhase(const TracePhase&) = delete;
  TracePhase& operator=(const TracePhase&) = delete;
};

// ------------------------------------------------------- device buffers
// The engine's stream-ordered memory pool on the current device (one per
// device, created on first use).  Freed blocks stay in the pool for the next
// allocation instead of going back to the driver at every synchronisation
// (the default pool's behaviour): a trie build frees and re-allocates
// gigabytes between its synchronisations.  eh_context_destroy trims it.
cudaMemPool_t device_pool();
void trim_device_pool(int device);

// A stream-ordered free is complete, and its block merged with the free
// blocks beside it, only once the stream has run past it.  Large allocations
// made while frees were still pending were slow without the pool growing
// (the bitset ranks of an R-MAT-22 layout: 2 ms every call, up to hundreds of
// ms at random calls; end to end 28.2 ms with spikes against 24.7 ms steady
// when each free waits for its stream), so a free waits for its stream,
// except while the stream is being captured into a graph.
inline void settle_free(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) == cudaSuccess && st == cudaStreamCaptureStatusNone) cudaStreamSynchronize(s);
}

// Stream-ordered device allocations (from device_pool()) owned by RAII
// handles; a trie and its layouts live in a handful of these.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = 0;
  DevBuf() = default;
  DevBuf(size_t count, cudaStream_t stream) { alloc(count, stream); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; s = o.s;
      o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  void alloc(size_t count, cudaStream_t stream) {
    release();
    s = stream;
    n = count;
    if (count) {
      cudaError_t e = cudaMallocFromPoolAsync((void**)&p, count * sizeof(T), device_pool(), stream);
      if (e != cudaSuccess) {
        p = nullptr;
        n = 0;
        cudaGetLastError();
        throw Error{EH_ERR_OOM, "device allocation of " + std::to_string(count * sizeof(T)) + " bytes failed"};
      }
    }
  }
  void release() {
    if (p) {
      cudaFreeAsync(p, s);
      settle_free(s);
    }
    p = nullptr;
    n = 0;
  }
  ~DevBuf() { release(); }
  size_t bytes() const { return n * sizeof(T); }
};

// --------------------------------------------------------- device helpers
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// inclusive warp scan
template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
  const uint32_t l = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(kFull, v, o);
    if (l >= (uint32_t)o) v += t;
  }
  return v;
}

// ------------------------------------------------------------------- rng
// splitmix64 as a counter-based generator: draw i of a stream is a pure
// function of (seed, i); the host oracle uses the same function.
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// draw `index` of the stream whose seed was mixed once: splitmix64(seed)
__host__ __device__ __forceinline__ uint64_t rand64(uint64_t seed_mixed, uint64_t index) {
  return splitmix64(seed_mixed ^ splitmix64(index));
}

inline int bits_for(uint64_t maxv) {
  int b = 1;
  while (b < 64 && (maxv >> b)) b++;
  return b;
}

// ------------------------------------------------------------ primitives
// Device-wide exclusive scan of n elements (in may equal out).  Returns
// the total through *total_dev when non-null (device pointer, one T).
template <typename T>
void exclusive_scan(const T* in, T* out, uint64_t n, T* total_dev, cudaStream_t s);
// The same with its tile sums in caller memory; allocates nothing.
uint64_t scan_scratch_elems(uint64_t n);
uint32_t scan_launches(uint64_t n);
template <typename T>
void exclusive_scan_scratch(const T* in, T* out, uint64_t n, T* total_dev, T* scratch, uint64_t scratch_elems,
                            cudaStream_t s);

// LSD radix sort of n 64-bit keys on their low `bits` bits, in place
// (tmp must hold n keys).
void radix_sort_u64(uint64_t* keys, uint64_t* tmp, uint64_t n, int bits, cudaStream_t s);
// The same with a uint32 payload per key, stable (vtmp holds n values).
void radix_sort_kv(uint64_t* keys, uint64_t* ktmp, uint32_t* vals, uint32_t* vtmp, uint64_t n, int bits,
                   cudaStream_t s);
// Stable order of uint32 payloads by 32-bit keys (low `bits` bits): returns
// the buffer, vals or vtmp, that holds the payloads in key order; the keys
// are not kept (no key writes on the last pass, no copy back).
uint32_t* radix_sort_payload_u32(uint32_t* keys, uint32_t* ktmp, uint32_t* vals, uint32_t* vtmp, uint64_t n, int bits,
                                 cudaStream_t s);

// Keep the first of each run of equal keys (keys sorted).  Writes the
// compacted keys to out and the count to *count_host (synchronises).
uint64_t unique_sorted_u64(const uint64_t* keys, uint64_t* out, uint64_t n, cudaStream_t s);

// max of n u32 values (synchronises)
uint32_t max_u32(const uint32_t* a, uint64_t n, cudaStream_t s);

}  // namespace eh
