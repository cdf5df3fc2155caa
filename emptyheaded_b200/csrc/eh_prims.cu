// Device-wide primitives written for this engine: exclusive scan, LSD radix
// sort of 64-bit keys, unique, max.  They replace the reference's TBB sort
// (storage_engine/src/Trie.cpp:403-404) and its sequential run detection
// (Trie.cpp:192-224, 291-302) inside the trie build.
#include "eh_common.cuh"

namespace eh {

// ================================================================== scan
// Three-phase scan: per-tile reduce, scan of tile sums (recursive), per-tile
// scan with the tile's offset.  Tile = 256 threads x 8 items.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* warp_tot, T* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T inc = warp_incl_scan(v);
  if (lane == 31) warp_tot[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    T w = lane < (kScanThreads / 32) ? warp_tot[lane] : T(0);
    T wi = warp_incl_scan(w);
    if (lane < (kScanThreads / 32)) warp_tot[lane] = wi - w;
    if (lane == (kScanThreads / 32) - 1) *total = wi;
  }
  __syncthreads();
  return inc - v + warp_tot[wid];
}

template <typename T>
__global__ void scan_reduce_kernel(const T* __restrict__ in, uint64_t n, T* __restrict__ tile_sums) {
  __shared__ T warp_tot[kScanThreads / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  T s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    uint64_t i = base + (uint64_t)k * kScanThreads + threadIdx.x;
    if (i < n) s += in[i];
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) warp_tot[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    T w = threadIdx.x < (kScanThreads / 32) ? warp_tot[threadIdx.x] : T(0);
    w = warp_sum(w);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = w;
  }
}

template <typename T>
__global__ void scan_tile_kernel(const T* __restrict__ in, T* __restrict__ out, uint64_t n,
                                 const T* __restrict__ tile_offsets, T* __restrict__ total_dev) {
  __shared__ T warp_tot[kScanThreads / 32];
  __shared__ T tot;
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    uint64_t i = base + k;
    v[k] = i < n ? in[i] : T(0);
    s += v[k];
  }
  T ex = block_excl_scan(s, warp_tot, &tot);
  const T off = tile_offsets ? tile_offsets[blockIdx.x] : T(0);
  T run = off + ex;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    uint64_t i = base + k;
    if (i < n) out[i] = run;
    run += v[k];
  }
  if (total_dev && blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) *total_dev = run;
}

template <typename T>
void exclusive_scan(const T* in, T* out, uint64_t n, T* total_dev, cudaStream_t s) {
  if (n == 0) {
    if (total_dev) EH_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(T), s));
    return;
  }
  const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    scan_tile_kernel<T><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, total_dev);
    EH_CHECK_LAUNCH();
    return;
  }
  DevBuf<T> sums(tiles, s);
  scan_reduce_kernel<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, sums.p);
  EH_CHECK_LAUNCH();
  exclusive_scan<T>(sums.p, sums.p, tiles, nullptr, s);
  scan_tile_kernel<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, sums.p, total_dev);
  EH_CHECK_LAUNCH();
}
template void exclusive_scan<uint32_t>(const uint32_t*, uint32_t*, uint64_t, uint32_t*, cudaStream_t);
template void exclusive_scan<uint64_t>(const uint64_t*, uint64_t*, uint64_t, uint64_t*, cudaStream_t);

// Kernels exclusive_scan launches for n inputs.
uint32_t scan_launches(uint64_t n) {
  if (n == 0) return 0;
  const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  return tiles == 1 ? 1u : 2u + scan_launches(tiles);
}

// Tile-sum elements exclusive_scan_scratch needs for n inputs (all levels).
uint64_t scan_scratch_elems(uint64_t n) {
  uint64_t need = 0;
  while (n > (uint64_t)kScanTile) {
    n = (n + kScanTile - 1) / kScanTile;
    need += n;
  }
  return need;
}

// exclusive_scan with its tile sums in caller memory (scratch_elems >=
// scan_scratch_elems(n)): allocates nothing.
template <typename T>
void exclusive_scan_scratch(const T* in, T* out, uint64_t n, T* total_dev, T* scratch, uint64_t scratch_elems,
                            cudaStream_t s) {
  if (n == 0) {
    if (total_dev) EH_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(T), s));
    return;
  }
  const uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    scan_tile_kernel<T><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, total_dev);
    EH_CHECK_LAUNCH();
    return;
  }
  EH_REQUIRE(scratch_elems >= tiles, EH_ERR_INVALID, "scan scratch too small");
  T* sums = scratch;
  scan_reduce_kernel<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, sums);
  EH_CHECK_LAUNCH();
  exclusive_scan_scratch<T>(sums, sums, tiles, nullptr, scratch + tiles, scratch_elems - tiles, s);
  scan_tile_kernel<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, sums, total_dev);
  EH_CHECK_LAUNCH();
}
template void exclusive_scan_scratch<uint32_t>(const uint32_t*, uint32_t*, uint64_t, uint32_t*, uint32_t*, uint64_t,
                                               cudaStream_t);

// ============================================================ radix sort
// LSD, 8-bit digits.  One pass = histogram per tile (digit-major counters),
// exclusive scan of the counters, stable scatter.  A tile is 8 warps x 16
// rounds x 32 keys; each warp ranks its keys stably with __match_any_sync
// against a warp-private digit histogram in shared memory.
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;  // 4096 keys
constexpr int kRadix = 256;

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const K* __restrict__ keys, uint64_t n,
                                                                  int shift, uint32_t* __restrict__ counts,
                                                                  uint32_t tiles) {
  __shared__ uint32_t h[kRadix];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll 4
  for (int r = 0; r < kSortRounds; r++) {
    uint64_t i = base + (uint64_t)r * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xff], 1u);
  }
  __syncthreads();
  counts[(uint64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// kVals: a uint32 payload travels with each key.  The tile's keys are first
// placed in digit order in shared memory (stable: tile digit start + the
// warp's offset within the digit + the key's rank in its warp), then written
// out in that order, so consecutive threads write consecutive slots of one
// digit's run (coalesced) instead of 256 scattered runs per round.  With
// write_keys = 0 only the payloads are written (the last pass of a sort whose
// caller reads the payloads alone).
template <typename K, bool kVals>
__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(const K* __restrict__ keys,
                                                                     K* __restrict__ out, uint64_t n,
                                                                     int shift,
                                                                     const uint32_t* __restrict__ offsets,
                                                                     uint32_t tiles,
                                                                     const uint32_t* __restrict__ vin,
                                                                     uint32_t* __restrict__ vout, int write_keys) {
  __shared__ uint32_t whist[kSortWarps][kRadix];
  __shared__ uint32_t tile_off[kRadix];
  __shared__ uint32_t tstart[kRadix];
  __shared__ uint32_t wtot[kSortWarps];
  extern __shared__ __align__(16) unsigned char sort_smem[];  // kSortTile keys, then (kVals) kSortTile payloads
  K* skeys = reinterpret_cast<K*>(sort_smem);
  uint32_t* svals = reinterpret_cast<uint32_t*>(skeys + kSortTile);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&whist[0][0])[i] = 0;
  tile_off[threadIdx.x] = offsets[(uint64_t)threadIdx.x * tiles + blockIdx.x];
  __syncthreads();
  // warp w owns keys [base + w*512, base + (w+1)*512), round-major
  const uint64_t tbase = (uint64_t)blockIdx.x * kSortTile;
  const uint64_t wbase = tbase + (uint64_t)wid * (32 * kSortRounds);
  K k[kSortRounds];
  uint32_t pos[kSortRounds];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < kSortRounds; r++) {
    const uint64_t i = wbase + (uint64_t)r * 32 + lane;
    const bool valid = i < n;
    k[r] = valid ? keys[i] : 0;
    const uint32_t d = valid ? (uint32_t)((k[r] >> shift) & 0xff) : 0x100u;
    const uint32_t peers = __match_any_sync(kFull, d);
    const uint32_t rank = __popc(peers & lt);
    const int leader = __ffs(peers) - 1;
    uint32_t basecnt = 0;
    if (valid) basecnt = whist[wid][d];
    __syncwarp();
    if (valid && lane == leader) whist[wid][d] = basecnt + __popc(peers);
    __syncwarp();
    pos[r] = basecnt + rank;  // offset among this warp's keys of digit d
  }
  __syncthreads();
  // per-digit exclusive prefix over warps (thread t owns digit t), and the
  // tile's digit starts (exclusive scan over digits)
  uint32_t run = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; w++) {
    const uint32_t c = whist[w][threadIdx.x];
    whist[w][threadIdx.x] = run;
    run += c;
  }
  const uint32_t inc = warp_incl_scan(run);
  if (lane == 31) wtot[wid] = inc;
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < wid; w++) before += wtot[w];
  tstart[threadIdx.x] = before + inc - run;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortRounds; r++) {
    const uint64_t i = wbase + (uint64_t)r * 32 + lane;
    if (i < n) {
      const uint32_t d = (uint32_t)((k[r] >> shift) & 0xff);
      const uint32_t li = tstart[d] + whist[wid][d] + pos[r];
      skeys[li] = k[r];
      if (kVals) svals[li] = vin[i];
    }
  }
  __syncthreads();
  const uint32_t cnt = (uint32_t)min((uint64_t)kSortTile, n - tbase);
  for (uint32_t j = threadIdx.x; j < cnt; j += kSortThreads) {
    const K key = skeys[j];
    const uint32_t d = (uint32_t)((key >> shift) & 0xff);
    const uint32_t dst = tile_off[d] + (j - tstart[d]);
    if (write_keys) out[dst] = key;
    if (kVals) vout[dst] = svals[j];
  }
}

template <typename K>
static size_t scatter_smem(bool vals) {
  return (size_t)kSortTile * (sizeof(K) + (vals ? 4 : 0));
}

template <typename K>
static void set_scatter_smem() {
  static bool done = false;  // the staged scatter takes more than the default 48 KB
  if (done) return;
  EH_CUDA(cudaFuncSetAttribute(radix_scatter_kernel<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)scatter_smem<K>(true)));
  EH_CUDA(cudaFuncSetAttribute(radix_scatter_kernel<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)scatter_smem<K>(false)));
  done = true;
}

// LSD passes; with vals != nullptr a uint32 payload follows its key
// (stable).  copy_back: the sorted keys (and payloads) end in keys / vals;
// otherwise only the payloads are produced, in the buffer returned (vals or
// vtmp), and the keys are left unspecified.
template <typename K>
static uint32_t* radix_sort_impl(K* keys, K* tmp, uint32_t* vals, uint32_t* vtmp, uint64_t n, int bits,
                                 bool copy_back, cudaStream_t s) {
  if (n < 2) return vals;
  EH_REQUIRE(n < (1ull << 32), EH_ERR_UNSUPPORTED, "radix sort supports fewer than 2^32 keys");
  const uint32_t tiles = (uint32_t)((n + kSortTile - 1) / kSortTile);
  DevBuf<uint32_t> counts((uint64_t)kRadix * tiles, s);
  set_scatter_smem<K>();
  K* src = keys;
  K* dst = tmp;
  uint32_t* vsrc = vals;
  uint32_t* vdst = vtmp;
  for (int shift = 0; shift < bits; shift += 8) {
    const int write_keys = copy_back || shift + 8 < bits;
    radix_hist_kernel<K><<<tiles, kSortThreads, 0, s>>>(src, n, shift, counts.p, tiles);
    EH_CHECK_LAUNCH();
    exclusive_scan<uint32_t>(counts.p, counts.p, (uint64_t)kRadix * tiles, nullptr, s);
    if (vals)
      radix_scatter_kernel<K, true><<<tiles, kSortThreads, scatter_smem<K>(true), s>>>(
          src, dst, n, shift, counts.p, tiles, vsrc, vdst, write_keys);
    else
      radix_scatter_kernel<K, false><<<tiles, kSortThreads, scatter_smem<K>(false), s>>>(
          src, dst, n, shift, counts.p, tiles, nullptr, nullptr, write_keys);
    EH_CHECK_LAUNCH();
    std::swap(src, dst);
    std::swap(vsrc, vdst);
  }
  if (copy_back && src != keys) {
    EH_CUDA(cudaMemcpyAsync(keys, src, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
    if (vals) EH_CUDA(cudaMemcpyAsync(vals, vsrc, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    return vals;
  }
  return vsrc;
}

void radix_sort_u64(uint64_t* keys, uint64_t* tmp, uint64_t n, int bits, cudaStream_t s) {
  radix_sort_impl<uint64_t>(keys, tmp, nullptr, nullptr, n, bits, true, s);
}

void radix_sort_kv(uint64_t* keys, uint64_t* ktmp, uint32_t* vals, uint32_t* vtmp, uint64_t n, int bits,
                   cudaStream_t s) {
  radix_sort_impl<uint64_t>(keys, ktmp, vals, vtmp, n, bits, true, s);
}

uint32_t* radix_sort_payload_u32(uint32_t* keys, uint32_t* ktmp, uint32_t* vals, uint32_t* vtmp, uint64_t n, int bits,
                                 cudaStream_t s) {
  EH_REQUIRE(bits >= 1 && bits <= 32, EH_ERR_INVALID, "32-bit keys sort on 1 to 32 bits");
  return radix_sort_impl<uint32_t>(keys, ktmp, vals, vtmp, n, bits, false, s);
}

// ================================================================ unique
__global__ void head_flags_kernel(const uint64_t* __restrict__ keys, uint64_t n, uint32_t* __restrict__ flags) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}
__global__ void compact_kernel(const uint64_t* __restrict__ keys, uint64_t n, const uint32_t* __restrict__ pos,
                               uint64_t* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (i == 0 || keys[i] != keys[i - 1]) out[pos[i]] = keys[i];
}

uint64_t unique_sorted_u64(const uint64_t* keys, uint64_t* out, uint64_t n, cudaStream_t s) {
  if (n == 0) return 0;
  DevBuf<uint32_t> pos(n, s);
  DevBuf<uint32_t> total(1, s);
  const int grid = num_sms() * 8;
  head_flags_kernel<<<grid, 256, 0, s>>>(keys, n, pos.p);
  EH_CHECK_LAUNCH();
  exclusive_scan<uint32_t>(pos.p, pos.p, n, total.p, s);
  compact_kernel<<<grid, 256, 0, s>>>(keys, n, pos.p, out);
  EH_CHECK_LAUNCH();
  uint32_t h = 0;
  EH_CUDA(cudaMemcpyAsync(&h, total.p, 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  return h;
}

// =================================================================== max
__global__ void max_kernel(const uint32_t* __restrict__ a, uint64_t n, uint32_t* __restrict__ out) {
  uint32_t m = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    m = max(m, a[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

uint32_t max_u32(const uint32_t* a, uint64_t n, cudaStream_t s) {
  DevBuf<uint32_t> out(1, s);
  EH_CUDA(cudaMemsetAsync(out.p, 0, 4, s));
  if (n) {
    max_kernel<<<num_sms() * 4, 256, 0, s>>>(a, n, out.p);
    EH_CHECK_LAUNCH();
  }
  uint32_t h = 0;
  EH_CUDA(cudaMemcpyAsync(&h, out.p, 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  return h;
}

}  // namespace eh
