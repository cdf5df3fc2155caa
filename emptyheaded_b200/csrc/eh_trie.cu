// Two-level trie construction on the device.
//
// Reference: Trie<A,M>::Trie (storage_engine/src/Trie.cpp:380-510) sorts row
// indices with a column-chasing comparator, finds distinct head values and
// per-head runs, and builds each set with hybrid::build.  Here:
//   rows -> packed 64-bit keys (col0 << b | col1) -> LSD radix sort ->
//   unique -> head flags + scan -> head[], off[], vals[] (CSR) ->
//   head_index[] (value -> head position, the dense form of the reference's
//   NextLevel array, trie/TrieBlock.hpp:26-48) -> per-set layout ->
//   range-bitset words + per-word ranks, block-bitset blocks.
// The CSR copy of every set is kept whatever its layout: it is the
// coalesced form the kernels stream; a bitset layout adds a probe structure.
#include <algorithm>
#include <cstring>

#include "eh_internal.cuh"

namespace eh {

__global__ void pack_rows_kernel(const uint32_t* __restrict__ c0, const uint32_t* __restrict__ c1, uint64_t n, int b,
                                 uint64_t* __restrict__ keys) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    keys[i] = ((uint64_t)c0[i] << b) | c1[i];
}

__global__ void head_flag_kernel(const uint64_t* __restrict__ keys, uint64_t n, int b, uint32_t* __restrict__ flag) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    flag[i] = (i == 0 || (keys[i] >> b) != (keys[i - 1] >> b)) ? 1u : 0u;
}

__global__ void csr_kernel(const uint64_t* __restrict__ keys, uint64_t n, int b, const uint32_t* __restrict__ hpos,
                           uint32_t* __restrict__ head, uint64_t* __restrict__ off, uint32_t* __restrict__ vals) {
  const uint64_t mask = (1ull << b) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    vals[i] = (uint32_t)(k & mask);
    if (i == 0 || (k >> b) != (keys[i - 1] >> b)) {
      head[hpos[i]] = (uint32_t)(k >> b);
      off[hpos[i]] = i;
    }
  }
}

__global__ void head_index_kernel(const uint32_t* __restrict__ head, uint32_t nh, int32_t* __restrict__ hidx) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x) hidx[head[i]] = (int32_t)i;
}

// set i's elements: child set for i < n_head, the head itself for i == n_head
struct SetSrc {
  const uint32_t* head;
  const uint64_t* off;
  const uint32_t* vals;
  uint32_t n_head;
  __device__ __forceinline__ void get(uint32_t i, const uint32_t*& p, uint64_t& len) const {
    if (i == n_head) { p = head; len = n_head; }
    else { p = vals + off[i]; len = off[i + 1] - off[i]; }
  }
};

// common::is_sparse (utils/common.hpp:60-66) on hybrid::get_type's
// range = last - first (layouts/hybrid.hpp:103-111).
__device__ __forceinline__ bool is_sparse(uint64_t len, uint64_t range) {
  if (len > 2) return ((double)range / (double)len) > 128.0;
  return true;
}

// max_words: per-set cap on range-bitset words under FORCED (0 = none)
__global__ void layout_heuristic_kernel(SetSrc src, uint32_t n_sets, int policy, int forced, uint64_t max_words,
                                        uint8_t* __restrict__ layout) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_sets; i += gridDim.x * blockDim.x) {
    const uint32_t* p;
    uint64_t len;
    src.get(i, p, len);
    const uint64_t range = len > 1 ? (uint64_t)(p[len - 1] - p[0]) : 0;
    uint8_t l = is_sparse(len, range) ? EH_LAYOUT_UINTEGER : EH_LAYOUT_RANGE_BITSET;
    if (policy == EH_POLICY_FORCED && i < src.n_head) {
      const uint64_t words = len ? (uint64_t)(p[len - 1] >> 6) - (p[0] >> 6) + 1 : 0;
      if (forced != EH_LAYOUT_RANGE_BITSET || max_words == 0 || (words <= max_words && words <= 16 * len + 64))
        l = (uint8_t)forced;
    }
    layout[i] = l;
  }
}

// Sets with more than kBigSet elements (the head set, hubs of a symmetric
// relation) are built by grid-wide passes, one set at a time; the
// warp-per-set kernels below skip them.
constexpr uint64_t kBigSet = 8192;

// sizes of each set's bitset structure: words (range bitset) or blocks
__global__ void aux_size_kernel(SetSrc src, uint32_t n_sets, const uint8_t* __restrict__ layout,
                                SetAux* __restrict__ aux, uint64_t* __restrict__ words, uint64_t* __restrict__ blocks) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = warp; i < n_sets; i += nwarps) {
    const uint32_t* p;
    uint64_t len;
    src.get(i, p, len);
    const uint8_t l = layout[i];
    uint64_t w = 0, nb = 0;
    uint32_t start = 0;
    if (len && l == EH_LAYOUT_RANGE_BITSET) {
      start = p[0] >> 6;
      w = (uint64_t)(p[len - 1] >> 6) - start + 1;
    } else if (len && l == EH_LAYOUT_BLOCK_BITSET && len <= kBigSet) {
      uint64_t c = 0;
      for (uint64_t j = lane; j < len; j += 32) c += (j == 0 || (p[j] >> 8) != (p[j - 1] >> 8)) ? 1 : 0;
      nb = warp_sum(c);
    }
    if (lane == 0) {
      words[i] = w;
      blocks[i] = nb;
      aux[i].start = start;
      aux[i].n = (uint32_t)(w ? w : nb);
    }
  }
}

__global__ void aux_offsets_kernel(uint32_t n_sets, const uint8_t* __restrict__ layout,
                                   const uint64_t* __restrict__ woff, const uint64_t* __restrict__ boff,
                                   SetAux* __restrict__ aux) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_sets; i += gridDim.x * blockDim.x)
    aux[i].off = layout[i] == EH_LAYOUT_BLOCK_BITSET ? boff[i] : woff[i];
}

// fill the words of every range-bitset set and their prefix ranks; one warp per set
__global__ void bitset_fill_kernel(SetSrc src, uint32_t n_sets, const uint8_t* __restrict__ layout,
                                   const SetAux* __restrict__ aux, uint64_t* __restrict__ words,
                                   uint32_t* __restrict__ rank) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = warp; i < n_sets; i += nwarps) {
    if (layout[i] != EH_LAYOUT_RANGE_BITSET) continue;
    const uint32_t* p;
    uint64_t len;
    src.get(i, p, len);
    if (!len || len > kBigSet) continue;
    const SetAux a = aux[i];
    uint64_t* w = words + a.off;
    uint32_t* r = rank + a.off;
    for (uint32_t j = lane; j < a.n; j += 32) w[j] = 0;
    __syncwarp();
    for (uint64_t j = lane; j < len; j += 32)
      atomicOr((unsigned long long*)&w[(p[j] >> 6) - a.start], 1ull << (p[j] & 63));
    __syncwarp();
    uint32_t run = 0;
    for (uint32_t base = 0; base < a.n; base += 32) {
      const uint32_t j = base + lane;
      // the words were built by atomics at L2: read them from L2
      const uint32_t c = j < a.n ? (uint32_t)__popcll(__ldcg(&w[j])) : 0u;
      const uint32_t inc = warp_incl_scan(c);
      if (j < a.n) r[j] = run + inc - c;
      run += __shfl_sync(kFull, inc, 31);
    }
  }
}

// block bitsets (layouts/block_bitset.hpp:112-131): per non-empty 256-value
// block its id, the index of its first element, and 4 words
__global__ void block_fill_kernel(SetSrc src, uint32_t n_sets, const uint8_t* __restrict__ layout,
                                  const SetAux* __restrict__ aux, uint32_t* __restrict__ bid,
                                  uint32_t* __restrict__ brank, uint64_t* __restrict__ bwords) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = warp; i < n_sets; i += nwarps) {
    if (layout[i] != EH_LAYOUT_BLOCK_BITSET) continue;
    const uint32_t* p;
    uint64_t len;
    src.get(i, p, len);
    if (!len || len > kBigSet) continue;
    const SetAux a = aux[i];
    for (uint32_t j = lane; j < 4 * a.n; j += 32) bwords[4 * a.off + j] = 0;
    __syncwarp();
    uint32_t blk = 0;  // running block count before this 32-element chunk
    for (uint64_t base = 0; base < len; base += 32) {
      const uint64_t j = base + lane;
      const bool valid = j < len;
      const uint32_t x = valid ? p[j] : 0;
      const bool first = valid && (j == 0 || (x >> 8) != (p[j - 1] >> 8));
      const uint32_t ball = __ballot_sync(kFull, first);
      const uint32_t b = blk + __popc(ball & lanemask_lt());  // this block's index when `first`
      // block index of element j: blocks started at or before j, minus one
      const uint32_t my_block = blk + __popc(ball & (lanemask_lt() | (1u << lane))) - 1;
      if (first) {
        bid[a.off + b] = x >> 8;
        brank[a.off + b] = (uint32_t)j;
      }
      if (valid) atomicOr((unsigned long long*)&bwords[4 * (a.off + my_block) + ((x >> 6) & 3)], 1ull << (x & 63));
      blk += __popc(ball);
    }
  }
}

// ---- grid-wide passes over one big set
__global__ void big_sets_kernel(SetSrc src, uint32_t n_sets, const uint8_t* __restrict__ layout,
                                uint32_t* __restrict__ idx, unsigned int* __restrict__ count) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_sets; i += gridDim.x * blockDim.x) {
    const uint8_t l = layout[i];
    if (l != EH_LAYOUT_RANGE_BITSET && l != EH_LAYOUT_BLOCK_BITSET) continue;
    const uint64_t len = i == src.n_head ? src.n_head : src.off[i + 1] - src.off[i];
    if (len > kBigSet) idx[atomicAdd(count, 1u)] = i;
  }
}

// first element of each 256-value block of set i (flag per element)
__global__ void big_block_flags_kernel(SetSrc src, uint32_t i, uint32_t* __restrict__ flag,
                                       unsigned long long* __restrict__ nblocks) {
  const uint32_t* p;
  uint64_t len;
  src.get(i, p, len);
  unsigned long long c = 0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < len; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t f = (j == 0 || (p[j] >> 8) != (p[j - 1] >> 8)) ? 1u : 0u;
    flag[j] = f;
    c += f;
  }
  c = warp_sum(c);
  if (lane_id() == 0 && c) atomicAdd(nblocks, c);
}

__global__ void big_block_count_kernel(const unsigned long long* __restrict__ nblocks, uint32_t i,
                                       uint64_t* __restrict__ blocks, SetAux* __restrict__ aux) {
  blocks[i] = *nblocks;
  aux[i].n = (uint32_t)*nblocks;
}

__global__ void big_bitset_fill_kernel(SetSrc src, uint32_t i, const SetAux* __restrict__ aux,
                                       uint64_t* __restrict__ words) {
  const uint32_t* p;
  uint64_t len;
  src.get(i, p, len);
  const SetAux a = aux[i];
  uint64_t* w = words + a.off;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < len; j += (uint64_t)gridDim.x * blockDim.x)
    atomicOr((unsigned long long*)&w[(p[j] >> 6) - a.start], 1ull << (p[j] & 63));
}

__global__ void big_popc_kernel(const SetAux* __restrict__ aux, uint32_t i, const uint64_t* __restrict__ words,
                                uint32_t* __restrict__ popc) {
  const SetAux a = aux[i];
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < a.n; j += gridDim.x * blockDim.x)
    popc[j] = (uint32_t)__popcll(__ldcg(words + a.off + j));
}

// pos = exclusive scan of the block-start flags: element j lies in block
// pos[j] + flag[j] - 1
__global__ void big_block_fill_kernel(SetSrc src, uint32_t i, const SetAux* __restrict__ aux,
                                      const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                                      uint32_t* __restrict__ bid, uint32_t* __restrict__ brank,
                                      uint64_t* __restrict__ bwords) {
  const uint32_t* p;
  uint64_t len;
  src.get(i, p, len);
  const SetAux a = aux[i];
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < len; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t x = p[j];
    const uint32_t blk = pos[j] + flag[j] - 1;
    if (flag[j]) {
      bid[a.off + blk] = x >> 8;
      brank[a.off + blk] = (uint32_t)j;
    }
    atomicOr((unsigned long long*)&bwords[4 * ((uint64_t)a.off + blk) + ((x >> 6) & 3)], 1ull << (x & 63));
  }
}

// per head entry a: sum over children v in head of d+(v) (pairs the
// triangle loop nest probes below a)
__global__ void wedge_kernel(TrieView t, uint64_t* __restrict__ wedges) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = warp; i < t.n_head; i += nwarps) {
    uint64_t s = 0;
    for (uint64_t j = t.off[i] + lane; j < t.off[i + 1]; j += 32) {
      const int32_t h = t.head_index[t.vals[j]];
      if (h >= 0) s += t.off[h + 1] - t.off[h];
    }
    s = warp_sum(s);
    if (lane == 0) wedges[i] = s;
  }
}

// red[0] = largest set, red[1] = sum of squared set sizes
__global__ void set_size_stats_kernel(const uint64_t* __restrict__ off, uint32_t nh, unsigned long long* red) {
  unsigned long long mx = 0, sq = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x) {
    const unsigned long long d = off[i + 1] - off[i];
    mx = d > mx ? d : mx;
    sq += d * d;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long m2 = __shfl_xor_sync(kFull, mx, o);
    mx = m2 > mx ? m2 : mx;
  }
  sq = warp_sum(sq);
  if (lane_id() == 0) {
    atomicMax(&red[0], mx);
    atomicAdd(&red[1], sq);
  }
}

// sets per layout code: per-thread counts, warp sums, one atomic per warp
// and code (a global atomic per set on four addresses serialised at L2)
__global__ void layout_hist_kernel(const uint8_t* __restrict__ layout, uint32_t n, uint32_t* __restrict__ hist) {
  uint32_t c[4] = {0, 0, 0, 0};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t l = layout[i] & 3;
    c[0] += l == 0;
    c[1] += l == 1;
    c[2] += l == 2;
    c[3] += l == 3;
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t v = warp_sum(c[k]);
    if (lane_id() == 0 && v) atomicAdd(&hist[k], v);
  }
}

__global__ void sum_f32_kernel(const float* __restrict__ a, uint32_t n, double* __restrict__ sum) {
  double v = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v += a[i];
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  if (lane_id() == 0 && v != 0) atomicAdd(sum, v);
}

static SetSrc set_src(const eh_trie* t) { return SetSrc{t->head.p, t->off.p, t->vals.p, t->n_head}; }

// Build the probe structures for the layouts in t->layout.
static void build_layout_structs(eh_context* ctx, eh_trie* t) {
  cudaStream_t s = ctx->stream;
  const uint32_t n_sets = t->n_head + 1;
  const int grid = num_sms() * 8;
  SetSrc src = set_src(t);
  TracePhase ph_size("structs.sizes", s);
  t->aux.alloc(n_sets, s);
  DevBuf<uint64_t> words(n_sets + 1, s), blocks(n_sets + 1, s), tot(2, s);
  aux_size_kernel<<<grid, 256, 0, s>>>(src, n_sets, t->layout.p, t->aux.p, words.p, blocks.p);
  EH_CHECK_LAUNCH();
  // the big sets, and the block counts of big block-bitset sets
  std::vector<uint32_t> big;
  {
    DevBuf<uint32_t> idx(n_sets, s);
    DevBuf<unsigned int> cnt(1, s);
    EH_CUDA(cudaMemsetAsync(cnt.p, 0, 4, s));
    big_sets_kernel<<<grid, 256, 0, s>>>(src, n_sets, t->layout.p, idx.p, cnt.p);
    EH_CHECK_LAUNCH();
    unsigned int nb = 0;
    EH_CUDA(cudaMemcpyAsync(&nb, cnt.p, 4, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    big.resize(nb);
    if (nb) EH_CUDA(cudaMemcpyAsync(big.data(), idx.p, nb * 4, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
  }
  std::vector<uint8_t> big_layout(big.size());
  std::vector<uint64_t> big_len(big.size());
  for (size_t k = 0; k < big.size(); k++) {
    const uint32_t i = big[k];
    uint64_t o[2] = {0, t->n_head};
    EH_CUDA(cudaMemcpyAsync(&big_layout[k], t->layout.p + i, 1, cudaMemcpyDeviceToHost, s));
    if (i < t->n_head) EH_CUDA(cudaMemcpyAsync(o, t->off.p + i, 16, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    big_len[k] = o[1] - o[0];
  }
  uint64_t big_max = 0;
  for (uint64_t l : big_len) big_max = std::max(big_max, l);
  DevBuf<uint32_t> bflag(big_max ? big_max : 1, s), bpos(big_max ? big_max : 1, s), btot(1, s);
  DevBuf<unsigned long long> bcount(1, s);
  for (size_t k = 0; k < big.size(); k++) {
    if (big_layout[k] != EH_LAYOUT_BLOCK_BITSET) continue;
    EH_CUDA(cudaMemsetAsync(bcount.p, 0, 8, s));
    big_block_flags_kernel<<<grid, 256, 0, s>>>(src, big[k], bflag.p, bcount.p);
    EH_CHECK_LAUNCH();
    big_block_count_kernel<<<1, 1, 0, s>>>(bcount.p, big[k], blocks.p, t->aux.p);
    EH_CHECK_LAUNCH();
  }
  exclusive_scan<uint64_t>(words.p, words.p, n_sets, tot.p, s);
  exclusive_scan<uint64_t>(blocks.p, blocks.p, n_sets, tot.p + 1, s);
  aux_offsets_kernel<<<grid, 256, 0, s>>>(n_sets, t->layout.p, words.p, blocks.p, t->aux.p);
  EH_CHECK_LAUNCH();
  uint64_t h[2];
  EH_CUDA(cudaMemcpyAsync(h, tot.p, 16, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  ph_size.end();
  TracePhase ph_fill("structs.bitset_fill", s);
  t->bs_words.alloc(h[0] ? h[0] : 1, s);
  t->bs_rank.alloc(h[0] ? h[0] : 1, s);
  t->bb_id.alloc(h[1] ? h[1] : 1, s);
  t->bb_rank.alloc(h[1] ? h[1] : 1, s);
  t->bb_words.alloc(h[1] ? 4 * h[1] : 1, s);
  if (h[0]) {
    bitset_fill_kernel<<<grid, 256, 0, s>>>(src, n_sets, t->layout.p, t->aux.p, t->bs_words.p, t->bs_rank.p);
    EH_CHECK_LAUNCH();
  }
  ph_fill.end();
  TracePhase ph_bfill("structs.block_fill", s);
  if (h[1]) {
    block_fill_kernel<<<grid, 256, 0, s>>>(src, n_sets, t->layout.p, t->aux.p, t->bb_id.p, t->bb_rank.p,
                                           t->bb_words.p);
    EH_CHECK_LAUNCH();
  }
  ph_bfill.end();
  TracePhase ph_big("structs.big_sets", s);
  for (size_t k = 0; k < big.size(); k++) {
    const uint32_t i = big[k];
    SetAux a{};
    EH_CUDA(cudaMemcpyAsync(&a, t->aux.p + i, sizeof(SetAux), cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    if (!a.n) continue;
    if (big_layout[k] == EH_LAYOUT_RANGE_BITSET) {
      EH_CUDA(cudaMemsetAsync(t->bs_words.p + a.off, 0, (size_t)a.n * 8, s));
      big_bitset_fill_kernel<<<grid, 256, 0, s>>>(src, i, t->aux.p, t->bs_words.p);
      EH_CHECK_LAUNCH();
      // ranks: exclusive prefix of the words' popcounts
      DevBuf<uint32_t> popc(a.n, s);
      big_popc_kernel<<<grid, 256, 0, s>>>(t->aux.p, i, t->bs_words.p, popc.p);
      EH_CHECK_LAUNCH();
      exclusive_scan<uint32_t>(popc.p, t->bs_rank.p + a.off, a.n, btot.p, s);
    } else {
      EH_CUDA(cudaMemsetAsync(t->bb_words.p + 4 * (uint64_t)a.off, 0, (size_t)a.n * 32, s));
      EH_CUDA(cudaMemsetAsync(bcount.p, 0, 8, s));
      big_block_flags_kernel<<<grid, 256, 0, s>>>(src, i, bflag.p, bcount.p);
      EH_CHECK_LAUNCH();
      exclusive_scan<uint32_t>(bflag.p, bpos.p, big_len[k], btot.p, s);
      big_block_fill_kernel<<<grid, 256, 0, s>>>(src, i, t->aux.p, bflag.p, bpos.p, t->bb_id.p, t->bb_rank.p,
                                                 t->bb_words.p);
      EH_CHECK_LAUNCH();
    }
  }
  ph_big.end();
  TracePhase ph_hist("structs.hist", s);
  DevBuf<uint32_t> hist(4, s);
  EH_CUDA(cudaMemsetAsync(hist.p, 0, 16, s));
  if (t->n_head) {
    layout_hist_kernel<<<grid, 256, 0, s>>>(t->layout.p, t->n_head, hist.p);
    EH_CHECK_LAUNCH();
  }
  uint32_t hh[4];
  uint8_t head_layout = EH_LAYOUT_UINTEGER;
  EH_CUDA(cudaMemcpyAsync(hh, hist.p, 16, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaMemcpyAsync(&head_layout, t->layout.p + t->n_head, 1, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  t->info.n_range_bitset = hh[EH_LAYOUT_RANGE_BITSET];
  t->info.n_uinteger = hh[EH_LAYOUT_UINTEGER];
  t->info.n_block_bitset = hh[EH_LAYOUT_BLOCK_BITSET];
  t->info.head_layout = head_layout;
  t->info.bitset_words = h[0];
  t->info.block_count = h[1];
}

void build_layout_structs_public(eh_context* ctx, eh_trie* t) { build_layout_structs(ctx, t); }

static void update_bytes(eh_trie* t) {
  t->info.device_bytes = t->head.bytes() + t->head_index.bytes() + t->off.bytes() + t->vals.bytes() +
                         t->layout.bytes() + t->aux.bytes() + t->bs_words.bytes() + t->bs_rank.bytes() +
                         t->bb_id.bytes() + t->bb_rank.bytes() + t->bb_words.bytes() + t->wedges.bytes() +
                         t->rev_off.bytes() + t->rev_lo.bytes() + t->rev_hi.bytes() + t->rev_src.bytes() +
                         t->rev_wpre.bytes() + t->work_pred.bytes();
}

void trie_layout(eh_context* ctx, eh_trie* t, const eh_layout_config* cfg) {
  cudaStream_t s = ctx->stream;
  const uint32_t n_sets = t->n_head + 1;
  const int policy = cfg ? cfg->policy : EH_POLICY_HEURISTIC;
  const int forced = cfg ? cfg->forced_layout : EH_LAYOUT_UINTEGER;
  EH_REQUIRE(policy == EH_POLICY_HEURISTIC || policy == EH_POLICY_LEARNED || policy == EH_POLICY_FORCED ||
                 policy == EH_POLICY_EXPLICIT,
             EH_ERR_INVALID, "unknown layout policy");
  if (policy == EH_POLICY_EXPLICIT) {
    EH_REQUIRE(cfg->layouts != nullptr || t->n_head == 0, EH_ERR_INVALID, "explicit layout policy needs layouts");
    for (uint32_t i = 0; i < t->n_head; i++) {
      const uint8_t l = cfg->layouts[i];
      EH_REQUIRE(l == EH_LAYOUT_UINTEGER || l == EH_LAYOUT_RANGE_BITSET || l == EH_LAYOUT_BLOCK_BITSET,
                 EH_ERR_INVALID, "unknown layout in the explicit assignment");
    }
  }
  EH_REQUIRE(forced == EH_LAYOUT_UINTEGER || forced == EH_LAYOUT_RANGE_BITSET || forced == EH_LAYOUT_BLOCK_BITSET,
             EH_ERR_INVALID, "unknown forced layout");
  TracePhase ph("layout.choose", s);
  t->layout.alloc(n_sets, s);
  const uint64_t max_words = cfg ? cfg->max_bitset_bytes / 12 : 0;
  layout_heuristic_kernel<<<num_sms() * 4, 256, 0, s>>>(set_src(t), n_sets, policy, forced, max_words,
                                                         t->layout.p);
  EH_CHECK_LAUNCH();
  if (policy == EH_POLICY_EXPLICIT && t->n_head) {
    EH_CUDA(cudaMemcpyAsync(t->layout.p, cfg->layouts, t->n_head, cudaMemcpyHostToDevice, s));
    EH_CUDA(cudaStreamSynchronize(s));  // the host array may go away after the call
  }
  t->work_pred.release();
  t->pred_per_probe = 0;
  if (policy == EH_POLICY_LEARNED) {
    EH_REQUIRE(cfg->model != nullptr, EH_ERR_INVALID, "learned layout policy needs a model");
    if (t->n_head && t->rev_pairs) t->work_pred.alloc(t->n_head, s);
    model_choose_layouts(ctx, cfg->model, t, cfg->max_bitset_bytes, cfg->min_gain, t->layout.p, t->work_pred.p);
    if (t->work_pred.p) {
      DevBuf<double> sum(1, s);
      EH_CUDA(cudaMemsetAsync(sum.p, 0, 8, s));
      sum_f32_kernel<<<num_sms() * 4, 256, 0, s>>>(t->work_pred.p, t->n_head, sum.p);
      EH_CHECK_LAUNCH();
      double h = 0;
      EH_CUDA(cudaMemcpyAsync(&h, sum.p, 8, cudaMemcpyDeviceToHost, s));
      EH_CUDA(cudaStreamSynchronize(s));
      t->pred_per_probe = h / (double)t->rev_pairs;
    }
  }
  ph.end();
  TracePhase ph_s("layout.structs", s);
  build_layout_structs(ctx, t);
  update_bytes(t);
}

// value -> head position over the value domain [0, n_nodes)
static void build_head_index(eh_context* ctx, eh_trie* t) {
  cudaStream_t s = ctx->stream;
  t->head_index.alloc(t->n_nodes ? t->n_nodes : 1, s);
  EH_CUDA(cudaMemsetAsync(t->head_index.p, 0xff, (size_t)(t->n_nodes ? t->n_nodes : 1) * 4, s));
  if (t->n_head) {
    head_index_kernel<<<num_sms() * 8, 256, 0, s>>>(t->head.p, t->n_head, t->head_index.p);
    EH_CHECK_LAUNCH();
  }
}

// wedges per head entry, their total, the largest set, sum of squared sizes
static void build_stats(eh_context* ctx, eh_trie* t) {
  cudaStream_t s = ctx->stream;
  const int grid = num_sms() * 8;
  t->wedges.alloc(t->n_head ? t->n_head : 1, s);
  DevBuf<uint64_t> tot(1, s);
  if (t->n_head) {
    wedge_kernel<<<grid, 256, 0, s>>>(t->view(), t->wedges.p);
    EH_CHECK_LAUNCH();
    DevBuf<uint64_t> scratch(t->n_head, s);
    exclusive_scan<uint64_t>(t->wedges.p, scratch.p, t->n_head, tot.p, s);
    EH_CUDA(cudaMemcpyAsync(&t->total_wedges, tot.p, 8, cudaMemcpyDeviceToHost, s));
  }
  EH_CUDA(cudaStreamSynchronize(s));
  t->info.rows = t->rows;
  t->info.n_head = t->n_head;
  t->info.n_nodes = t->n_nodes;
  uint32_t mx = 0;
  t->sum_sq_deg = 0;
  if (t->n_head) {
    DevBuf<unsigned long long> red(2, s);
    EH_CUDA(cudaMemsetAsync(red.p, 0, 16, s));
    set_size_stats_kernel<<<grid, 256, 0, s>>>(t->off.p, t->n_head, red.p);
    EH_CHECK_LAUNCH();
    unsigned long long h[2];
    EH_CUDA(cudaMemcpyAsync(h, red.p, 16, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    mx = (uint32_t)h[0];
    t->sum_sq_deg = h[1];
  }
  t->info.max_set = mx;
}

void trie_build_from_csr(eh_context* ctx, eh_trie* t) {
  cudaStream_t s = ctx->stream;
  {
    TracePhase ph("build.index+stats", s);
    build_head_index(ctx, t);
    build_stats(ctx, t);
  }
  TracePhase ph("build.reverse", s);
  trie_build_reverse(ctx, t);
}

void trie_build(eh_context* ctx, const uint32_t* c0, const uint32_t* c1, uint64_t n, const eh_layout_config* cfg,
                eh_trie* t) {
  cudaStream_t s = ctx->stream;
  const int grid = num_sms() * 8;
  EH_CUDA(cudaEventRecord(ctx->ev0, s));
  const uint32_t m0 = n ? max_u32(c0, n, s) : 0, m1 = n ? max_u32(c1, n, s) : 0;
  const int b = bits_for(m1), ba = bits_for(m0);
  EH_REQUIRE(b + ba <= 64, EH_ERR_UNSUPPORTED, "value range too wide");
  uint64_t r = 0;
  t->n_nodes = n ? std::max(m0, m1) + 1 : 0;
  if (n) {
    TracePhase ph("build.sort+csr", s);
    DevBuf<uint64_t> keys(n, s), tmp(n, s);
    pack_rows_kernel<<<grid, 256, 0, s>>>(c0, c1, n, b, keys.p);
    EH_CHECK_LAUNCH();
    radix_sort_u64(keys.p, tmp.p, n, b + ba, s);
    r = unique_sorted_u64(keys.p, tmp.p, n, s);
    DevBuf<uint32_t> hpos(r, s), nh(1, s);
    head_flag_kernel<<<grid, 256, 0, s>>>(tmp.p, r, b, hpos.p);
    EH_CHECK_LAUNCH();
    exclusive_scan<uint32_t>(hpos.p, hpos.p, r, nh.p, s);
    uint32_t n_head = 0;
    EH_CUDA(cudaMemcpyAsync(&n_head, nh.p, 4, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    t->n_head = n_head;
    t->rows = r;
    t->head.alloc(n_head, s);
    t->off.alloc(n_head + 1, s);
    t->vals.alloc(r, s);
    csr_kernel<<<grid, 256, 0, s>>>(tmp.p, r, b, hpos.p, t->head.p, t->off.p, t->vals.p);
    EH_CHECK_LAUNCH();
    EH_CUDA(cudaMemcpyAsync(t->off.p + n_head, &r, 8, cudaMemcpyHostToDevice, s));
    EH_CUDA(cudaStreamSynchronize(s));  // &r is a host stack address
  } else {
    t->off.alloc(1, s);
    EH_CUDA(cudaMemsetAsync(t->off.p, 0, 8, s));
  }
  trie_build_from_csr(ctx, t);
  trie_layout(ctx, t, cfg);
  EH_CUDA(cudaEventRecord(ctx->ev1, s));
  EH_CUDA(cudaEventSynchronize(ctx->ev1));
  float ms = 0;
  EH_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  t->info.build_ms = ms;
}

// ---------------------------------------------------------- reverse level
__global__ void seg_kernel(const uint64_t* __restrict__ off, uint32_t nh, uint32_t* __restrict__ seg) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = warp; i < nh; i += nwarps)
    for (uint64_t e = off[i] + lane; e < off[i + 1]; e += 32) seg[e] = i;
}

// counts rows that are not "up" (b <= a), not "down" (b >= a), rows (a,b)
// whose mirror (b,a) is absent, and self-loops
template <bool kMirror>
__global__ void direction_kernel(TrieView t, const uint32_t* __restrict__ seg, unsigned long long* __restrict__ cnt) {
  unsigned long long not_up = 0, not_down = 0, no_mirror = 0, loops = 0;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < t.rows; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = t.head[seg[e]], b = t.vals[e];
    not_up += b <= a;
    not_down += b >= a;
    loops += a == b;
    if (!kMirror) continue;
    const int32_t hb = t.head_index[b];
    bool found = false;
    if (hb >= 0) {
      uint64_t lo = t.off[hb], hi = t.off[hb + 1];
      while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (t.vals[mid] < a) lo = mid + 1; else hi = mid;
      }
      found = lo < t.off[hb + 1] && t.vals[lo] == a;
    }
    no_mirror += !found;
  }
  not_up = warp_sum(not_up);
  not_down = warp_sum(not_down);
  no_mirror = warp_sum(no_mirror);
  loops = warp_sum(loops);
  if (lane_id() == 0) {
    atomicAdd(&cnt[0], not_up);
    atomicAdd(&cnt[1], not_down);
    atomicAdd(&cnt[2], no_mirror);
    atomicAdd(&cnt[3], loops);
  }
}

// candidate range inside N(a) for row e = (a -> b), by direction
__device__ __forceinline__ void rev_range(int dir, uint64_t e, uint64_t a_lo, uint64_t a_hi, uint64_t& lo,
                                          uint64_t& hi) {
  if (dir == DIR_UP || dir == DIR_SYM) { lo = e + 1; hi = a_hi; }
  else if (dir == DIR_DOWN) { lo = a_lo; hi = e; }
  else { lo = a_lo; hi = a_hi; }
}

// key = head position of b (sentinel for rows the plans never read),
// payload = the row; rows arrive in row order, so a stable sort on the key
// alone leaves each b's rows in row order
__global__ void rev_key_kernel(TrieView t, const uint32_t* __restrict__ seg, int dir, uint32_t sentinel,
                               uint32_t* __restrict__ keys, uint32_t* __restrict__ rowid, uint32_t* __restrict__ cnt) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < t.rows; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t ha = seg[e];
    const uint32_t a = t.head[ha], b = t.vals[e];
    const int32_t hb = t.head_index[b];
    uint64_t lo, hi;
    rev_range(dir, e, t.off[ha], t.off[ha + 1], lo, hi);
    const bool keep = hb >= 0 && hi > lo && (dir != DIR_SYM || a < b);
    keys[e] = keep ? (uint32_t)hb : sentinel;
    rowid[e] = (uint32_t)e;
    if (keep) atomicAdd(&cnt[hb], 1u);
  }
}

__global__ void widen_u32_kernel(const uint32_t* __restrict__ in, uint64_t n, uint64_t* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[i];
}

__global__ void rev_fill_kernel(TrieView t, const uint32_t* __restrict__ seg, int dir,
                                const uint32_t* __restrict__ rowid, uint64_t n, uint32_t* __restrict__ lo_out,
                                uint32_t* __restrict__ hi_out, uint32_t* __restrict__ src_out,
                                uint64_t* __restrict__ work) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t e = rowid[k];
    const uint32_t ha = seg[e];
    uint64_t lo, hi;
    rev_range(dir, e, t.off[ha], t.off[ha + 1], lo, hi);
    lo_out[k] = (uint32_t)lo;
    hi_out[k] = (uint32_t)hi;
    src_out[k] = ha;
    work[k] = hi - lo;
  }
}

static void reverse_from_keys(eh_context* ctx, eh_trie* t, DevBuf<uint32_t>& seg, DevBuf<uint32_t>& keys,
                              DevBuf<uint32_t>& ktmp, DevBuf<uint32_t>& rowid, DevBuf<uint32_t>& vtmp,
                              DevBuf<uint32_t>& per);

void trie_build_reverse(eh_context* ctx, eh_trie* t) {
  cudaStream_t s = ctx->stream;
  const int grid = num_sms() * 8;
  t->dir = DIR_GENERAL;
  t->rev_entries = 0;
  t->rev_pairs = 0;
  t->rev_off.alloc(t->n_head + 1, s);
  EH_CUDA(cudaMemsetAsync(t->rev_off.p, 0, (t->n_head + 1) * 8, s));
  if (!t->rows) {
    t->rev_lo.alloc(1, s);
    t->rev_hi.alloc(1, s);
    return;
  }
  EH_REQUIRE(t->rows < (1ull << 32), EH_ERR_UNSUPPORTED, "tries with 2^32 rows or more are not supported");
  DevBuf<uint32_t> seg(t->rows, s);
  TracePhase ph_dir("reverse.direction", s);
  seg_kernel<<<grid, 256, 0, s>>>(t->off.p, t->n_head, seg.p);
  EH_CHECK_LAUNCH();
  // direction: up / down from one cheap pass; the mirror search only when
  // the relation is neither
  DevBuf<unsigned long long> cnt(4, s);
  EH_CUDA(cudaMemsetAsync(cnt.p, 0, 32, s));
  direction_kernel<false><<<grid, 256, 0, s>>>(t->view(), seg.p, cnt.p);
  EH_CHECK_LAUNCH();
  unsigned long long c[4];
  EH_CUDA(cudaMemcpyAsync(c, cnt.p, 32, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  if (c[0] == 0) {
    t->dir = DIR_UP;
  } else if (c[1] == 0) {
    t->dir = DIR_DOWN;
  } else {
    EH_CUDA(cudaMemsetAsync(cnt.p, 0, 32, s));
    direction_kernel<true><<<grid, 256, 0, s>>>(t->view(), seg.p, cnt.p);
    EH_CHECK_LAUNCH();
    EH_CUDA(cudaMemcpyAsync(c, cnt.p, 32, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    // a symmetric relation takes the oriented schedule (each undirected
    // triangle once, times 3!) only without self-loops
    t->dir = (c[2] == 0 && c[3] == 0) ? DIR_SYM : DIR_GENERAL;
  }
  ph_dir.end();
  // group the rows a->b the plans read by b (stable: row order within b);
  // head positions are below 2^32, so 32-bit keys on bits_for(n_head) bits
  const int bh = bits_for(t->n_head);
  const uint32_t sentinel = (uint32_t)((1ull << bh) - 1);  // above every head position
  DevBuf<uint32_t> keys(t->rows, s), ktmp(t->rows, s);
  DevBuf<uint32_t> rowid(t->rows, s), vtmp(t->rows, s);
  DevBuf<uint32_t> per(t->n_head + 1, s);
  EH_CUDA(cudaMemsetAsync(per.p, 0, (t->n_head + 1) * 4, s));
  TracePhase ph_key("reverse.keys", s);
  rev_key_kernel<<<grid, 256, 0, s>>>(t->view(), seg.p, t->dir, sentinel, keys.p, rowid.p, per.p);
  EH_CHECK_LAUNCH();
  ph_key.end();
  reverse_from_keys(ctx, t, seg, keys, ktmp, rowid, vtmp, per);
}

// The reverse level from its keys (head position of b per row, sentinel for
// rows no plan reads), the row ids and the per-b row counts: a stable sort of
// the row ids by key, offsets, and the per-entry ranges and work.
static void reverse_from_keys(eh_context* ctx, eh_trie* t, DevBuf<uint32_t>& seg, DevBuf<uint32_t>& keys,
                              DevBuf<uint32_t>& ktmp, DevBuf<uint32_t>& rowid, DevBuf<uint32_t>& vtmp,
                              DevBuf<uint32_t>& per) {
  cudaStream_t s = ctx->stream;
  const int grid = num_sms() * 8;
  const int bh = bits_for(t->n_head);
  TracePhase ph_sort("reverse.sort", s);
  const uint32_t* sorted = radix_sort_payload_u32(keys.p, ktmp.p, rowid.p, vtmp.p, t->rows, bh, s);
  // only the sorted row ids are read from here on: hand the sort's other
  // buffers (768 MB at R-MAT-22) back to the pool before the reverse arrays
  // are allocated
  keys.release();
  ktmp.release();
  if (sorted == rowid.p)
    vtmp.release();
  else
    rowid.release();
  ph_sort.end();
  TracePhase ph_fill("reverse.offsets+fill", s);
  {
    DevBuf<uint64_t> per64(t->n_head + 1, s);
    widen_u32_kernel<<<grid, 256, 0, s>>>(per.p, t->n_head + 1, per64.p);
    EH_CHECK_LAUNCH();
    DevBuf<uint64_t> tot(1, s);
    exclusive_scan<uint64_t>(per64.p, t->rev_off.p, t->n_head + 1, tot.p, s);
    uint64_t n64 = 0;
    EH_CUDA(cudaMemcpyAsync(&n64, tot.p, 8, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    t->rev_entries = n64;
  }
  const uint64_t n = t->rev_entries;
  t->rev_lo.alloc(n ? n : 1, s);
  t->rev_hi.alloc(n ? n : 1, s);
  t->rev_src.alloc(n ? n : 1, s);
  t->rev_wpre.alloc(n + 1, s);
  EH_CUDA(cudaMemsetAsync(t->rev_wpre.p, 0, (n + 1) * 8, s));
  if (n) {
    rev_fill_kernel<<<grid, 256, 0, s>>>(t->view(), seg.p, t->dir, sorted, n, t->rev_lo.p, t->rev_hi.p,
                                         t->rev_src.p, t->rev_wpre.p);
    EH_CHECK_LAUNCH();
    exclusive_scan<uint64_t>(t->rev_wpre.p, t->rev_wpre.p, n, t->rev_wpre.p + n, s);
    EH_CUDA(cudaMemcpyAsync(&t->rev_pairs, t->rev_wpre.p + n, 8, cudaMemcpyDeviceToHost, s));
  }
  EH_CUDA(cudaStreamSynchronize(s));
}

// Rows [r0, r1) of a CSR whose values have just arrived from the host: the
// largest value, the direction counts (rows not going up, not going down,
// self-loops), and the reverse level's keys as if every row went up (the
// common case; trie_build_from_host_csr recomputes them when it is not).
// Values at or above n_alloc are outside the head index and match no head
// entry.
__global__ void host_chunk_kernel(TrieView t, uint64_t r0, uint64_t r1, const uint32_t* __restrict__ seg,
                                  uint32_t n_alloc, uint32_t sentinel, uint32_t* __restrict__ keys,
                                  uint32_t* __restrict__ rowid, uint32_t* __restrict__ per,
                                  unsigned int* __restrict__ vmax, unsigned long long* __restrict__ cnt) {
  unsigned int mx = 0;
  unsigned long long not_up = 0, not_down = 0, loops = 0;
  for (uint64_t e = r0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < r1;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t ha = seg[e];
    const uint32_t a = t.head[ha], b = t.vals[e];
    mx = max(mx, b);
    not_up += b <= a;
    not_down += b >= a;
    loops += a == b;
    const int32_t hb = b < n_alloc ? t.head_index[b] : -1;
    const bool keep = hb >= 0 && e + 1 < t.off[ha + 1];
    keys[e] = keep ? (uint32_t)hb : sentinel;
    rowid[e] = (uint32_t)e;
    if (keep) atomicAdd(&per[hb], 1u);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(kFull, mx, o));
  not_up = warp_sum(not_up);
  not_down = warp_sum(not_down);
  loops = warp_sum(loops);
  if (lane_id() == 0) {
    atomicMax(vmax, mx);
    atomicAdd(&cnt[0], not_up);
    atomicAdd(&cnt[1], not_down);
    atomicAdd(&cnt[3], loops);
  }
}

// A trie from a CSR in host memory (head[n_head] sorted distinct values,
// off[n_head+1], vals[rows] sorted within each set), with the copy of vals
// overlapped with the work that needs only the rows already arrived: vals go
// up in chunks on the context's copy stream, and behind each chunk the
// context stream computes the row sources, the direction counts and the
// reverse level's keys.  When the relation turns out not to go up, or a value
// lies outside the domain the head index was sized for, the reverse level is
// rebuilt by the regular path; the trie is the same either way.
void trie_build_from_host_csr(eh_context* ctx, eh_trie* t, const uint32_t* head, const uint64_t* off,
                              const uint32_t* vals, uint32_t n_nodes_hint) {
  cudaStream_t s = ctx->stream;
  const int grid = num_sms() * 8;
  TracePhase ph_all("host_csr.build", s);
  t->head.alloc(t->n_head ? t->n_head : 1, s);
  t->off.alloc(t->n_head + 1, s);
  t->vals.alloc(t->rows ? t->rows : 1, s);
  if (t->n_head) EH_CUDA(cudaMemcpyAsync(t->head.p, head, (size_t)t->n_head * 4, cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaMemcpyAsync(t->off.p, off, ((size_t)t->n_head + 1) * 8, cudaMemcpyHostToDevice, s));
  if (!t->rows || !t->n_head) {
    if (t->rows) EH_CUDA(cudaMemcpyAsync(t->vals.p, vals, t->rows * 4, cudaMemcpyHostToDevice, s));
    const uint32_t mh = t->n_head ? max_u32(t->head.p, t->n_head, s) : 0;
    const uint32_t mv = t->rows ? max_u32(t->vals.p, t->rows, s) : 0;
    t->n_nodes = (t->n_head || t->rows) ? std::max(n_nodes_hint, std::max(mh, mv) + 1) : 0;
    trie_build_from_csr(ctx, t);
    return;
  }
  // vals in chunks on the copy stream, after the allocation on the context stream
  if (!ctx->copy_stream) EH_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  constexpr int kChunks = 8;
  cudaEvent_t ev[kChunks + 1] = {};
  struct Events {
    cudaEvent_t* e;
    ~Events() {
      for (int i = 0; i <= kChunks; i++)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } guard{ev};
  for (int i = 0; i <= kChunks; i++) EH_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
  EH_CUDA(cudaEventRecord(ev[kChunks], s));
  EH_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ev[kChunks], 0));
  uint64_t bound[kChunks + 1];
  for (int i = 0; i <= kChunks; i++) bound[i] = t->rows * (uint64_t)i / kChunks;
  for (int i = 0; i < kChunks; i++) {
    if (bound[i + 1] > bound[i])
      EH_CUDA(cudaMemcpyAsync(t->vals.p + bound[i], vals + bound[i], (bound[i + 1] - bound[i]) * 4,
                              cudaMemcpyHostToDevice, ctx->copy_stream));
    EH_CUDA(cudaEventRecord(ev[i], ctx->copy_stream));
  }
  // the head index from the head alone (values beyond it are outside every set's head)
  const uint32_t mh = max_u32(t->head.p, t->n_head, s);
  const uint32_t n_alloc = std::max(n_nodes_hint, mh + 1);
  t->n_nodes = n_alloc;
  build_head_index(ctx, t);
  DevBuf<uint32_t> seg(t->rows, s);
  seg_kernel<<<grid, 256, 0, s>>>(t->off.p, t->n_head, seg.p);
  EH_CHECK_LAUNCH();
  const int bh = bits_for(t->n_head);
  const uint32_t sentinel = (uint32_t)((1ull << bh) - 1);
  DevBuf<uint32_t> keys(t->rows, s), ktmp(t->rows, s), rowid(t->rows, s), vtmp(t->rows, s);
  DevBuf<uint32_t> per(t->n_head + 1, s);
  DevBuf<unsigned long long> cnt(4, s);
  DevBuf<unsigned int> vmax(1, s);
  EH_CUDA(cudaMemsetAsync(per.p, 0, ((size_t)t->n_head + 1) * 4, s));
  EH_CUDA(cudaMemsetAsync(cnt.p, 0, 32, s));
  EH_CUDA(cudaMemsetAsync(vmax.p, 0, 4, s));
  for (int i = 0; i < kChunks; i++) {
    EH_CUDA(cudaStreamWaitEvent(s, ev[i], 0));
    if (bound[i + 1] > bound[i]) {
      host_chunk_kernel<<<grid, 256, 0, s>>>(t->view(), bound[i], bound[i + 1], seg.p, n_alloc, sentinel, keys.p,
                                             rowid.p, per.p, vmax.p, cnt.p);
      EH_CHECK_LAUNCH();
    }
  }
  unsigned long long c[4];
  unsigned int vm = 0;
  EH_CUDA(cudaMemcpyAsync(c, cnt.p, 32, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaMemcpyAsync(&vm, vmax.p, 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  if (vm >= n_alloc) {  // a value beyond the hint and the head: the whole domain again
    t->n_nodes = vm + 1;
    build_head_index(ctx, t);
  }
  {
    TracePhase ph("build.index+stats", s);
    build_stats(ctx, t);
  }
  TracePhase ph("build.reverse", s);
  if (vm < n_alloc && c[0] == 0) {  // every row goes up: the keys stand
    t->dir = DIR_UP;
    t->rev_off.alloc(t->n_head + 1, s);
    reverse_from_keys(ctx, t, seg, keys, ktmp, rowid, vtmp, per);
  } else {
    seg.release();
    keys.release();
    ktmp.release();
    rowid.release();
    vtmp.release();
    trie_build_reverse(ctx, t);
  }
}

// Reference-format bytes of one set (see eh_trie_set_bytes in eh_b200.h).
void trie_set_bytes(const eh_trie* t, uint32_t set_index, std::vector<uint8_t>& out, uint8_t* layout_out) {
  cudaStream_t s = t->ctx->stream;
  const bool is_head = set_index == UINT32_MAX;
  EH_REQUIRE(is_head || set_index < t->n_head, EH_ERR_INVALID, "set index out of range");
  const uint32_t i = is_head ? t->n_head : set_index;
  uint8_t layout = 0;
  SetAux a{};
  uint64_t o[2] = {0, 0};
  EH_CUDA(cudaMemcpyAsync(&layout, t->layout.p + i, 1, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaMemcpyAsync(&a, t->aux.p + i, sizeof(SetAux), cudaMemcpyDeviceToHost, s));
  if (!is_head) EH_CUDA(cudaMemcpyAsync(o, t->off.p + i, 16, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  const uint64_t len = is_head ? t->n_head : o[1] - o[0];
  const uint32_t* elems = is_head ? t->head.p : t->vals.p + o[0];
  if (layout_out) *layout_out = layout;
  out.clear();
  if (!len) return;
  if (layout == EH_LAYOUT_UINTEGER) {
    out.resize(len * 4);
    EH_CUDA(cudaMemcpyAsync(out.data(), elems, len * 4, cudaMemcpyDeviceToHost, s));
  } else if (layout == EH_LAYOUT_RANGE_BITSET) {
    out.resize(8 + (size_t)a.n * 12);
    const uint64_t start = a.start;
    memcpy(out.data(), &start, 8);
    EH_CUDA(cudaMemcpyAsync(out.data() + 8, t->bs_words.p + a.off, (size_t)a.n * 8, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaMemcpyAsync(out.data() + 8 + (size_t)a.n * 8, t->bs_rank.p + a.off, (size_t)a.n * 4,
                            cudaMemcpyDeviceToHost, s));
  } else if (layout == EH_LAYOUT_BLOCK_BITSET) {
    std::vector<uint32_t> ids(a.n), rk(a.n);
    std::vector<uint64_t> w((size_t)a.n * 4);
    EH_CUDA(cudaMemcpyAsync(ids.data(), t->bb_id.p + a.off, (size_t)a.n * 4, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaMemcpyAsync(rk.data(), t->bb_rank.p + a.off, (size_t)a.n * 4, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaMemcpyAsync(w.data(), t->bb_words.p + 4 * a.off, (size_t)a.n * 32, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    out.resize((size_t)a.n * 40);
    for (uint32_t k = 0; k < a.n; k++) {
      memcpy(out.data() + 40 * (size_t)k, &ids[k], 4);
      memcpy(out.data() + 40 * (size_t)k + 4, &rk[k], 4);
      memcpy(out.data() + 40 * (size_t)k + 8, &w[4 * (size_t)k], 32);
    }
  }
  EH_CUDA(cudaStreamSynchronize(s));
}

}  // namespace eh
