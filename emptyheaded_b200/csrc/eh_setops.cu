// Pairwise set intersection for every layout pair, count and materialize.
//
// Reference: ops::set_intersect (trie/set/ops/intersection/set.hpp:9-167)
// dispatches on the two layouts:
//   uint ∩ uint      uinteger.hpp:1209-1261 (shuffle, or galloping when the
//                    cardinality ratio exceeds 32), rare = the smaller set
//   uint ∩ bitset    hetero.hpp:29-60 (probe each uint in the bitset)
//   bitset ∩ bitset  bitset.hpp:619-661 (AND over the overlapping words)
//   block variants   hetero.hpp:107-309, bitset.hpp:685-757
// Here one warp handles one pair:
//   uint ∩ uint      the smaller set is streamed 32 elements at a time; each
//                    lane probes the larger set by branch-free binary search
//                    (shared memory when it fits)
//   X ∩ bitset       the other set is streamed, one word test per element
//   bitset ∩ bitset  one 64-bit word of each range per lane over their
//                    overlap (coalesced), AND + popcount, warp reduction
//   X ∩ block        streamed elements probe the block ids
// Materialized results are written in increasing order (ballot compaction
// of the streamed side, or bit order of the AND-ed words).
#include <algorithm>
#include <cstring>

#include "eh_internal.cuh"

namespace eh {

void build_layout_structs_public(eh_context* ctx, eh_trie* t);

struct PairOut {
  unsigned long long* counts;
  const uint64_t* out_off;  // null: count only
  uint32_t* out;
};

__device__ __forceinline__ bool contains_sorted(const uint32_t* p, uint32_t n, uint32_t w, bool shared) {
  if (!n) return false;
  uint32_t base = 0;
  while (n > 1) {
    const uint32_t half = n >> 1;
    const uint32_t v = shared ? p[base + half] : __ldg(p + base + half);
    base = (v <= w) ? base + half : base;
    n -= half;
  }
  return (shared ? p[base] : __ldg(p + base)) == w;
}

// membership of w in set i of trie t, by the set's layout
__device__ __forceinline__ bool member(const TrieView& t, uint32_t i, uint32_t w, const uint32_t* sm_list,
                                       uint32_t sm_n) {
  const uint8_t l = t.layout[i];
  const SetAux a = t.aux[i];
  if (l == EH_LAYOUT_RANGE_BITSET) {
    const uint32_t idx = (w >> 6) - a.start;
    if (idx >= a.n) return false;
    return (__ldg(t.bs_words + a.off + idx) >> (w & 63)) & 1ull;
  }
  if (l == EH_LAYOUT_BLOCK_BITSET) {
    const uint32_t id = w >> 8;
    uint32_t lo = 0, hi = a.n;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(t.bb_id + a.off + mid) < id) lo = mid + 1; else hi = mid;
    }
    if (lo >= a.n || __ldg(t.bb_id + a.off + lo) != id) return false;
    return (__ldg(t.bb_words + 4 * (a.off + lo) + ((w >> 6) & 3)) >> (w & 63)) & 1ull;
  }
  if (sm_list) return contains_sorted(sm_list, sm_n, w, true);
  const uint64_t s0 = t.off[i];
  return contains_sorted(t.vals + s0, (uint32_t)(t.off[i + 1] - s0), w, false);
}

constexpr int kPairWarps = 4;
constexpr int kPairCap = 2048;  // u32 per warp

__global__ void __launch_bounds__(32 * kPairWarps) pair_kernel(TrieView t, const uint32_t* __restrict__ pa,
                                                                const uint32_t* __restrict__ pb, uint32_t n_pairs,
                                                                PairOut out) {
  __shared__ uint32_t smem[kPairWarps][kPairCap];
  const uint32_t lane = lane_id();
  const uint32_t wid = threadIdx.x >> 5;
  const uint32_t gw = blockIdx.x * kPairWarps + wid;
  const uint32_t nw = gridDim.x * kPairWarps;
  uint32_t* sm = smem[wid];
  for (uint32_t p = gw; p < n_pairs; p += nw) {
    uint32_t A = pa[p], B = pb[p];
    const uint64_t la = t.off[A + 1] - t.off[A], lb = t.off[B + 1] - t.off[B];
    uint32_t* dst = out.out_off ? out.out + out.out_off[p] : nullptr;
    uint64_t count = 0;
    if (la && lb) {
      const uint8_t ya = t.layout[A], yb = t.layout[B];
      if (ya == EH_LAYOUT_RANGE_BITSET && yb == EH_LAYOUT_RANGE_BITSET) {
        // AND over the overlapping word range
        const SetAux a = t.aux[A], b = t.aux[B];
        const uint32_t s = max(a.start, b.start);
        const uint32_t e = min(a.start + a.n, b.start + b.n);
        const uint64_t* wa = t.bs_words + a.off + (s - a.start);
        const uint64_t* wb = t.bs_words + b.off + (s - b.start);
        const uint32_t nwds = e > s ? e - s : 0;
        uint64_t written = 0;
        for (uint32_t base = 0; base < nwds; base += 32) {
          const uint32_t j = base + lane;
          const uint64_t x = j < nwds ? (__ldg(wa + j) & __ldg(wb + j)) : 0ull;
          const uint32_t c = (uint32_t)__popcll(x);
          const uint32_t inc = warp_incl_scan(c);
          if (dst) {
            uint64_t pos = written + inc - c;
            uint64_t y = x;
            while (y) {
              const int bit = __ffsll((long long)y) - 1;
              dst[pos++] = ((s + j) << 6) | (uint32_t)bit;
              y &= y - 1;
            }
          }
          written += __shfl_sync(kFull, inc, 31);
        }
        count = written;
      } else {
        // stream one side, probe the other
        uint32_t S = A, P = B;  // streamed, probed
        uint64_t ls = la;
        const bool a_bits = ya != EH_LAYOUT_UINTEGER, b_bits = yb != EH_LAYOUT_UINTEGER;
        if (a_bits && !b_bits) { S = B; P = A; ls = lb; }
        else if (!a_bits && !b_bits && la > lb) { S = B; P = A; ls = lb; }  // rare = smaller
        const uint64_t lp = t.off[P + 1] - t.off[P];
        const uint32_t* smp = nullptr;
        if (t.layout[P] == EH_LAYOUT_UINTEGER && lp <= (uint64_t)kPairCap) {
          for (uint32_t j = lane; j < lp; j += 32) sm[j] = __ldg(t.vals + t.off[P] + j);
          __syncwarp();
          smp = sm;
        }
        const uint32_t* sv = t.vals + t.off[S];
        uint64_t written = 0;
        for (uint64_t base = 0; base < ls; base += 32) {
          const uint64_t j = base + lane;
          bool hit = false;
          uint32_t w = 0;
          if (j < ls) {
            w = __ldg(sv + j);
            hit = member(t, P, w, smp, (uint32_t)lp);
          }
          const uint32_t ball = __ballot_sync(kFull, hit);
          if (dst && hit) dst[written + __popc(ball & lanemask_lt())] = w;
          written += __popc(ball);
        }
        count = written;
        __syncwarp();
      }
    }
    if (lane == 0) out.counts[p] = count;
  }
}

void set_intersect_batch(eh_context* ctx, const uint32_t* elems, const uint64_t* set_off, uint32_t n_sets,
                         const uint8_t* layouts, const uint32_t* pair_a, const uint32_t* pair_b, uint32_t n_pairs,
                         uint64_t* counts, const uint64_t* out_off, uint32_t* out_elems) {
  cudaStream_t s = ctx->stream;
  EH_REQUIRE(n_sets > 0, EH_ERR_INVALID, "no sets");
  EH_REQUIRE(set_off[0] == 0, EH_ERR_INVALID, "set_off[0] must be 0");
  const uint64_t total = set_off[n_sets];
  uint32_t max_val = 0;
  for (uint32_t k = 0; k < n_sets; k++) {
    EH_REQUIRE(set_off[k + 1] >= set_off[k], EH_ERR_INVALID, "set_off must be non-decreasing");
    const uint8_t l = layouts[k];
    EH_REQUIRE(l == EH_LAYOUT_UINTEGER || l == EH_LAYOUT_RANGE_BITSET || l == EH_LAYOUT_BLOCK_BITSET, EH_ERR_INVALID,
               "unknown layout code");
    for (uint64_t j = set_off[k] + 1; j < set_off[k + 1]; j++)
      EH_REQUIRE(elems[j] > elems[j - 1], EH_ERR_INVALID, "sets must be strictly increasing");
    if (set_off[k + 1] > set_off[k]) max_val = std::max(max_val, elems[set_off[k + 1] - 1]);
  }
  for (uint32_t p = 0; p < n_pairs; p++)
    EH_REQUIRE(pair_a[p] < n_sets && pair_b[p] < n_sets, EH_ERR_INVALID, "pair index out of range");
  if (!n_pairs) return;

  eh_trie t;
  t.ctx = ctx;
  t.n_head = n_sets;
  t.rows = total;
  t.n_nodes = std::max<uint32_t>(max_val + 1, n_sets);
  std::vector<uint32_t> head(n_sets);
  for (uint32_t k = 0; k < n_sets; k++) head[k] = k;
  t.head.alloc(n_sets, s);
  t.off.alloc(n_sets + 1, s);
  t.vals.alloc(total ? total : 1, s);
  t.layout.alloc(n_sets + 1, s);
  std::vector<uint8_t> lay(layouts, layouts + n_sets);
  lay.push_back(EH_LAYOUT_UINTEGER);  // the id head is never probed
  EH_CUDA(cudaMemcpyAsync(t.head.p, head.data(), n_sets * 4, cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaMemcpyAsync(t.off.p, set_off, (n_sets + 1) * 8, cudaMemcpyHostToDevice, s));
  if (total) EH_CUDA(cudaMemcpyAsync(t.vals.p, elems, total * 4, cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaMemcpyAsync(t.layout.p, lay.data(), n_sets + 1, cudaMemcpyHostToDevice, s));
  build_layout_structs_public(ctx, &t);

  DevBuf<uint32_t> da(n_pairs, s), db(n_pairs, s);
  DevBuf<unsigned long long> dc(n_pairs, s);
  EH_CUDA(cudaMemcpyAsync(da.p, pair_a, n_pairs * 4, cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaMemcpyAsync(db.p, pair_b, n_pairs * 4, cudaMemcpyHostToDevice, s));
  DevBuf<uint64_t> doff;
  DevBuf<uint32_t> dout;
  uint64_t out_cap = 0;
  if (out_off) {
    for (uint32_t p = 0; p < n_pairs; p++) {
      const uint64_t la = set_off[pair_a[p] + 1] - set_off[pair_a[p]];
      const uint64_t lb = set_off[pair_b[p] + 1] - set_off[pair_b[p]];
      out_cap = std::max(out_cap, out_off[p] + std::min(la, lb));
    }
    doff.alloc(n_pairs, s);
    dout.alloc(out_cap ? out_cap : 1, s);
    EH_CUDA(cudaMemcpyAsync(doff.p, out_off, n_pairs * 8, cudaMemcpyHostToDevice, s));
  }
  PairOut po{dc.p, out_off ? doff.p : nullptr, out_off ? dout.p : nullptr};
  const int grid = std::min<int>(num_sms() * 8, (n_pairs + kPairWarps - 1) / kPairWarps);
  pair_kernel<<<grid, 32 * kPairWarps, 0, s>>>(t.view(), da.p, db.p, n_pairs, po);
  EH_CHECK_LAUNCH();
  EH_CUDA(cudaMemcpyAsync(counts, dc.p, n_pairs * 8, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  if (out_off && out_cap) {
    // one copy of the whole output region (each pair's region beyond its
    // count is reserved for it by the caller)
    EH_CUDA(cudaMemcpyAsync(out_elems, dout.p, out_cap * 4, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
  }
}

}  // namespace eh
