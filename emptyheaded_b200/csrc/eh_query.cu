// Generic-join COUNT executors for the named plans.
//
// Reference loop nest (triangle, order [a,b,c]; EHGenerator.scala:273-480,
// TrieBuilder.cpp:242-274, ParTrieBuilder::par_foreach_aggregate
// TrieBuilder.hpp:152-157):
//     for a in head ∩ head (parallel, par::for_range chunks):
//       for b in N(a) ∩ head:
//         count += |N(b) ∩ N(a)|          (ops::set_intersect, set.hpp:9-167)
// The same pairwise intersections are scheduled here grouped by b: N(b) is
// staged once in shared memory in its stored layout (uint -> sorted list,
// range bitset -> words, block bitset -> ids + words) and every row a->b
// streams the part of N(a) that can still meet N(b) (the reverse level of
// the trie, built with it).  The sum is unchanged: it is the same set of
// (a,b) intersections.  Work items are (b, range of rows a->b) chunks of
// about `chunk_pairs` probes, pulled by warps of a persistent kernel from
// an atomic queue, heaviest b first.
#include <algorithm>

#include "eh_internal.cuh"

namespace eh {

// Register budget of the intersection kernels, set by their launch bounds
// (threads per block, optional blocks per SM); the block size knob is
// capped to match.
#ifndef EH_TRI_MAX_THREADS
#define EH_TRI_MAX_THREADS 512
#endif
#ifdef EH_TRI_MIN_BLOCKS
#define EH_TRI_LAUNCH_BOUNDS __launch_bounds__(EH_TRI_MAX_THREADS, EH_TRI_MIN_BLOCKS)
#else
#define EH_TRI_LAUNCH_BOUNDS __launch_bounds__(EH_TRI_MAX_THREADS)
#endif
constexpr int kMaxWarps = EH_TRI_MAX_THREADS / 32;  // per block
constexpr int kDefaultWarps = kMaxWarps < 8 ? kMaxWarps : 8;
constexpr uint32_t kDefaultLongRow = 32;  // rows with at least this many candidates run warp-wide
#ifndef EH_LONG_UNROLL
#define EH_LONG_UNROLL 4
#endif
constexpr int kLongUnroll = EH_LONG_UNROLL;  // independent candidate loads per lane per trip
#ifndef EH_SHORT_UNROLL
#define EH_SHORT_UNROLL 4
#endif
constexpr int kShortUnroll = EH_SHORT_UNROLL;  // flattened (row, element) pairs per lane per trip
#ifndef EH_WORD_UNROLL
#define EH_WORD_UNROLL 1
#endif
constexpr int kWordUnroll = EH_WORD_UNROLL;  // flattened (row, word) pairs per lane per trip
#ifndef EH_LONG_WORD_UNROLL
#define EH_LONG_WORD_UNROLL 1
#endif
constexpr int kLongWordUnroll = EH_LONG_WORD_UNROLL;  // 16-byte N(a) loads per lane per trip of a long word row
#ifndef EH_WORD_ROW_NUM
#define EH_WORD_ROW_NUM 5
#endif
#ifndef EH_WORD_ROW_DEN
#define EH_WORD_ROW_DEN 4
#endif
// a row runs word by word when words * num < candidates * den: a word costs
// about 1.25 candidate probes (measured on B200 at R-MAT-22: 5/4 against 1/1
// 8.34 vs 8.46 ms with the per-set best layouts, 9.87 vs 9.91 with the rule)
constexpr uint32_t kWordRowNum = EH_WORD_ROW_NUM, kWordRowDen = EH_WORD_ROW_DEN;
#ifndef EH_LONG_WORDS
#define EH_LONG_WORDS 32
#endif
constexpr int kLongWords = EH_LONG_WORDS;  // word rows with at least this many words run warp-wide
#ifndef EH_FLAT_CLIQUE
#define EH_FLAT_CLIQUE 48
#endif
constexpr uint32_t kFlatClique = EH_FLAT_CLIQUE;  // 4-clique: S up to this size has its pairs flattened
// Defaults measured on B200 at R-MAT-22 (4 KB of staging per warp leaves
// room for 32 resident warps; 32K-probe items amortise staging); the
// autotuner (emptyheaded_b200/autotune.py) re-picks them per trie.
constexpr int kDefaultSmemWords = 1024;  // per warp
constexpr int kDefaultChunk = 32768;

struct RevView {
  const uint64_t* rev_off;
  const uint32_t* rev_lo;
  const uint32_t* rev_hi;
  const uint32_t* rev_src;
  const uint64_t* rev_wpre;
  int dir;
};

struct Item {  // 16 bytes
  uint32_t hb, kb, ke, g;
};

struct ExecParams {
  int warps;
  int smem_words;
  uint32_t chunk;
  uint32_t shard_index, shard_count;
  uint32_t long_row;
  uint32_t s_cap;  // 4-clique: S buffers in global memory of this many words per warp (0: in shared memory)
  bool smem_given; // the caller chose smem_words
  bool no_block_items;  // stage every N(b) per warp (no block items)
};

static ExecParams exec_params(const eh_exec_config* cfg) {
  ExecParams p;
  p.warps = (cfg && cfg->warps_per_block > 0) ? cfg->warps_per_block : kDefaultWarps;
  p.smem_words = (cfg && cfg->smem_words > 0) ? cfg->smem_words : kDefaultSmemWords;
  p.chunk = (cfg && cfg->chunk_pairs > 0) ? (uint32_t)cfg->chunk_pairs : (uint32_t)kDefaultChunk;
  p.long_row = (cfg && cfg->long_row > 0) ? (uint32_t)cfg->long_row : kDefaultLongRow;
  p.shard_count = (cfg && cfg->shard_count > 1) ? (uint32_t)cfg->shard_count : 1u;
  p.shard_index = (cfg && cfg->shard_count > 1) ? (uint32_t)cfg->shard_index : 0u;
  EH_REQUIRE(p.shard_index < p.shard_count, EH_ERR_INVALID, "shard_index must be below shard_count");
  p.s_cap = 0;
  p.smem_given = cfg && cfg->smem_words > 0;
  p.no_block_items = cfg && cfg->no_block_items;
  p.warps = std::max(1, std::min(p.warps, kMaxWarps));
  p.smem_words = std::max(64, std::min(p.smem_words, 16384)) & ~1;
  return p;
}

// ---------------------------------------------------------------- planning
// items per head entry b: ceil(work(b) / chunk)
__global__ void plan_count_kernel(RevView r, uint32_t nh, uint32_t chunk, uint32_t* __restrict__ nitems) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nh; b += gridDim.x * blockDim.x) {
    const uint64_t w = r.rev_wpre[r.rev_off[b + 1]] - r.rev_wpre[r.rev_off[b]];
    nitems[b] = (uint32_t)((w + chunk - 1) / chunk);
  }
}
// item i of b covers the rows whose work prefix falls in [i, i+1) * W/n;
// items are written in reverse head order so the queue starts at the
// largest-degree b (ids are degree-ordered) and small items come last.
// first row k in [lo, hi) with wpre[k] >= target (hi if none)
__device__ __forceinline__ uint64_t first_row_at(const uint64_t* __restrict__ wpre, uint64_t lo, uint64_t hi,
                                                 uint64_t target) {
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (wpre[mid] < target) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// One thread per item: item q belongs to the last head entry b with
// ipos[b] <= q (ipos is the exclusive scan of the items per entry, so entries
// without items share the next entry's offset and are never found), is item
// i = q - ipos[b] of b, and covers the rows from the first one at target i to
// the first one at target i + 1 -- two independent searches over b's rows.
// The work prefix is non-decreasing, so these are the bounds a serial cut of
// b's items one after the other finds, at any number of items per entry.
__global__ void plan_fill_kernel(RevView r, uint32_t nh, const uint32_t* __restrict__ nitems,
                                 const uint32_t* __restrict__ ipos, uint32_t total, uint32_t g,
                                 Item* __restrict__ items) {
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nh;  // first entry with ipos > q
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (ipos[mid] <= q) lo = mid + 1; else hi = mid;
    }
    const uint32_t b = lo - 1;  // q < total = ipos[nh-1] + nitems[nh-1], so lo >= 1
    const uint32_t i = q - ipos[b], n = nitems[b];
    const uint64_t k0 = r.rev_off[b], k1 = r.rev_off[b + 1];
    const uint64_t w0 = r.rev_wpre[k0], W = r.rev_wpre[k1] - w0;
    const uint64_t kb = i ? first_row_at(r.rev_wpre, k0, k1, w0 + (W * i) / n) : k0;
    const uint64_t ke = i + 1 < n ? first_row_at(r.rev_wpre, kb, k1, w0 + (W * (i + 1)) / n) : k1;
    items[total - 1 - q] = Item{b, (uint32_t)kb, (uint32_t)ke, g};
  }
}


// u32 words a compressed staging (P_ZBITS, below) of a W-word range bitset
// with len elements takes at most: a (presence mask, rank) pair per 32 words
// and at most min(len, W) non-zero 64-bit words
__host__ __device__ __forceinline__ uint32_t zbits_words(uint32_t W, uint32_t len) {
  const uint32_t groups = (W + 31) / 32;
  return 2 * groups + 2 * (len < W ? len : W);
}

// Work of head entry b is staged in one of two classes: per warp (N(b)
// fits a warp's shared region, or must be probed in global memory) or per
// block (N(b) needs more than a warp's region but fits the block's: every
// warp of the block works on the rows of one staged N(b)).  A block item
// holds `warps` times a warp item's work.
__device__ __forceinline__ uint32_t staged_words(const TrieView& t, uint32_t b, uint32_t warp_words) {
  const uint8_t l = t.layout[b];
  if (l == EH_LAYOUT_RANGE_BITSET) {
    const uint32_t raw = 2u * t.aux[b].n;
    if (raw <= warp_words) return raw;
    const uint32_t z = zbits_words(t.aux[b].n, (uint32_t)(t.off[b + 1] - t.off[b]));
    return z <= warp_words ? z : raw;  // compressed in a warp, or raw across a block
  }
  if (l == EH_LAYOUT_UINTEGER) return (uint32_t)(t.off[b + 1] - t.off[b]);
  return 0xffffffffu;  // block bitsets are probed in global memory
}

// A block item keeps every warp of the block on one staged N(b); a b with
// little work would leave most of them idle, so only a b with at least this
// many probes becomes block items (about 32 batches of 32 rows at R-MAT's
// row lengths); the others stay warp items probing N(b) in global memory.
#ifndef EH_MIN_BLOCK_WORK
#define EH_MIN_BLOCK_WORK (1ull << 17)
#endif
constexpr uint64_t kMinBlockWork = EH_MIN_BLOCK_WORK;

struct PlanShape {
  uint32_t chunk;        // probes per warp item
  const float* pred;     // predicted cycles of each head entry's work (learned layouts), or null
  double unit;           // predicted cycles per warp item
  uint32_t warp_words;   // staging capacity of a warp (u32 words)
  uint32_t block_words;  // staging capacity of a block; 0: no block items
  uint32_t warps;        // warps per block
};

__global__ void plan_split_kernel(TrieView t, RevView r, PlanShape ps, uint32_t* __restrict__ nw,
                                  uint32_t* __restrict__ nb) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < t.n_head; b += gridDim.x * blockDim.x) {
    const uint64_t w = r.rev_wpre[r.rev_off[b + 1]] - r.rev_wpre[r.rev_off[b]];
    const uint32_t sw = staged_words(t, b, ps.warp_words);
    const bool blk = ps.block_words && sw > ps.warp_words && sw <= ps.block_words && w >= kMinBlockWork;
    const uint64_t mult = blk ? ps.warps : 1;
    uint64_t n = 0;
    if (w) {
      if (ps.pred) {
        n = (uint64_t)ceil((double)ps.pred[b] / (ps.unit * (double)mult));
        n = max((uint64_t)1, min(n, (w + 63) / 64));
      } else {
        n = (w + ps.chunk * mult - 1) / (ps.chunk * mult);
      }
    }
    nw[b] = blk ? 0u : (uint32_t)n;
    nb[b] = blk ? (uint32_t)n : 0u;
  }
}

struct Plan {
  DevBuf<Item> items;  // block items first, then warp items
  uint32_t n = 0;      // all items
  uint32_t nb = 0;     // block items
};

// returns the kernels it launched
static uint32_t build_plan(eh_context* ctx, const eh_trie* t, const PlanShape& shape, uint32_t g, Plan& plan) {
  cudaStream_t s = ctx->stream;
  plan.n = plan.nb = 0;
  if (!t->rev_entries) return 0;
  RevView r{t->rev_off.p, t->rev_lo.p, t->rev_hi.p, t->rev_src.p, t->rev_wpre.p, t->dir};
  PlanShape ps = shape;
  if (!(t->work_pred.p && t->pred_per_probe > 0)) ps.pred = nullptr;
  ps.unit = t->pred_per_probe * shape.chunk;
  DevBuf<uint32_t> nw(t->n_head, s), nb(t->n_head, s), pw(t->n_head, s), pb(t->n_head, s), tot(2, s);
  const int grid = num_sms() * 4;
  TracePhase ph_split("plan.split+scan", s);
  plan_split_kernel<<<grid, 256, 0, s>>>(t->view(), r, ps, nw.p, nb.p);
  EH_CHECK_LAUNCH();
  exclusive_scan<uint32_t>(nw.p, pw.p, t->n_head, tot.p, s);
  exclusive_scan<uint32_t>(nb.p, pb.p, t->n_head, tot.p + 1, s);
  uint32_t h[2] = {0, 0};
  EH_CUDA(cudaMemcpyAsync(h, tot.p, 8, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  ph_split.end();
  TracePhase ph_fill("plan.fill", s);
  plan.nb = h[1];
  plan.n = h[0] + h[1];
  plan.items.alloc(plan.n ? plan.n : 1, s);
  if (h[1]) {
    plan_fill_kernel<<<grid, 256, 0, s>>>(r, t->n_head, nb.p, pb.p, h[1], g, plan.items.p);
    EH_CHECK_LAUNCH();
  }
  if (h[0]) {
    plan_fill_kernel<<<grid, 256, 0, s>>>(r, t->n_head, nw.p, pw.p, h[0], g, plan.items.p + h[1]);
    EH_CHECK_LAUNCH();
  }
  return 1 + 2 * scan_launches(t->n_head) + (h[0] ? 1 : 0) + (h[1] ? 1 : 0);
}


// L2 eviction priority for the word rows' loads of N(a)'s bitset words: the
// sources of the word rows are the density rule's dense sets (75 MB of words
// at R-MAT-22, each read ~130 times in a query), so they are kept ahead of the
// streamed candidate values (createpolicy + ld.global.nc.L2::cache_hint).
__device__ __forceinline__ uint64_t l2_policy_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ ulonglong2 ld2_hint(const uint64_t* a, uint64_t pol) {
  ulonglong2 v;
  asm("ld.global.nc.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;" : "=l"(v.x), "=l"(v.y) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ uint64_t ld64_hint(const uint64_t* a, uint64_t pol) {
  uint64_t v;
  asm("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(a), "l"(pol));
  return v;
}
// ------------------------------------------------------------------ probes
// Probe structures for the staged set N(b), one per stored layout.
// P_ZBITS: a range bitset too large to stage word for word, staged
// compressed: per group of 32 words a presence mask (bit i: word 32k + i is
// non-zero) beside the count of non-zero words before the group, read
// together in one 8-byte load, and then only the non-zero words.  A probe
// whose word is empty costs one shared load; the others two.
enum { P_SBITS = 0, P_GBITS = 1, P_SLIST = 2, P_GLIST = 3, P_GBLOCK = 4, P_ZBITS = 5 };

struct Staged {
  const uint64_t* words;  // P_SBITS (shared) / P_GBITS (global); P_ZBITS: the non-zero words (shared)
  const uint32_t* list;   // P_SLIST (shared) / P_GLIST (global)
  const uint32_t* ids;    // P_GBLOCK
  const uint64_t* bwords; // P_GBLOCK
  const uint2* pz;        // P_ZBITS: group k: x = presence mask of words 32k.., y = non-zero words before 32k
  uint32_t start;         // first word index (bitsets)
  uint32_t n;             // words / list length / blocks
};


// branch-free lower bound over a sorted run of n >= 1 values
template <bool kShared>
__device__ __forceinline__ bool list_contains(const uint32_t* p, uint32_t n, uint32_t w) {
  uint32_t base = 0;
  while (n > 1) {
    const uint32_t half = n >> 1;
    const uint32_t v = kShared ? p[base + half] : __ldg(p + base + half);
    base = (v <= w) ? base + half : base;
    n -= half;
  }
  return (kShared ? p[base] : __ldg(p + base)) == w;
}

template <int P>
__device__ __forceinline__ uint32_t probe(const Staged& s, uint32_t w) {
  if (P == P_ZBITS) {
    const uint32_t idx = (w >> 6) - s.start;
    if (idx >= s.n) return 0;  // also catches w below the first word (wraps)
    const uint2 g = s.pz[idx >> 5];
    if (!((g.x >> (idx & 31)) & 1u)) return 0;
    const uint32_t below = g.x & ((1u << (idx & 31)) - 1u);
    return (uint32_t)(s.words[g.y + __popc(below)] >> (w & 63)) & 1u;
  }
  if (P == P_SBITS || P == P_GBITS) {
    const uint32_t idx = (w >> 6) - s.start;
    if (idx >= s.n) return 0;  // also catches w below the first word (wraps)
    const uint64_t word = (P == P_SBITS) ? s.words[idx] : __ldg(s.words + idx);
    return (uint32_t)(word >> (w & 63)) & 1u;
  } else if (P == P_SLIST || P == P_GLIST) {
    return list_contains<P == P_SLIST>(s.list, s.n, w) ? 1u : 0u;
  } else {  // block bitset: find block id w >> 8, test its word
    const uint32_t id = w >> 8;
    uint32_t lo = 0, hi = s.n;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(s.ids + mid) < id) lo = mid + 1; else hi = mid;
    }
    if (lo >= s.n || __ldg(s.ids + lo) != id) return 0;
    return (uint32_t)(__ldg(s.bwords + 4 * (uint64_t)lo + ((w >> 6) & 3)) >> (w & 63)) & 1u;
  }
}

// What a hit does besides counting: kMode 0 counts only; 1 adds it to the
// annotation of the row's source (and, on a symmetric relation, of the
// matched element) -- the annotated bag of TrieBuilder::set_annotation;
// 2 writes the tuple (a, b, c) to the item's slice of the output columns
// -- the materialized Triangle(a,b,c) of TrieBuilder::build_set.
enum { MODE_COUNT = 0, MODE_ANNOT = 1, MODE_MAT = 2 };

constexpr int kHot = 4;  // MODE_ANNOT: head entries with block-local counters
struct Int4 {
  int32_t v[kHot];
};

struct Sink {
  unsigned long long* annot;  // MODE_ANNOT
  uint32_t* ma;               // MODE_MAT: output columns
  uint32_t* mb;
  uint32_t* mc;
  uint64_t base;              // MODE_MAT: first row of this item's slice
  unsigned int* slot;         // MODE_MAT: the warp's running row count (shared)
  uint32_t b;                 // MODE_MAT: value of the staged head entry b
  const int32_t* hot;         // MODE_ANNOT: the kHot largest sets' head entries (-1: none)
  unsigned long long* hot_acc;  // MODE_ANNOT: their block-local counts (shared)
  // MODE_ANNOT on a symmetric relation: every matched element is in the
  // staged N(b); when it is staged with room to spare, each element has a
  // shared counter (wcnt, by position in N(b)) flushed once per item
  uint32_t* wcnt;             // null: matched elements go to the annotation directly
  int wmode;                  // P_SLIST (position by search) or P_SBITS (position by rank)
  const uint32_t* wlist;      // P_SLIST: the staged list, wn elements
  const uint64_t* wwords;     // P_SBITS: the staged words, wn of them from word wstart
  const uint32_t* wrank;      // P_SBITS: elements before each staged word
  uint32_t wstart, wn;
};

// owner lane of flattened pair q: the number of lanes whose inclusive
// prefix is <= q (q < total guarantees a result below 32)
__device__ __forceinline__ uint32_t owner_lane(uint32_t incl, uint32_t q) {
  uint32_t j = 0;
#pragma unroll
  for (int step = 16; step; step >>= 1) {
    const uint32_t tj = __shfl_sync(kFull, incl, j + step - 1);
    if (tj <= q) j += step;
  }
  return j;
}

// kSrcAgg: the caller adds the row source's share of the annotation for a
// run of hits at once (add_src), so a hit adds only the matched element's
// share; a hub source in many rows would otherwise take one atomic per hit.
template <int kMode, bool kSrcAgg = false>
__device__ __forceinline__ void on_hit(const TrieView& t, const RevView& r, const Sink& sk, uint32_t src,
                                       uint32_t w) {
  if (kMode == MODE_ANNOT) {
    if (r.dir == DIR_SYM) {
      if (!kSrcAgg) atomicAdd(sk.annot + src, 2ull);
      if (sk.wcnt) {  // the matched element's position in the staged N(b)
        uint32_t pos;
        if (sk.wmode == P_SLIST) {
          uint32_t lo = 0, hi = sk.wn;
          while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sk.wlist[mid] < w) lo = mid + 1; else hi = mid;
          }
          pos = lo;
        } else {
          const uint32_t idx = (w >> 6) - sk.wstart;
          pos = sk.wrank[idx] + (uint32_t)__popcll(sk.wwords[idx] & ((1ull << (w & 63)) - 1));
        }
        atomicAdd(sk.wcnt + pos, 1u);
        return;
      }
      // the matched element: a hub is the third vertex of a large share of
      // all triangles, so the largest sets count in shared memory first
      const int32_t hx = __ldg(t.head_index + w);
      int k = 0;
#pragma unroll
      for (; k < kHot; k++)
        if (hx == sk.hot[k]) break;
      if (k < kHot) atomicAdd(sk.hot_acc + k, 2ull);
      else atomicAdd(sk.annot + hx, 2ull);
    } else if (!kSrcAgg) {
      atomicAdd(sk.annot + src, 1ull);
    }
  } else if (kMode == MODE_MAT) {
    const uint32_t a = __ldg(t.head + src), b = sk.b;
    if (r.dir == DIR_SYM) {
      // one undirected triangle a < b < w stands for all 3! orderings
      const uint64_t o = sk.base + atomicAdd(sk.slot, 6u);
      const uint32_t p[6][3] = {{a, b, w}, {a, w, b}, {b, a, w}, {b, w, a}, {w, a, b}, {w, b, a}};
#pragma unroll
      for (int k = 0; k < 6; k++) {
        sk.ma[o + k] = p[k][0];
        sk.mb[o + k] = p[k][1];
        sk.mc[o + k] = p[k][2];
      }
    } else {
      const uint64_t o = sk.base + atomicAdd(sk.slot, 1u);
      sk.ma[o] = a;
      sk.mb[o] = b;
      sk.mc[o] = w;
    }
  }
}

template <int kMode>
__device__ __forceinline__ void add_src(const RevView& r, const Sink& sk, uint32_t src, uint64_t hits) {
  if (kMode == MODE_ANNOT && hits) atomicAdd(sk.annot + src, (r.dir == DIR_SYM ? 2ull : 1ull) * hits);
}

// Rows whose source set N(a) is also a range bitset, against a bitset N(b),
// are intersected word by word (64-bit AND + popcount over the overlap of
// the candidate value range [v0, v1] with both word ranges) whenever the
// words, weighted by kWordRowNum / kWordRowDen (a word against a candidate
// probe), are fewer than the row's candidate elements; the reference's
// bitset ∩ bitset path (ops/intersection/bitset.hpp:526-567, 619-661).
// Word rows run warp-cooperatively one row at a time (coalesced 8-byte
// loads of N(a)'s words); the other rows are flattened (row, element)
// pairs over the lanes, two pairs per lane per trip for memory-level
// parallelism.
template <int P, int kMode>
__device__ __forceinline__ uint64_t stream_rows(const Staged& st, const TrieView& t, const RevView& r, uint32_t kb,
                                                uint32_t ke, uint32_t long_row, const Sink& sk) {
  constexpr bool kBits = (P == P_SBITS || P == P_GBITS);
  const uint32_t lane = lane_id();
  uint64_t cnt = 0;
  const uint64_t pol_keep = l2_policy_last();
  for (uint32_t k0 = kb; k0 < ke; k0 += 32) {
    const uint32_t k = k0 + lane;
    uint32_t lo = 0, len = 0, src = 0;
    if (k < ke) {
      lo = __ldg(r.rev_lo + k);
      len = __ldg(r.rev_hi + k) - lo;
      if (kMode != MODE_COUNT || kBits) src = __ldg(r.rev_src + k);
    }
    // ---- word rows
    if (kBits) {
      bool word_row = false;
      uint32_t v0 = 0, v1 = 0, wlo = 0, whi = 0;
      uint64_t abase = 0;
      if (len && __ldg(t.layout + src) == EH_LAYOUT_RANGE_BITSET) {
        v0 = __ldg(t.vals + lo);
        v1 = __ldg(t.vals + lo + len - 1);
        const SetAux aa = t.aux[src];
        const uint32_t lo_w = max(max(v0 >> 6, aa.start), st.start);
        const uint32_t hi_w = min(min(v1 >> 6, aa.start + aa.n - 1), st.start + st.n - 1);
        const uint32_t words = hi_w >= lo_w ? hi_w - lo_w + 1 : 0;
        if (words * kWordRowNum < len * kWordRowDen) {
          word_row = true;
          wlo = lo_w;
          whi = hi_w;
          abase = aa.off - aa.start;  // word w of N(a) is bs_words[abase + w]
        }
      }
      uint32_t nw = (word_row && whi >= wlo) ? whi - wlo + 1 : 0u;
      if (word_row) len = 0;  // handled here, not in the element loop
      // long word rows (at least a warp's width of words): one row at a time
      // across the warp, each lane ANDing the word pairs 2 lane, 2 lane + 64,
      // ... read from N(a) with one aligned 16-byte load (the reference's
      // 128-bit AND), no owner search
      {
        const bool is_long = nw >= (uint32_t)kLongWords;
        uint32_t rows = __ballot_sync(kFull, is_long);
        if (is_long) nw = 0;
        while (rows) {
          const int j = __ffs(rows) - 1;
          rows &= rows - 1;
          const uint32_t lo_w = __shfl_sync(kFull, wlo, j), hi_w = __shfl_sync(kFull, whi, j);
          const uint32_t b0 = __shfl_sync(kFull, v0, j), b1 = __shfl_sync(kFull, v1, j);
          const uint64_t base = __shfl_sync(kFull, abase, j);
          const uint32_t sj = (kMode != MODE_COUNT) ? __shfl_sync(kFull, src, j) : 0u;
          const uint32_t w_first = b0 >> 6, w_last = b1 >> 6;
          uint32_t row_hits = 0;
          // The row's words lo_w..hi_w are read in pairs from an even pool
          // index, 16-byte aligned (allocations are at least 16-byte
          // aligned): pair q holds the row's words q - par and q + 1 - par,
          // where par = 1 when the row starts at an odd pool index (its first
          // pair then begins with the word before lo_w: in the pool, since
          // that index is >= 1, and masked).  Offsets stay non-negative; a
          // word index is formed only for words inside the row.  A pair is
          // read whole only when both its words are in the row's range or the
          // first one is the word before it, so no read passes N(a)'s last word.
          const uint32_t par = (uint32_t)((base + lo_w) & 1ull);
          const uint32_t end = hi_w - lo_w + 1 + par;         // pair offsets run below end
          const uint64_t g0 = base + lo_w - par;              // even pool index of offset 0
          const uint32_t wa = lo_w - par;                     // word of offset 0 (mod 2^32)
          const uint32_t sa = wa - st.start;                  // its staged index (mod 2^32)
          for (uint32_t q0 = 2 * lane; q0 < end; q0 += 64 * kLongWordUnroll) {
            uint64_t x[2 * kLongWordUnroll], y[2 * kLongWordUnroll];
#pragma unroll
            for (int u = 0; u < kLongWordUnroll; u++) {
              const uint32_t q = q0 + 64 * u;
              if (q + 2 <= end) {
                const ulonglong2 v = ld2_hint(t.bs_words + g0 + q, pol_keep);
                x[2 * u] = v.x;
                x[2 * u + 1] = v.y;
              } else {
                x[2 * u] = q < end ? ld64_hint(t.bs_words + g0 + q, pol_keep) : 0ull;
                x[2 * u + 1] = 0ull;
              }
#pragma unroll
              for (int h = 0; h < 2; h++) {
                const uint32_t qh = q + h;
                const bool in = qh >= par && qh < end;  // a word of the row
                y[2 * u + h] = in ? ((P == P_SBITS) ? st.words[sa + qh] : __ldg(st.words + (sa + qh))) : 0ull;
              }
            }
#pragma unroll
            for (int u = 0; u < 2 * kLongWordUnroll; u++) {
              const uint32_t w = wa + (q0 + 64 * (u >> 1) + (u & 1));  // meaningful where y is non-zero
              if (w == w_first) y[u] &= ~0ull << (b0 & 63);
              if (w == w_last) y[u] &= ~0ull >> (63 - (b1 & 63));
              x[u] &= y[u];
              row_hits += __popcll(x[u]);
            }
            if (kMode == MODE_MAT || (kMode == MODE_ANNOT && r.dir == DIR_SYM)) {
#pragma unroll
              for (int u = 0; u < 2 * kLongWordUnroll; u++) {
                uint64_t z = x[u];  // non-zero only for words inside the row
                const uint32_t w = wa + (q0 + 64 * (u >> 1) + (u & 1));
                while (z) {
                  const uint32_t bit = __ffsll((long long)z) - 1;
                  on_hit<kMode, true>(t, r, sk, sj, (w << 6) | bit);
                  z &= z - 1;
                }
              }
            }
          }
          cnt += row_hits;
          if (kMode == MODE_ANNOT) {  // the row's source once per row
            const uint32_t rh = warp_sum(row_hits);
            if (lane == 0) add_src<kMode>(r, sk, sj, rh);
          }
        }
      }
      // the other word rows of this batch, flattened into (row, word) pairs
      // over the lanes like the short element rows below: one trip covers
      // the words of many rows
      const uint32_t wincl = warp_incl_scan(nw);
      const uint32_t wtotal = __shfl_sync(kFull, wincl, 31);
      const uint32_t wexcl = wincl - nw;
      for (uint32_t p = 0; p < wtotal; p += 32 * kWordUnroll) {
        uint64_t x[kWordUnroll];
        uint32_t wv[kWordUnroll], sj[kWordUnroll];
#pragma unroll
        for (int u = 0; u < kWordUnroll; u++) {
          const uint32_t q = p + 32 * u + lane;
          const uint32_t j = owner_lane(wincl, q);
          const uint32_t lo_w = __shfl_sync(kFull, wlo, j), ex = __shfl_sync(kFull, wexcl, j);
          const uint32_t b0 = __shfl_sync(kFull, v0, j), b1 = __shfl_sync(kFull, v1, j);
          const uint64_t base = __shfl_sync(kFull, abase, j);
          sj[u] = (kMode != MODE_COUNT) ? __shfl_sync(kFull, src, j) : 0u;
          x[u] = 0;
          wv[u] = 0;
          if (q < wtotal) {
            const uint32_t w = lo_w + (q - ex);
            uint64_t m = ~0ull;
            if (w == (b0 >> 6)) m &= ~0ull << (b0 & 63);
            if (w == (b1 >> 6)) m &= ~0ull >> (63 - (b1 & 63));
            const uint64_t bw = (P == P_SBITS) ? st.words[w - st.start] : __ldg(st.words + (w - st.start));
            x[u] = ld64_hint(t.bs_words + base + w, pol_keep) & bw & m;
            wv[u] = w;
          }
        }
#pragma unroll
        for (int u = 0; u < kWordUnroll; u++) {
          const uint32_t hits = __popcll(x[u]);
          cnt += hits;
          if (kMode == MODE_ANNOT) add_src<kMode>(r, sk, sj[u], hits);
          if (kMode == MODE_MAT || (kMode == MODE_ANNOT && r.dir == DIR_SYM)) {
            uint64_t y = x[u];
            while (y) {
              const uint32_t bit = __ffsll((long long)y) - 1;
              on_hit<kMode, true>(t, r, sk, sj[u], (wv[u] << 6) | bit);
              y &= y - 1;
            }
          }
        }
      }
    }
    // ---- long element rows: two rows at a time across the warp, each lane
    // loading kLongUnroll coalesced elements of both before it probes any,
    // no owner search
    {
      const bool is_long = len >= long_row;
      uint32_t rows = __ballot_sync(kFull, is_long);
      const uint32_t rlen = len;
      if (is_long) len = 0;
      while (rows) {
        const int j = __ffs(rows) - 1;
        rows &= rows - 1;
        int j2 = j;
        bool two = false;
        if (rows) {
          j2 = __ffs(rows) - 1;
          rows &= rows - 1;
          two = true;
        }
        const uint32_t rlo = __shfl_sync(kFull, lo, j), rn = __shfl_sync(kFull, rlen, j);
        const uint32_t rlo2 = __shfl_sync(kFull, lo, j2);
        const uint32_t rn2 = two ? __shfl_sync(kFull, rlen, j2) : 0u;
        uint32_t src_j = 0, src_j2 = 0;
        if (kMode != MODE_COUNT) {
          src_j = __shfl_sync(kFull, src, j);
          src_j2 = __shfl_sync(kFull, src, j2);
        }
        const uint32_t* row = t.vals + rlo;
        const uint32_t* row2 = t.vals + rlo2;
        uint32_t row_hits = 0, row_hits2 = 0;
        const uint32_t rmax = rn > rn2 ? rn : rn2;
        for (uint32_t i = lane; i < rmax; i += 32 * kLongUnroll) {
          uint32_t w[kLongUnroll], w2[kLongUnroll];
#pragma unroll
          for (int u = 0; u < kLongUnroll; u++) {
            w[u] = (i + 32 * u < rn) ? __ldg(row + i + 32 * u) : 0u;
            w2[u] = (i + 32 * u < rn2) ? __ldg(row2 + i + 32 * u) : 0u;
          }
#pragma unroll
          for (int u = 0; u < kLongUnroll; u++) {
            if (i + 32 * u < rn) {
              const uint32_t h = probe<P>(st, w[u]);
              row_hits += h;
              if (kMode != MODE_COUNT && h) on_hit<kMode, true>(t, r, sk, src_j, w[u]);
            }
            if (i + 32 * u < rn2) {
              const uint32_t h = probe<P>(st, w2[u]);
              row_hits2 += h;
              if (kMode != MODE_COUNT && h) on_hit<kMode, true>(t, r, sk, src_j2, w2[u]);
            }
          }
        }
        cnt += row_hits + row_hits2;
        if (kMode == MODE_ANNOT) {  // each row's source once per row
          const uint32_t rh = warp_sum(row_hits);
          const uint32_t rh2 = warp_sum(row_hits2);
          if (lane == 0) {
            add_src<kMode>(r, sk, src_j, rh);
            if (two) add_src<kMode>(r, sk, src_j2, rh2);
          }
        }
      }
    }
    // ---- short element rows, flattened
    const uint32_t incl = warp_incl_scan(len);
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t excl = incl - len;
    for (uint32_t p = 0; p < total; p += 32 * kShortUnroll) {
      uint32_t w[kShortUnroll], sj[kShortUnroll];
#pragma unroll
      for (int u = 0; u < kShortUnroll; u++) {
        const uint32_t q = p + 32 * u + lane;
        const uint32_t j = owner_lane(incl, q);
        const uint32_t loj = __shfl_sync(kFull, lo, j), exj = __shfl_sync(kFull, excl, j);
        sj[u] = (kMode != MODE_COUNT) ? __shfl_sync(kFull, src, j) : 0u;
        w[u] = q < total ? __ldg(t.vals + loj + (q - exj)) : 0u;
      }
#pragma unroll
      for (int u = 0; u < kShortUnroll; u++) {
        const uint32_t q = p + 32 * u + lane;
        const uint32_t h = q < total ? probe<P>(st, w[u]) : 0u;
        cnt += h;
        if (kMode == MODE_ANNOT) {
          // lanes of one row are adjacent: one source atomic per row present
          const uint32_t grp = __match_any_sync(kFull, sj[u]);
          const uint32_t hm = __ballot_sync(kFull, h) & grp;
          if (lane == (uint32_t)(__ffs(grp) - 1)) add_src<kMode>(r, sk, sj[u], __popc(hm));
        }
        if (kMode != MODE_COUNT && h) on_hit<kMode, true>(t, r, sk, sj[u], w[u]);
      }
    }
  }
  return cnt;
}

// Stage N(b) in the warp's shared region according to its layout; returns
// the probe mode.
__device__ __forceinline__ int stage_set(const TrieView& t, uint32_t hb, uint32_t* sm, int cap_words, Staged& st,
                                         bool zlist = false) {
  const uint32_t lane = lane_id();
  const uint8_t layout = t.layout[hb];
  const SetAux a = t.aux[hb];
  const uint64_t s0 = t.off[hb];
  const uint32_t len = (uint32_t)(t.off[hb + 1] - s0);
  if (layout == EH_LAYOUT_RANGE_BITSET) {
    st.start = a.start;
    st.n = a.n;
    if (2 * a.n <= (uint32_t)cap_words) {
      uint64_t* sw = reinterpret_cast<uint64_t*>(sm);
      for (uint32_t j = lane; j < a.n; j += 32) sw[j] = __ldg(t.bs_words + a.off + j);
      __syncwarp();
      st.words = sw;
      return P_SBITS;
    }
    if (zbits_words(a.n, len) <= (uint32_t)cap_words) {
      // compressed: 32 words per step, 4 steps of loads in flight
      const uint32_t groups = (a.n + 31) / 32;
      uint2* pz = reinterpret_cast<uint2*>(sm);
      uint64_t* zw = reinterpret_cast<uint64_t*>(sm + 2 * groups);
      const uint64_t* src = t.bs_words + a.off;
      uint32_t run = 0;
      for (uint32_t g0 = 0; g0 < groups; g0 += 4) {
        uint64_t x[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const uint32_t j = (g0 + u) * 32 + lane;
          x[u] = j < a.n ? __ldg(src + j) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          if (g0 + u < groups) {
            const uint32_t bal = __ballot_sync(kFull, x[u] != 0ull);
            if (x[u]) zw[run + __popc(bal & lanemask_lt())] = x[u];
            if (lane == 0) pz[g0 + u] = make_uint2(bal, run);
            run += __popc(bal);
          }
        }
      }
      __syncwarp();
      st.pz = pz;
      st.words = zw;
      return P_ZBITS;
    }
    st.words = t.bs_words + a.off;
    return P_GBITS;
  }
  if (layout == EH_LAYOUT_BLOCK_BITSET) {
    st.ids = t.bb_id + a.off;
    st.bwords = t.bb_words + 4 * a.off;
    st.n = a.n;
    return P_GBLOCK;
  }
  st.n = len;
  // A uint list staged in the triangle COUNT kernel becomes a compressed bitmap
  // (the P_ZBITS form, built from the sorted elements: presence bits by
  // shared atomics, ranks by a warp scan, each element's bit OR-ed into its
  // non-zero word) when that fits: two shared loads per probe in place of a
  // ~8-step binary search (R-MAT-22, density rule: 49.8 -> 28.7 warp-cycles
  // per probe including the build, kernel 9.91 -> 8.19 ms).  The annotated
  // pass keeps the list: its per-element counters are indexed by position in it.
  if (zlist && len >= 2) {
    const uint32_t first = __ldg(t.vals + s0), last = __ldg(t.vals + s0 + len - 1);
    const uint32_t W = (last >> 6) - (first >> 6) + 1;
    if (zbits_words(W, len) <= (uint32_t)cap_words) {
      const uint32_t groups = (W + 31) / 32, start = first >> 6;
      uint2* pz = reinterpret_cast<uint2*>(sm);
      uint64_t* zw = reinterpret_cast<uint64_t*>(sm + 2 * groups);
      for (uint32_t g = lane; g < groups; g += 32) pz[g] = make_uint2(0u, 0u);
      __syncwarp();
      for (uint32_t j = lane; j < len; j += 32) {  // presence of each element's word
        const uint32_t k = (__ldg(t.vals + s0 + j) >> 6) - start;
        atomicOr(&pz[k >> 5].x, 1u << (k & 31));
      }
      __syncwarp();
      uint32_t run = 0;  // non-zero words before each group: a scan over the groups
      for (uint32_t g0 = 0; g0 < groups; g0 += 32) {
        const uint32_t g = g0 + lane;
        const uint32_t c = g < groups ? __popc(pz[g].x) : 0u;
        const uint32_t incl = warp_incl_scan(c);
        if (g < groups) pz[g].y = run + incl - c;
        run += __shfl_sync(kFull, incl, 31);
      }
      for (uint32_t j = lane; j < run; j += 32) zw[j] = 0ull;
      __syncwarp();
      for (uint32_t j = lane; j < len; j += 32) {  // each element's bit in its word
        const uint32_t v = __ldg(t.vals + s0 + j);
        const uint32_t k = (v >> 6) - start;
        const uint2 g = pz[k >> 5];
        atomicOr(reinterpret_cast<unsigned long long*>(zw + g.y + __popc(g.x & ((1u << (k & 31)) - 1u))),
                 1ull << (v & 63));
      }
      __syncwarp();
      st.pz = pz;
      st.words = zw;
      st.start = start;
      st.n = W;
      return P_ZBITS;
    }
  }
  if (len <= (uint32_t)cap_words) {
    for (uint32_t j = lane; j < len; j += 32) sm[j] = __ldg(t.vals + s0 + j);
    __syncwarp();
    st.list = sm;
    return P_SLIST;
  }
  st.list = t.vals + s0;
  return P_GLIST;
}

// stage_set for a block item: every thread of the block copies, into the
// block's whole shared region (the caller synchronises the block after).
__device__ __forceinline__ int stage_set_block(const TrieView& t, uint32_t hb, uint32_t* sm, int cap_words,
                                               Staged& st) {
  const uint8_t layout = t.layout[hb];
  const SetAux a = t.aux[hb];
  const uint64_t s0 = t.off[hb];
  const uint32_t len = (uint32_t)(t.off[hb + 1] - s0);
  if (layout == EH_LAYOUT_RANGE_BITSET) {
    st.start = a.start;
    st.n = a.n;
    if (2 * a.n <= (uint32_t)cap_words) {
      uint64_t* sw = reinterpret_cast<uint64_t*>(sm);
      for (uint32_t j = threadIdx.x; j < a.n; j += blockDim.x) sw[j] = __ldg(t.bs_words + a.off + j);
      st.words = sw;
      return P_SBITS;
    }
    st.words = t.bs_words + a.off;
    return P_GBITS;
  }
  if (layout == EH_LAYOUT_BLOCK_BITSET) {
    st.ids = t.bb_id + a.off;
    st.bwords = t.bb_words + 4 * a.off;
    st.n = a.n;
    return P_GBLOCK;
  }
  st.n = len;
  if (len <= (uint32_t)cap_words) {
    for (uint32_t j = threadIdx.x; j < len; j += blockDim.x) sm[j] = __ldg(t.vals + s0 + j);
    st.list = sm;
    return P_SLIST;
  }
  st.list = t.vals + s0;
  return P_GLIST;
}

template <int kMode>
__device__ __forceinline__ uint64_t rows_of(int mode, const Staged& st, const TrieView& t, const RevView& r,
                                            uint32_t kb, uint32_t ke, uint32_t long_row, const Sink& sk) {
  switch (mode) {
    case P_SBITS: return stream_rows<P_SBITS, kMode>(st, t, r, kb, ke, long_row, sk);
    case P_GBITS: return stream_rows<P_GBITS, kMode>(st, t, r, kb, ke, long_row, sk);
    case P_SLIST: return stream_rows<P_SLIST, kMode>(st, t, r, kb, ke, long_row, sk);
    case P_GLIST: return stream_rows<P_GLIST, kMode>(st, t, r, kb, ke, long_row, sk);
    case P_ZBITS: return stream_rows<P_ZBITS, kMode>(st, t, r, kb, ke, long_row, sk);
    default: return stream_rows<P_GBLOCK, kMode>(st, t, r, kb, ke, long_row, sk);
  }
}

struct QueryOut {
  uint32_t shard_index, shard_count;  // this launch runs items shard_index + q * shard_count
  uint32_t long_row;                  // size-class boundary of rows (warp-wide vs flattened)
  unsigned long long* total;   // per graph results (one per trie)
  unsigned long long* annot;   // per head entry annotation or null
  float* records;              // per item timing records or null
  unsigned int* queue;         // atomic queue head
  unsigned long long* item_counts;  // per item count x count_mult (materialize sizing) or null
  uint32_t count_mult;
  const unsigned long long* item_off;  // MODE_MAT: first output row of each item
  uint32_t *ma, *mb, *mc;      // MODE_MAT: output columns
  const uint32_t* sel;         // 4-clique: bit per node value of a selected partner set, or null
  int32_t hot[kHot];           // MODE_ANNOT on a symmetric relation: largest sets' head entries, -1 if none
  uint32_t* gsbuf;             // 4-clique: per-warp S buffers in global memory (sets too large for
  uint32_t gcap;               //   shared memory), gcap words each; null: S in shared memory
  uint32_t n_bitems;           // MODE_COUNT: items[0, n_bitems) are block items, the rest warp items
  unsigned int* bqueue;        // atomic queue head of the block items
};

template <int kMode>
__global__ void EH_TRI_LAUNCH_BOUNDS triangle_kernel(const TrieView* __restrict__ views,
                                                        const RevView* __restrict__ revs,
                                                        const Item* __restrict__ items, uint32_t n_items,
                                                        int cap_words, QueryOut out) {
  extern __shared__ uint32_t smem[];
  __shared__ unsigned int slot[kMaxWarps];  // MODE_MAT: rows written by the warp's item so far
  __shared__ unsigned long long hot_acc[kHot];
  __shared__ int32_t hot[kHot];
  if (kMode == MODE_ANNOT) {
    if (threadIdx.x < kHot) {
      hot_acc[threadIdx.x] = 0;
      hot[threadIdx.x] = out.hot[threadIdx.x];
    }
    __syncthreads();
  }
  const uint32_t lane = lane_id();
  const uint32_t wid = threadIdx.x >> 5;
  uint32_t* sm = smem + (size_t)wid * cap_words;
  unsigned long long acc = 0;
  uint32_t cur_g = 0xffffffffu;
  // Block items first (MODE_COUNT only): the block pulls an item, stages its
  // N(b) across the whole shared region, and its warps take the rows 32 at a
  // time from a block counter.  Then each warp pulls warp items on its own.
  __shared__ unsigned int s_q, s_next;
  const uint32_t nwarps = blockDim.x >> 5;
  bool block_phase = kMode == MODE_COUNT && out.n_bitems > 0;
  const uint32_t n_witems = n_items - (kMode == MODE_COUNT ? out.n_bitems : 0u);
  for (;;) {
    uint32_t it;
    if (block_phase) {
      if (threadIdx.x == 0) {
        s_q = atomicAdd(out.bqueue, 1u);
        s_next = 0;
      }
      __syncthreads();
      const uint64_t bi64 = (uint64_t)out.shard_index + (uint64_t)s_q * out.shard_count;
      if (bi64 >= out.n_bitems) {  // the same on every thread of the block
        block_phase = false;
        continue;
      }
      it = (uint32_t)bi64;
    } else {
      uint32_t q = 0;
      if (lane == 0) q = atomicAdd(out.queue, 1u);
      q = __shfl_sync(kFull, q, 0);
      const uint64_t it64 = (uint64_t)out.shard_index + (uint64_t)q * out.shard_count;
      if (it64 >= n_witems) break;
      it = (uint32_t)it64 + (kMode == MODE_COUNT ? out.n_bitems : 0u);
    }
    const Item item = items[it];
    if (item.g != cur_g) {  // flush the running count of the previous graph
      if (lane == 0 && cur_g != 0xffffffffu && acc) atomicAdd(out.total + cur_g, acc);
      acc = 0;
      cur_g = item.g;
    }
    const TrieView t = views[item.g];
    const RevView r = revs[item.g];
    long long t0 = 0;
    if (out.records && lane == 0) t0 = clock64();
    Sink sk{out.annot, out.ma, out.mb, out.mc, 0, &slot[wid], 0, hot, hot_acc, nullptr, 0, nullptr, nullptr,
            nullptr, 0, 0};
    if (kMode == MODE_MAT) {
      if (lane == 0) slot[wid] = 0;
      __syncwarp();
      sk.base = out.item_off[it];
      sk.b = t.head[item.hb];
    }
    Staged st;
    int mode;
    if (block_phase) {
      mode = stage_set_block(t, item.hb, smem, cap_words * (int)nwarps, st);
      __syncthreads();
    } else {
      mode = stage_set(t, item.hb, sm, cap_words, st, kMode == MODE_COUNT);
    }
    const uint64_t b0 = t.off[item.hb];
    const uint32_t blen = (uint32_t)(t.off[item.hb + 1] - b0);
    if (kMode == MODE_ANNOT && r.dir == DIR_SYM && (mode == P_SLIST || mode == P_SBITS)) {
      // per-element counters after the staged structure, if they fit
      const uint32_t used = mode == P_SLIST ? st.n : 3 * st.n;  // list, or words (2 per) + ranks
      if (used + blen <= (uint32_t)cap_words) {
        sk.wmode = mode;
        sk.wn = st.n;
        sk.wlist = st.list;
        sk.wwords = st.words;
        sk.wstart = st.start;
        if (mode == P_SBITS) {
          uint32_t* rk = sm + 2 * st.n;
          const uint32_t* grk = t.bs_rank + t.aux[item.hb].off;
          for (uint32_t j = lane; j < st.n; j += 32) rk[j] = __ldg(grk + j);
          sk.wrank = rk;
        }
        sk.wcnt = sm + used;
        for (uint32_t j = lane; j < blen; j += 32) sk.wcnt[j] = 0;
        __syncwarp();
      }
    }
    uint64_t c = 0;
    if (block_phase) {
      for (;;) {
        uint32_t batch = 0;
        if (lane == 0) batch = atomicAdd(&s_next, 1u);
        batch = __shfl_sync(kFull, batch, 0);
        const uint64_t k0 = (uint64_t)item.kb + 32ull * batch;
        if (k0 >= item.ke) break;
        const uint32_t k1 = k0 + 32 < (uint64_t)item.ke ? (uint32_t)(k0 + 32) : item.ke;
        c += rows_of<kMode>(mode, st, t, r, (uint32_t)k0, k1, out.long_row, sk);
      }
    } else {
      c = rows_of<kMode>(mode, st, t, r, item.kb, item.ke, out.long_row, sk);
    }
    c = warp_sum(c);
    if (kMode == MODE_ANNOT && sk.wcnt) {  // flush the item's per-element counts
      __syncwarp();
      for (uint32_t j = lane; j < blen; j += 32) {
        const uint32_t n = sk.wcnt[j];
        if (n) atomicAdd(out.annot + __ldg(t.head_index + __ldg(t.vals + b0 + j)), 2ull * n);
      }
    }
    if (kMode == MODE_ANNOT && r.dir == DIR_SYM && lane == 0 && c) atomicAdd(out.annot + item.hb, 2ull * c);
    if (out.item_counts && lane == 0) out.item_counts[it] = c * out.count_mult;
    acc += c;
    if (block_phase) __syncthreads();  // every warp is done with the staged set
    else __syncwarp();                 // the staged region is reused by the next item
    if (out.records && (block_phase ? threadIdx.x == 0 : lane == 0)) {
      const long long t1 = clock64();
      const uint32_t len = blen;
      const uint64_t pairs = r.rev_wpre[item.ke] - r.rev_wpre[item.kb];
      const uint32_t first = t.vals[b0], last = t.vals[b0 + len - 1];
      float* rec = out.records + 8 * (size_t)it;
      rec[0] = (float)len;
      rec[1] = (float)pairs;
      rec[2] = (float)len / (float)(last - first + 1);
      rec[3] = (float)(last - first);
      rec[4] = (float)t.layout[item.hb];
      rec[5] = (float)mode;
      rec[6] = __uint_as_float(item.hb);  // set id, bit pattern
      rec[7] = (float)(t1 - t0) * (block_phase ? (float)nwarps : 1.f);  // warp-cycles
    }
  }
  if (lane == 0 && cur_g != 0xffffffffu && acc) atomicAdd(out.total + cur_g, acc);
  if (kMode == MODE_ANNOT) {  // every warp leaves the loop above; then flush the block's hot counts
    __syncthreads();
    if (threadIdx.x < kHot && hot[threadIdx.x] >= 0 && hot_acc[threadIdx.x])
      atomicAdd(out.annot + hot[threadIdx.x], hot_acc[threadIdx.x]);
  }
}

// ------------------------------------------------------------ 4-clique
// For every row a->b: S = candidates(a,b) ∩ N(b) is materialised in the
// warp's shared region, then for each c in S the elements d of S are probed
// in N(c).  On an up- or down-oriented relation (or a symmetric one, rows
// a<b) only the d on the far side of c can close a 4-clique; on a general
// relation (self-loops, rows in both directions that are not symmetric) the
// candidates are the whole N(a) and every d of S is probed: the count is the
// number of assignments (a,b,c,d) with all six rows present, which is what
// the reference's N-way loop nest counts (TrieBuilder.cpp:276-348).
__device__ __forceinline__ uint32_t probe_global_set(const TrieView& t, uint32_t hc, uint32_t w) {
  const uint8_t layout = t.layout[hc];
  const SetAux a = t.aux[hc];
  if (layout == EH_LAYOUT_RANGE_BITSET) {
    Staged st;
    st.words = t.bs_words + a.off;
    st.start = a.start;
    st.n = a.n;
    return probe<P_GBITS>(st, w);
  }
  if (layout == EH_LAYOUT_BLOCK_BITSET) {
    Staged st;
    st.ids = t.bb_id + a.off;
    st.bwords = t.bb_words + 4 * a.off;
    st.n = a.n;
    return probe<P_GBLOCK>(st, w);
  }
  const uint64_t s0 = t.off[hc];
  const uint32_t n = (uint32_t)(t.off[hc + 1] - s0);
  if (!n) return 0;
  return list_contains<false>(t.vals + s0, n, w) ? 1u : 0u;
}

__device__ __forceinline__ uint32_t sel_bit(const uint32_t* sel, uint32_t x) {
  return (__ldg(sel + (x >> 5)) >> (x & 31)) & 1u;
}

// With a selection (sel != null, bit per node value of the partner set
// {a : (a,v) in Edge}), only 4-cliques whose root a is selected count.  On
// an oriented relation the row's a is the plan's root: other rows are
// skipped.  On a symmetric relation the one undirected clique found stands
// for its 4! orderings, of which 3! start at each member: the hit counts
// the members that are selected (the host multiplies by 3!).
template <int P>
__device__ uint64_t clique_rows(const Staged& st, const TrieView& t, const RevView& r, uint32_t kb, uint32_t ke,
                                uint32_t* sbuf, uint32_t cap, const uint32_t* sel, uint32_t wb) {
  const uint32_t lane = lane_id();
  const bool up = r.dir != DIR_DOWN;
  const bool general = r.dir == DIR_GENERAL;
  uint64_t cnt = 0;
  for (uint32_t k = kb; k < ke; k++) {
    uint32_t wab = 0;
    if (sel) {
      const uint32_t wa = sel_bit(sel, __ldg(t.head + __ldg(r.rev_src + k)));
      if (r.dir != DIR_SYM && !wa) continue;  // warp-uniform: k is the same on every lane
      wab = wa + wb;
    }
    const uint32_t lo = __ldg(r.rev_lo + k), hi = __ldg(r.rev_hi + k);
    // S = N(a)[lo, hi) ∩ N(b), compacted in order
    uint32_t ns = 0;
    for (uint32_t base = lo; base < hi; base += 32) {
      const uint32_t e = base + lane;
      uint32_t w = 0, hit = 0;
      if (e < hi) {
        w = __ldg(t.vals + e);
        hit = probe<P>(st, w);
      }
      const uint32_t ball = __ballot_sync(kFull, hit);
      if (hit) {
        const uint32_t pos = ns + __popc(ball & lanemask_lt());
        if (pos < cap) sbuf[pos] = w;
      }
      ns += __popc(ball);
    }
    __syncwarp();
    if (ns > cap) ns = cap;  // capacity bound checked by the host planner
    // small S: the (c, d) pairs flattened over the lanes, so a warp step
    // probes 32 pairs whatever the length of each c's run
    if (ns <= kFlatClique) {
      const uint32_t np = general ? ns * ns : ns * (ns - 1) / 2;
      for (uint32_t p = lane; p < np; p += 32) {
        uint32_t i, j;  // the pair's positions in S: i < j unless general
        if (general) {
          i = p / ns;
          j = p - i * ns;
        } else {
          // row i of the triangular pair index holds ns - 1 - i pairs and
          // starts at i * ns - i * (i + 1) / 2; a float guess, then exact steps
          const float m = (float)(2 * ns - 1);
          int g = (int)floorf((m - sqrtf(fmaxf(m * m - 8.f * (float)p, 0.f))) * 0.5f);
          g = max(0, min(g, (int)ns - 2));
          i = (uint32_t)g;
          while (i + 1 < ns - 1 && (i + 1) * ns - (i + 1) * (i + 2) / 2 <= p) i++;
          while (i > 0 && i * ns - i * (i + 1) / 2 > p) i--;
          j = p - (i * ns - i * (i + 1) / 2) + i + 1;
        }
        // up (and general): probe d = S[j] in N(S[i]); down: d = S[i] in N(S[j])
        const uint32_t c = (up || general) ? sbuf[i] : sbuf[j];
        const uint32_t dd = (up || general) ? sbuf[j] : sbuf[i];
        const int32_t hc = __ldg(t.head_index + c);
        if (hc < 0) continue;
        if (probe_global_set(t, (uint32_t)hc, dd))
          cnt += (sel && r.dir == DIR_SYM) ? wab + sel_bit(sel, c) + sel_bit(sel, dd) : 1u;
      }
      __syncwarp();
      continue;
    }
    // for each c = S[i]: count S elements beyond c (up) or before c (down) in N(c)
    for (uint32_t i = 0; i < ns; i++) {
      const uint32_t c = sbuf[i];
      const int32_t hc = __ldg(t.head_index + c);
      if (hc < 0) continue;
      const uint32_t jb = general ? 0 : (up ? i + 1 : 0), je = general ? ns : (up ? ns : i);
      if (sel && r.dir == DIR_SYM) {
        const uint32_t wabc = wab + sel_bit(sel, c);
        for (uint32_t j = jb + lane; j < je; j += 32)
          if (probe_global_set(t, (uint32_t)hc, sbuf[j])) cnt += wabc + sel_bit(sel, sbuf[j]);
      } else {
        for (uint32_t j = jb + lane; j < je; j += 32) cnt += probe_global_set(t, (uint32_t)hc, sbuf[j]);
      }
    }
    __syncwarp();
  }
  return cnt;
}

__global__ void EH_TRI_LAUNCH_BOUNDS clique4_kernel(const TrieView* __restrict__ views,
                                                       const RevView* __restrict__ revs,
                                                       const Item* __restrict__ items, uint32_t n_items,
                                                       int cap_words, QueryOut out) {
  extern __shared__ uint32_t smem[];
  const uint32_t lane = lane_id();
  const uint32_t wid = threadIdx.x >> 5;
  uint32_t* sm = smem + (size_t)wid * cap_words;
  // S after the staged set in the warp's region, or in its global buffer
  const int half = out.gsbuf ? cap_words : cap_words / 2;
  uint32_t* sbuf = out.gsbuf ? out.gsbuf + ((size_t)blockIdx.x * (blockDim.x >> 5) + wid) * out.gcap : sm + half;
  const uint32_t scap = out.gsbuf ? out.gcap : (uint32_t)half;
  unsigned long long acc = 0;
  uint32_t cur_g = 0xffffffffu;
  for (;;) {
    uint32_t q = 0;
    if (lane == 0) q = atomicAdd(out.queue, 1u);
    q = __shfl_sync(kFull, q, 0);
    const uint64_t it64 = (uint64_t)out.shard_index + (uint64_t)q * out.shard_count;
    if (it64 >= n_items) break;
    const uint32_t it = (uint32_t)it64;
    const Item item = items[it];
    if (item.g != cur_g) {
      if (lane == 0 && cur_g != 0xffffffffu && acc) atomicAdd(out.total + cur_g, acc);
      acc = 0;
      cur_g = item.g;
    }
    const TrieView t = views[item.g];
    const RevView r = revs[item.g];
    long long t0 = 0;
    if (out.records && lane == 0) t0 = clock64();
    Staged st;
    const int mode = stage_set(t, item.hb, sm, half, st);
    const uint32_t wb = out.sel ? sel_bit(out.sel, t.head[item.hb]) : 0u;
    uint64_t c;
    switch (mode) {
      case P_SBITS: c = clique_rows<P_SBITS>(st, t, r, item.kb, item.ke, sbuf, scap, out.sel, wb); break;
      case P_GBITS: c = clique_rows<P_GBITS>(st, t, r, item.kb, item.ke, sbuf, scap, out.sel, wb); break;
      case P_SLIST: c = clique_rows<P_SLIST>(st, t, r, item.kb, item.ke, sbuf, scap, out.sel, wb); break;
      case P_GLIST: c = clique_rows<P_GLIST>(st, t, r, item.kb, item.ke, sbuf, scap, out.sel, wb); break;
      case P_ZBITS: c = clique_rows<P_ZBITS>(st, t, r, item.kb, item.ke, sbuf, scap, out.sel, wb); break;
      default: c = clique_rows<P_GBLOCK>(st, t, r, item.kb, item.ke, sbuf, scap, out.sel, wb); break;
    }
    acc += warp_sum(c);
    __syncwarp();
    if (out.records && lane == 0) {  // the same record as the triangle kernel's
      const long long t1 = clock64();
      const uint64_t b0 = t.off[item.hb];
      const uint32_t len = (uint32_t)(t.off[item.hb + 1] - b0);
      const uint32_t first = t.vals[b0], last = t.vals[b0 + len - 1];
      float* rec = out.records + 8 * (size_t)it;
      rec[0] = (float)len;
      rec[1] = (float)(r.rev_wpre[item.ke] - r.rev_wpre[item.kb]);
      rec[2] = (float)len / (float)(last - first + 1);
      rec[3] = (float)(last - first);
      rec[4] = (float)t.layout[item.hb];
      rec[5] = (float)mode;
      rec[6] = __uint_as_float(item.hb);
      rec[7] = (float)(t1 - t0);
    }
  }
  if (lane == 0 && cur_g != 0xffffffffu && acc) atomicAdd(out.total + cur_g, acc);
}

// ------------------------------------------------- lollipop / barbell roots
constexpr uint64_t kRootBig = 32768;  // barbell root: larger sets get grid-wide passes

// LollipopAgg root, order [a,d]: sum_a T(a) * |N(a)|
// BarbellAgg root, order [a,x]: sum_a T(a) * sum_{x in N(a) ∩ head} T(x);
// Tv = T by value (0 off the head): one random load per row instead of two
template <bool kBarbell>
__global__ void root_kernel(TrieView t, const unsigned long long* __restrict__ T,
                            const unsigned long long* __restrict__ Tv, unsigned long long* __restrict__ total) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  unsigned long long acc = 0;
  for (uint32_t a = warp; a < t.n_head; a += nwarps) {
    const unsigned long long ta = T[a];
    if (!ta) continue;
    if (kBarbell && t.off[a + 1] - t.off[a] > kRootBig) continue;  // root_big_kernel's
    unsigned long long s = 0;
    if (kBarbell) {
      for (uint64_t e = t.off[a] + lane; e < t.off[a + 1]; e += 32) s += __ldg(Tv + __ldg(t.vals + e));
      s = warp_sum(s);
    } else {
      s = t.off[a + 1] - t.off[a];
    }
    acc += ta * s;
  }
  if (lane == 0 && acc) atomicAdd(total, acc);
}

// the barbell root of one large set a, grid-wide
__global__ void root_big_kernel(TrieView t, uint32_t a, const unsigned long long* __restrict__ T,
                                const unsigned long long* __restrict__ Tv, unsigned long long* __restrict__ total) {
  const unsigned long long ta = T[a];
  unsigned long long s = 0;
  for (uint64_t e = t.off[a] + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < t.off[a + 1];
       e += (uint64_t)gridDim.x * blockDim.x)
    s += __ldg(Tv + __ldg(t.vals + e));
  s = warp_sum(s);
  if (lane_id() == 0 && s) atomicAdd(total, ta * s);
}

__global__ void root_big_sets_kernel(TrieView t, uint32_t* __restrict__ idx, unsigned int* __restrict__ n) {
  for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < t.n_head; a += gridDim.x * blockDim.x)
    if (t.off[a + 1] - t.off[a] > kRootBig) idx[atomicAdd(n, 1u)] = a;
}

__global__ void t_by_value_kernel(TrieView t, const unsigned long long* __restrict__ T,
                                  unsigned long long* __restrict__ Tv) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < t.n_nodes; v += gridDim.x * blockDim.x) {
    const int32_t h = t.head_index[v];
    Tv[v] = h >= 0 ? T[h] : 0ull;
  }
}

// ---------------------------------------------------------------- driver
static RevView rev_view(const eh_trie* t) {
  return RevView{t->rev_off.p, t->rev_lo.p, t->rev_hi.p, t->rev_src.p, t->rev_wpre.p, t->dir};
}

static int blocks_per_sm(const void* kernel, int threads, size_t smem) {
  int b = 0;
  EH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem));
  return std::max(1, b);
}

// dynamic shared memory a block of `kernel` may use: the device's opt-in
// per-block limit less the kernel's own static shared memory
static size_t dynamic_smem_room(const void* kernel) {
  int dev = 0, optin = 0;
  EH_CUDA(cudaGetDevice(&dev));
  EH_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  EH_CUDA(cudaFuncGetAttributes(&fa, kernel));
  return (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
}

template <typename K>
static void set_smem_attr(K kernel, size_t smem) {
  EH_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
}

struct Launch {
  uint32_t launches = 0;
  float kernel_ms = 0;
};

// Runs the intersection kernel of `query` over the concatenated plans of
// n graphs; results accumulate into d_total[g].
// Everything a launch needs on the device, built once: the work plans of
// the tries concatenated into one queue, their views, the launch shape.
struct Prepared {
  DevBuf<Item> items;
  uint32_t n_items = 0;
  uint32_t n_bitems = 0;  // items[0, n_bitems) are block items
  uint64_t pairs = 0;
  DevBuf<TrieView> dv;
  DevBuf<RevView> dr;
  DevBuf<unsigned int> q;
  ExecParams ep{};
  size_t smem = 0;
  int grid = 1, threads = 32;
  int query = 0;
  bool annot = false;
  uint32_t plan_launches = 0;
  const uint32_t* sel = nullptr;  // 4-clique selection bitmap (QueryOut::sel)
  DevBuf<uint32_t> gs;            // 4-clique global S buffers (ExecParams::s_cap)
  int32_t hot[kHot] = {-1, -1, -1, -1};  // annotation: largest sets (QueryOut::hot)
};

// head entry with the largest set, excluding `ex` (-1 unused): max over
// (size << 32 | position)
__global__ void top_set_kernel(const uint64_t* __restrict__ off, uint32_t nh, Int4 ex,
                               unsigned long long* __restrict__ best) {
  unsigned long long m = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += gridDim.x * blockDim.x) {
    if ((int32_t)i == ex.v[0] || (int32_t)i == ex.v[1] || (int32_t)i == ex.v[2] || (int32_t)i == ex.v[3]) continue;
    m = max(m, (unsigned long long)(((off[i + 1] - off[i]) << 32) | i));
  }
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
  if (lane_id() == 0 && m) atomicMax(best, m);
}

// the kHot head entries with the largest sets of a trie (-1 where fewer)
static void hot_sets(eh_context* ctx, const eh_trie* t, int32_t* hot) {
  cudaStream_t s = ctx->stream;
  Int4 ex{{-1, -1, -1, -1}};
  DevBuf<unsigned long long> best(1, s);
  for (int k = 0; k < kHot; k++) hot[k] = -1;
  for (int k = 0; k < kHot && (uint32_t)k < t->n_head; k++) {
    EH_CUDA(cudaMemsetAsync(best.p, 0, 8, s));
    top_set_kernel<<<num_sms() * 4, 256, 0, s>>>(t->off.p, t->n_head, ex, best.p);
    EH_CHECK_LAUNCH();
    unsigned long long h = 0;
    EH_CUDA(cudaMemcpyAsync(&h, best.p, 8, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    if (!h) break;
    hot[k] = (int32_t)(h & 0xffffffffu);
    ex.v[k] = hot[k];
  }
}

static void prepare(eh_context* ctx, const eh_trie* const* tries, uint32_t n, int query, ExecParams ep, bool annot,
                    Prepared& P, bool block_items = false) {
  cudaStream_t s = ctx->stream;
  P.query = query;
  P.annot = annot;
  // the launch shape first: the plan's classes depend on the staging capacity
  // the annotated pass stages more of N(b) by default: its matched elements
  // then count in shared memory (measured on Chung-Lu 2^23: 2048 words per
  // warp 234 ms, 1024 245 ms)
  if (annot && !ep.smem_given) ep.smem_words = 2 * kDefaultSmemWords;
  P.threads = 32 * ep.warps;
  P.smem = (size_t)ep.smem_words * 4 * ep.warps;
  const void* kfn;
  if (query == EH_QUERY_CLIQUE4) kfn = (const void*)clique4_kernel;
  else if (annot) kfn = (const void*)triangle_kernel<MODE_ANNOT>;
  else kfn = (const void*)triangle_kernel<MODE_COUNT>;
  {
    size_t room = dynamic_smem_room(kfn);
    // the materializing pass launches MODE_MAT with the same shape
    if (!annot && query != EH_QUERY_CLIQUE4)
      room = std::min(room, dynamic_smem_room((const void*)triangle_kernel<MODE_MAT>));
    if (P.smem > room) {
      // shrink the per-warp region to what a block may hold (a staged set
      // that no longer fits is probed in global memory instead)
      EH_REQUIRE(query != EH_QUERY_CLIQUE4, EH_ERR_UNSUPPORTED, "4-clique staging exceeds shared memory");
      ep.smem_words = (int)((room / 4 / ep.warps) & ~(size_t)1);
      P.smem = (size_t)ep.smem_words * 4 * ep.warps;
    }
  }
  // block items only for the plain triangle COUNT
  const bool blocks = block_items && query == EH_QUERY_TRIANGLE && !annot && ep.warps > 1 && !ep.no_block_items;
  PlanShape shape{ep.chunk, nullptr, 0.0, (uint32_t)ep.smem_words,
                   blocks ? (uint32_t)ep.smem_words * (uint32_t)ep.warps : 0u, (uint32_t)ep.warps};
  std::vector<Plan> plans(n);
  uint32_t total_items = 0, total_b = 0;
  uint64_t pairs = 0;
  for (uint32_t g = 0; g < n; g++) {
    P.plan_launches += build_plan(ctx, tries[g], shape, g, plans[g]);
    total_items += plans[g].n;
    total_b += plans[g].nb;
    pairs += tries[g]->rev_pairs;
  }
  P.n_items = total_items;
  P.n_bitems = total_b;
  P.pairs = pairs;
  if (n == 1) {
    P.items = std::move(plans[0].items);
  } else {
    // every graph's block items, then every graph's warp items
    P.items.alloc(total_items ? total_items : 1, s);
    uint32_t ob = 0, ow = total_b;
    for (uint32_t g = 0; g < n; g++) {
      const uint32_t nb = plans[g].nb, nw = plans[g].n - plans[g].nb;
      if (nb)
        EH_CUDA(cudaMemcpyAsync(P.items.p + ob, plans[g].items.p, nb * sizeof(Item), cudaMemcpyDeviceToDevice, s));
      if (nw)
        EH_CUDA(cudaMemcpyAsync(P.items.p + ow, plans[g].items.p + nb, nw * sizeof(Item), cudaMemcpyDeviceToDevice,
                                s));
      ob += nb;
      ow += nw;
    }
  }
  std::vector<TrieView> hv(n);
  std::vector<RevView> hr(n);
  for (uint32_t g = 0; g < n; g++) {
    hv[g] = tries[g]->view();
    hr[g] = rev_view(tries[g]);
    // the intersection kernels read the values and the bitset words with
    // 16-byte loads at 16-byte aligned indices
    if ((reinterpret_cast<uintptr_t>(hv[g].vals) | reinterpret_cast<uintptr_t>(hv[g].bs_words)) & 15u)
      throw Error{EH_ERR_UNSUPPORTED, "trie arrays are not 16-byte aligned"};
  }
  P.dv.alloc(n, s);
  P.dr.alloc(n, s);
  P.q.alloc(2, s);
  EH_CUDA(cudaMemcpyAsync(P.dv.p, hv.data(), n * sizeof(TrieView), cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaMemcpyAsync(P.dr.p, hr.data(), n * sizeof(RevView), cudaMemcpyHostToDevice, s));
  if (query == EH_QUERY_CLIQUE4) set_smem_attr(clique4_kernel, P.smem);
  else if (annot) set_smem_attr(triangle_kernel<MODE_ANNOT>, P.smem);
  else set_smem_attr(triangle_kernel<MODE_COUNT>, P.smem);
  const int per_sm = blocks_per_sm(kfn, P.threads, P.smem);
  const uint64_t units = (uint64_t)total_b + (total_items - total_b + ep.warps - 1) / ep.warps;
  P.grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)num_sms() * per_sm, units));
  if (annot && n == 1 && tries[0]->dir == DIR_SYM) hot_sets(ctx, tries[0], P.hot);
  if (query == EH_QUERY_CLIQUE4 && ep.s_cap) {
    // one S buffer per resident warp, at most 2 GiB in all
    const uint64_t per_block = (uint64_t)ep.warps * ep.s_cap * 4;
    P.grid = std::max(1, (int)std::min<uint64_t>((uint64_t)P.grid, (2ull << 30) / per_block));
    P.gs.alloc((size_t)P.grid * ep.warps * ep.s_cap, s);
  }
  P.ep = ep;
  EH_CUDA(cudaStreamSynchronize(s));  // host staging vectors go out of scope
}

// Enqueue one run of a prepared launch: reset the queue, run the persistent
// kernel.  No host synchronisation: capturable in a CUDA graph.
static void launch(eh_context* ctx, Prepared& P, unsigned long long* d_total, unsigned long long* d_annot,
                   float* d_records) {
  cudaStream_t s = ctx->stream;
  if (!P.n_items) return;
  EH_CUDA(cudaMemsetAsync(P.q.p, 0, 8, s));
  const ExecParams& ep = P.ep;
  QueryOut out{ep.shard_index, ep.shard_count, ep.long_row, d_total, d_annot, d_records, P.q.p};
  out.n_bitems = P.n_bitems;
  out.bqueue = P.q.p + 1;
  out.sel = P.sel;
  for (int k = 0; k < kHot; k++) out.hot[k] = P.hot[k];
  out.gsbuf = ep.s_cap ? P.gs.p : nullptr;
  out.gcap = ep.s_cap;
  if (P.query == EH_QUERY_CLIQUE4)
    clique4_kernel<<<P.grid, P.threads, P.smem, s>>>(P.dv.p, P.dr.p, P.items.p, P.n_items, ep.smem_words, out);
  else if (P.annot)
    triangle_kernel<MODE_ANNOT><<<P.grid, P.threads, P.smem, s>>>(P.dv.p, P.dr.p, P.items.p, P.n_items, ep.smem_words,
                                                            out);
  else
    triangle_kernel<MODE_COUNT><<<P.grid, P.threads, P.smem, s>>>(P.dv.p, P.dr.p, P.items.p, P.n_items, ep.smem_words,
                                                             out);
  EH_CHECK_LAUNCH();
}

// Plan + run + wait; the intersection kernel is timed with events.
// 4-clique: the warp's shared region holds the staged N(b) and S
// (S <= the largest set) while that stays within 96 KB a block; beyond, S
// moves to per-warp global buffers (L2-resident in practice) and the whole
// region stages N(b).
static void size_clique_staging(ExecParams& ep, uint32_t max_set) {
  const int need = 2 * ((int)max_set + 1);
  if ((size_t)std::max(ep.smem_words, need) * 4 * ep.warps <= 96 * 1024) {
    if (ep.smem_words < need) ep.smem_words = (need + 1) & ~1;
  } else {
    ep.s_cap = max_set + 1;
  }
}

static Launch run_plans(eh_context* ctx, const eh_trie* const* tries, uint32_t n, int query, ExecParams ep,
                        bool annot, unsigned long long* d_total, unsigned long long* d_annot, float* d_records,
                        uint32_t* n_items_out, uint64_t* pairs_out, const uint32_t* sel = nullptr) {
  cudaStream_t s = ctx->stream;
  Launch L;
  Prepared P;
  {
    TracePhase ph("query.prepare", s);
    prepare(ctx, tries, n, query, ep, annot, P, true);
  }
  P.sel = sel;
  L.launches = P.plan_launches;
  *n_items_out = P.n_items;
  *pairs_out = P.pairs;
  if (!P.n_items) return L;
  EH_CUDA(cudaEventRecord(ctx->ev1, s));
  {
    TracePhase ph("query.kernel", s);
    launch(ctx, P, d_total, d_annot, d_records);
  }
  EH_CUDA(cudaEventRecord(ctx->ev2, s));
  L.launches += 1;
  EH_CUDA(cudaEventSynchronize(ctx->ev2));
  EH_CUDA(cudaEventElapsedTime(&L.kernel_ms, ctx->ev1, ctx->ev2));
  return L;
}

// Algorithmic bytes of the triangle plan: both uint32 inputs of every
// pairwise intersection the reference loop nest evaluates, read once each:
// 4 * sum over rows (a,b) of (d(a) + d(b)) = 4 * (sum_a d(a)^2 + wedges).
static uint64_t triangle_algorithmic_bytes(const eh_trie* t) { return 4 * (t->sum_sq_deg + t->total_wedges); }

static void fill_stats(eh_query_stats* st, float query_ms, const Launch& L, uint32_t items, uint64_t pairs,
                       uint64_t alg) {
  if (!st) return;
  st->query_ms = query_ms;
  st->kernel_ms = L.kernel_ms;
  st->launches = L.launches;
  st->work_items = items;
  st->wedges = pairs;
  st->algorithmic_bytes = alg;
}

// The root bag of the lollipop / barbell plans over a per-head-entry
// annotation T (the annotated bag's z, by head position of t; Tv: the same
// by node value, or null to derive it): LollipopAgg sum_a T(a) * |N(a)|,
// BarbellAgg sum_a T(a) * sum_{x in N(a)} Tv(x).  Adds into total[0];
// returns the kernels launched.
static uint32_t root_bag(eh_context* ctx, const eh_trie* t, int query, const unsigned long long* T,
                         const unsigned long long* Tv, unsigned long long* total) {
  cudaStream_t s = ctx->stream;
  if (!t->n_head) return 0;
  uint32_t launches = 0;
  if (query == EH_QUERY_LOLLIPOP) {
    root_kernel<false><<<num_sms() * 8, 256, 0, s>>>(t->view(), T, nullptr, total);
    EH_CHECK_LAUNCH();
    return 1;
  }
  DevBuf<unsigned long long> tv;
  if (!Tv) {
    tv.alloc(t->n_nodes ? t->n_nodes : 1, s);
    t_by_value_kernel<<<num_sms() * 8, 256, 0, s>>>(t->view(), T, tv.p);
    EH_CHECK_LAUNCH();
    Tv = tv.p;
    launches++;
  }
  root_kernel<true><<<num_sms() * 8, 256, 0, s>>>(t->view(), T, Tv, total);
  EH_CHECK_LAUNCH();
  launches++;
  if (t->info.max_set > kRootBig) {
    DevBuf<uint32_t> idx(t->n_head, s);
    DevBuf<unsigned int> nb(1, s);
    EH_CUDA(cudaMemsetAsync(nb.p, 0, 4, s));
    root_big_sets_kernel<<<num_sms() * 4, 256, 0, s>>>(t->view(), idx.p, nb.p);
    EH_CHECK_LAUNCH();
    unsigned int hn = 0;
    EH_CUDA(cudaMemcpyAsync(&hn, nb.p, 4, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    std::vector<uint32_t> big(hn);
    if (hn) EH_CUDA(cudaMemcpyAsync(big.data(), idx.p, 4ull * hn, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    for (uint32_t a : big) {
      root_big_kernel<<<num_sms() * 4, 256, 0, s>>>(t->view(), a, T, Tv, total);
      EH_CHECK_LAUNCH();
    }
    launches += 1 + hn;
  }
  return launches;
}

// z by node value (zero beyond n_values) -> the same by head position
__global__ void z_by_head_kernel(TrieView t, const unsigned long long* __restrict__ zv, uint32_t n_values,
                                 unsigned long long* __restrict__ T) {
  for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < t.n_head; a += gridDim.x * blockDim.x) {
    const uint32_t v = t.head[a];
    T[a] = v < n_values ? zv[v] : 0ull;
  }
}

// The root bag of lollipop / barbell over an annotation z given by value on
// the host (the generated root bags of an annotated intermediate,
// EHGenerator.scala:399-480 with TrieIterator::get_annotation,
// TrieIterator.cpp:45-59): LOLLIPOP sum_a z(a) |N(a)|, BARBELL
// sum_{(a,x)} z(a) z(x), modulo 2^64.
void query_weighted_root(eh_context* ctx, const eh_trie* t, int query, const uint64_t* z, uint32_t n_values,
                         uint64_t* result) {
  cudaStream_t s = ctx->stream;
  EH_REQUIRE(query == EH_QUERY_LOLLIPOP || query == EH_QUERY_BARBELL, EH_ERR_INVALID,
             "the weighted root bag is EH_QUERY_LOLLIPOP or EH_QUERY_BARBELL");
  EH_REQUIRE(t->ctx == ctx, EH_ERR_INVALID, "trie belongs to another context");
  EH_REQUIRE(n_values == 0 || z, EH_ERR_INVALID, "null annotation");
  const uint32_t nv = std::min(n_values, t->n_nodes);
  DevBuf<unsigned long long> zv(nv ? nv : 1, s), T(t->n_head ? t->n_head : 1, s), total(1, s);
  EH_CUDA(cudaMemsetAsync(total.p, 0, 8, s));
  if (nv) EH_CUDA(cudaMemcpyAsync(zv.p, z, 8ull * nv, cudaMemcpyHostToDevice, s));
  if (t->n_head) {
    z_by_head_kernel<<<num_sms() * 4, 256, 0, s>>>(t->view(), zv.p, nv, T.p);
    EH_CHECK_LAUNCH();
    if (query == EH_QUERY_BARBELL) {
      // Tv over the whole value domain: values of the relation outside its head still carry z
      DevBuf<unsigned long long> tv(t->n_nodes ? t->n_nodes : 1, s);
      EH_CUDA(cudaMemsetAsync(tv.p, 0, (size_t)(t->n_nodes ? t->n_nodes : 1) * 8, s));
      if (nv) EH_CUDA(cudaMemcpyAsync(tv.p, zv.p, 8ull * nv, cudaMemcpyDeviceToDevice, s));
      root_bag(ctx, t, query, T.p, tv.p, total.p);
      unsigned long long h = 0;
      EH_CUDA(cudaMemcpyAsync(&h, total.p, 8, cudaMemcpyDeviceToHost, s));
      EH_CUDA(cudaStreamSynchronize(s));
      *result = h;
      return;
    }
    root_bag(ctx, t, query, T.p, nullptr, total.p);
  }
  unsigned long long h = 0;
  EH_CUDA(cudaMemcpyAsync(&h, total.p, 8, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  *result = h;
}

// The annotated pass's per-head counters take one global atomic per hit
// (2.8 G on Chung-Lu 2^23).  Measured on B200 (Chung-Lu 2^23 lollipop): with
// the counters in the stream-ordered pool the pass ran at 243 or 184 ms
// depending on where the pool placed them (holding a 128 MB allocation before
// the query flipped it); in an allocation of their own from cudaMalloc it ran
// at 184 ms whatever the pool held.  The context keeps one such buffer, grown
// (with the stream drained first) when a larger trie needs it.
static unsigned long long* annot_buffer(eh_context* ctx, size_t n) {
  if (n > ctx->annot_cap) {
    EH_CUDA(cudaStreamSynchronize(ctx->stream));
    if (ctx->annot) EH_CUDA(cudaFree(ctx->annot));
    ctx->annot = nullptr;
    ctx->annot_cap = 0;
    if (cudaMalloc((void**)&ctx->annot, n * sizeof(unsigned long long)) != cudaSuccess) {
      cudaGetLastError();
      ctx->annot = nullptr;
      throw Error{EH_ERR_OOM, "device allocation of " + std::to_string(n * 8) + " bytes failed"};
    }
    ctx->annot_cap = n;
  }
  return ctx->annot;
}

void query_count_batched(eh_context* ctx, const eh_trie* const* tries, uint32_t n, int query,
                         const eh_exec_config* cfg, uint64_t* results, eh_query_stats* stats) {
  cudaStream_t s = ctx->stream;
  EH_REQUIRE(query >= EH_QUERY_TRIANGLE && query <= EH_QUERY_BARBELL, EH_ERR_INVALID, "unknown query");
  EH_REQUIRE(n > 0, EH_ERR_INVALID, "no tries");
  for (uint32_t g = 0; g < n; g++) {
    EH_REQUIRE(tries[g] != nullptr, EH_ERR_INVALID, "null trie");
    EH_REQUIRE(tries[g]->ctx == ctx, EH_ERR_INVALID, "trie belongs to another context");
  }
  ExecParams ep = exec_params(cfg);
  if (query == EH_QUERY_CLIQUE4) {
    uint32_t mx = 0;
    for (uint32_t g = 0; g < n; g++) mx = std::max(mx, tries[g]->info.max_set);
    size_clique_staging(ep, mx);
  }
  TracePhase ph_all("query.total", s);
  EH_CUDA(cudaEventRecord(ctx->ev0, s));
  DevBuf<unsigned long long> total(n, s);
  EH_CUDA(cudaMemsetAsync(total.p, 0, n * 8, s));
  uint32_t items = 0;
  uint64_t pairs = 0;
  Launch L;
  DevBuf<float> rec;
  const bool record = cfg && cfg->record_timings && n == 1;
  if (query == EH_QUERY_TRIANGLE || query == EH_QUERY_CLIQUE4) {
    float* recp = nullptr;
    if (record) {
      // one record per item; the plan size is known only after planning, so
      // size for the worst case of one item per head entry plus splits
      const uint64_t cap = tries[0]->n_head + tries[0]->rev_pairs / ep.chunk + 16;
      rec.alloc(8 * cap, s);
      recp = rec.p;
    }
    L = run_plans(ctx, tries, n, query, ep, false, total.p, nullptr, recp, &items, &pairs);
  } else {
    EH_REQUIRE(n == 1, EH_ERR_UNSUPPORTED, "batched lollipop/barbell is not supported");
    const eh_trie* t = tries[0];
    EH_REQUIRE(ep.shard_count == 1, EH_ERR_UNSUPPORTED, "lollipop/barbell run unsharded");
    float* recp = nullptr;
    if (record) {  // the annotated triangle pass's items (the root bag is not logged)
      rec.alloc(8 * (t->n_head + t->rev_pairs / ep.chunk + 16), s);
      recp = rec.p;
    }
    unsigned long long* T = annot_buffer(ctx, t->n_head ? t->n_head : 1);
    DevBuf<unsigned long long> dummy(1, s);
    EH_CUDA(cudaMemsetAsync(T, 0, (t->n_head ? t->n_head : 1) * 8, s));
    EH_CUDA(cudaMemsetAsync(dummy.p, 0, 8, s));
    L = run_plans(ctx, tries, 1, EH_QUERY_TRIANGLE, ep, true, dummy.p, T, recp, &items, &pairs);
    L.launches += root_bag(ctx, t, query, T, nullptr, total.p);
  }
  std::vector<unsigned long long> h(n);
  EH_CUDA(cudaMemcpyAsync(h.data(), total.p, n * 8, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaEventRecord(ctx->ev2, s));
  EH_CUDA(cudaEventSynchronize(ctx->ev2));
  float qms = 0;
  EH_CUDA(cudaEventElapsedTime(&qms, ctx->ev0, ctx->ev2));
  for (uint32_t g = 0; g < n; g++) {
    uint64_t v = h[g];
    const int dir = tries[g]->dir;
    // on a symmetric relation every undirected triangle is found once (rows
    // a<b) and the reference counts each of its 3! orderings; 4! for 4-cliques
    if (dir == DIR_SYM && query == EH_QUERY_TRIANGLE) v *= 6ull;
    if (dir == DIR_SYM && query == EH_QUERY_CLIQUE4) v *= 24ull;
    results[g] = v;
  }
  if (record) {
    ctx->timing_records.resize(8 * (size_t)items);
    if (items)
      EH_CUDA(cudaMemcpy(ctx->timing_records.data(), rec.p, 8 * (size_t)items * sizeof(float), cudaMemcpyDeviceToHost));
  }
  uint64_t alg = 0;
  for (uint32_t g = 0; g < n; g++) alg += triangle_algorithmic_bytes(tries[g]);
  fill_stats(stats, qms, L, items, pairs, alg);
}

void query_count(eh_context* ctx, const eh_trie* t, int query, const eh_exec_config* cfg, uint64_t* result,
                 eh_query_stats* stats) {
  const eh_trie* ts[1] = {t};
  query_count_batched(ctx, ts, 1, query, cfg, result, stats);
}

void triangle_annotation(eh_context* ctx, const eh_trie* t, const eh_exec_config* cfg, uint64_t* annot_dev) {
  cudaStream_t s = ctx->stream;
  ExecParams ep = exec_params(cfg);
  ep.shard_index = 0;
  ep.shard_count = 1;
  DevBuf<unsigned long long> dummy(1, s);
  EH_CUDA(cudaMemsetAsync(annot_dev, 0, (t->n_head ? t->n_head : 1) * 8, s));
  EH_CUDA(cudaMemsetAsync(dummy.p, 0, 8, s));
  uint32_t items;
  uint64_t pairs;
  const eh_trie* ts[1] = {t};
  run_plans(ctx, ts, 1, EH_QUERY_TRIANGLE, ep, true, dummy.p, (unsigned long long*)annot_dev, nullptr, &items,
            &pairs);
  EH_CUDA(cudaStreamSynchronize(s));
}

// ------------------------------------------------------------ selections
// An equality selection x = v on an attribute with one accessor is answered
// at the head of its relation (emitHeadContainsSelections,
// EHGenerator.scala:681-701): the selected bag holds the partners of v with
// annotation 1 each.  Edge(a,x) in order [x,a] gives
// partners(v) = {a : (a,v) ∈ Edge}: the head entries whose child set holds
// v.  One thread per head entry binary-searches v in its sorted list (kept
// whatever the set's layout).
//   bits: optional bitmap over node values, set for every partner a;
//   T:    optional per-head annotation, summed over the partners into
//         sums[0] and over N(v) ∩ head into sums[1];
//   sums[2] counts the partners.
__global__ void select_partners_kernel(TrieView t, uint32_t v, uint32_t* __restrict__ bits,
                                       const unsigned long long* __restrict__ T,
                                       unsigned long long* __restrict__ sums) {
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long s_in = 0, s_out = 0, n_in = 0;
  for (uint32_t i = tid; i < t.n_head; i += stride) {
    const uint64_t end = t.off[i + 1];
    uint64_t lo = t.off[i], hi = end;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (__ldg(t.vals + mid) < v) lo = mid + 1; else hi = mid;
    }
    if (lo < end && __ldg(t.vals + lo) == v) {
      n_in++;
      if (bits) {
        const uint32_t a = t.head[i];
        atomicOr(bits + (a >> 5), 1u << (a & 31));
      }
      if (T) s_in += T[i];
    }
  }
  if (T && v < t.n_nodes) {
    const int32_t hv = t.head_index[v];
    if (hv >= 0)
      for (uint64_t e = t.off[hv] + tid; e < t.off[hv + 1]; e += stride) {
        const int32_t hx = __ldg(t.head_index + __ldg(t.vals + e));
        if (hx >= 0) s_out += T[hx];
      }
  }
  s_in = warp_sum(s_in);
  s_out = warp_sum(s_out);
  n_in = warp_sum(n_in);
  if (lane_id() == 0) {
    if (s_in) atomicAdd(sums, s_in);
    if (s_out) atomicAdd(sums + 1, s_out);
    if (n_in) atomicAdd(sums + 2, n_in);
  }
}

// FliqueSelAgg(;z) :- 4-clique(a,b,c,d), Edge(a,x), x=v and
// BarbellSelAgg(;w) :- triangle(a,b,c), Edge(a,p), Edge(p,x),
// triangle(x,y,z), p=v (test/graph/travis.py:385-401, 472-487; plans
// QueryPlannerTest.scala:230-304).
//  4-clique: the 4-clique plan with its roots restricted to partners(v).
//  Barbell: bag_1_x_y_z reduces to the scalar sum_{x ∈ N(v)} T(x) and the
//  root bag to sum_{a ∈ partners(v)} T(a) times it, T the triangle
//  annotation of the lollipop/barbell bag.
void query_count_select(eh_context* ctx, const eh_trie* t, int query, uint32_t value, const eh_exec_config* cfg,
                        uint64_t* result, eh_query_stats* stats) {
  cudaStream_t s = ctx->stream;
  EH_REQUIRE(query == EH_QUERY_CLIQUE4_SEL || query == EH_QUERY_BARBELL_SEL, EH_ERR_INVALID,
             "selection queries are EH_QUERY_CLIQUE4_SEL and EH_QUERY_BARBELL_SEL");
  EH_REQUIRE(t->ctx == ctx, EH_ERR_INVALID, "trie belongs to another context");
  ExecParams ep = exec_params(cfg);
  EH_REQUIRE(ep.shard_count == 1, EH_ERR_UNSUPPORTED, "selection plans run unsharded");
  const bool clique = query == EH_QUERY_CLIQUE4_SEL;
  if (clique) {
    size_clique_staging(ep, t->info.max_set);
  }
  EH_CUDA(cudaEventRecord(ctx->ev0, s));
  DevBuf<unsigned long long> sums(4, s);  // partner sum, N(v) sum, partners, plan total
  EH_CUDA(cudaMemsetAsync(sums.p, 0, 32, s));
  const uint64_t nbits = t->n_nodes ? ((uint64_t)t->n_nodes + 31) / 32 : 1;
  DevBuf<uint32_t> bits;
  if (clique) {
    bits.alloc(nbits, s);
    EH_CUDA(cudaMemsetAsync(bits.p, 0, nbits * 4, s));
  }
  const int sgrid = num_sms() * 8;
  Launch L;
  if (t->n_head) {
    select_partners_kernel<<<sgrid, 256, 0, s>>>(t->view(), value, clique ? bits.p : nullptr, nullptr, sums.p);
    EH_CHECK_LAUNCH();
    L.launches++;
  }
  // Encoding::value_to_key.at(v) throws for a value in neither column
  int32_t hv = -1;
  if (value < t->n_nodes)
    EH_CUDA(cudaMemcpyAsync(&hv, t->head_index.p + value, 4, cudaMemcpyDeviceToHost, s));
  unsigned long long h[4] = {0, 0, 0, 0};
  EH_CUDA(cudaMemcpyAsync(h, sums.p, 32, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  EH_REQUIRE(hv >= 0 || h[2] > 0, EH_ERR_INVALID,
             "selection value " + std::to_string(value) + " is not in the relation");
  uint32_t items = 0;
  uint64_t pairs = 0;
  const eh_trie* ts[1] = {t};
  uint64_t v = 0;
  if (h[2] > 0) {  // no partners: the selected bag is empty and so is the join
    if (clique) {
      Launch K = run_plans(ctx, ts, 1, EH_QUERY_CLIQUE4, ep, false, sums.p + 3, nullptr, nullptr, &items, &pairs,
                           bits.p);
      L.launches += K.launches;
      L.kernel_ms = K.kernel_ms;
      EH_CUDA(cudaMemcpyAsync(h, sums.p, 32, cudaMemcpyDeviceToHost, s));
      EH_CUDA(cudaStreamSynchronize(s));
      v = h[3];
      if (t->dir == DIR_SYM) v *= 6ull;  // 3! orderings start at each selected member
    } else if (hv >= 0) {
      DevBuf<unsigned long long> T(t->n_head, s), dummy(1, s);
      EH_CUDA(cudaMemsetAsync(T.p, 0, (size_t)t->n_head * 8, s));
      EH_CUDA(cudaMemsetAsync(dummy.p, 0, 8, s));
      EH_CUDA(cudaMemsetAsync(sums.p, 0, 32, s));
      Launch K = run_plans(ctx, ts, 1, EH_QUERY_TRIANGLE, ep, true, dummy.p, T.p, nullptr, &items, &pairs);
      select_partners_kernel<<<sgrid, 256, 0, s>>>(t->view(), value, nullptr, T.p, sums.p);
      EH_CHECK_LAUNCH();
      L.launches += K.launches + 1;
      L.kernel_ms = K.kernel_ms;
      EH_CUDA(cudaMemcpyAsync(h, sums.p, 32, cudaMemcpyDeviceToHost, s));
      EH_CUDA(cudaStreamSynchronize(s));
      v = (uint64_t)h[0] * (uint64_t)h[1];
    }
  }
  EH_CUDA(cudaEventRecord(ctx->ev2, s));
  EH_CUDA(cudaEventSynchronize(ctx->ev2));
  float qms = 0;
  EH_CUDA(cudaEventElapsedTime(&qms, ctx->ev0, ctx->ev2));
  *result = v;
  fill_stats(stats, qms, L, items, pairs, triangle_algorithmic_bytes(t));
}

// ------------------------------------------------------------ materialize
// Triangle(a,b,c) :- Edge(a,b),Edge(b,c),Edge(a,c) as tuples sorted by
// (a,b,c): the rows Trie::foreach (Trie.cpp:130-160) yields on the
// reference's materialized output trie (TrieBuilder::build_set /
// allocate_next / set_level, TrieBuilder.cpp:44-221, 376-410).  One counting
// run sizes every work item's slice, a second run writes the tuples into
// the slices, and two stable key-value radix sorts (by c, then by (a,b))
// order them.
__global__ void iota_kernel(uint32_t* __restrict__ v, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}
__global__ void widen_kernel(const uint32_t* __restrict__ c, uint64_t n, uint64_t* __restrict__ k) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    k[i] = c[i];
}
// keys2[i] = a[idx[i]] << bb | b[idx[i]], vals2[i] = c value (keys1[i])
__global__ void ab_key_kernel(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                              const uint32_t* __restrict__ idx, const uint64_t* __restrict__ csorted, uint64_t n,
                              int bb, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t j = idx[i];
    keys[i] = ((uint64_t)a[j] << bb) | b[j];
    vals[i] = (uint32_t)csorted[i];
  }
}
__global__ void split_ab_kernel(const uint64_t* __restrict__ keys, uint64_t n, int bb, uint32_t* __restrict__ a,
                                uint32_t* __restrict__ b) {
  const uint64_t mask = (1ull << bb) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    a[i] = (uint32_t)(keys[i] >> bb);
    b[i] = (uint32_t)(keys[i] & mask);
  }
}

// TriangleProj(a,b): the reference's plan drops attributes that are neither
// materialized, selected nor aggregated (codegen/query/QueryPlan.scala:245),
// so c is never intersected: the rows are (a,b) with b in N(a) ∩ head, in
// trie order.  One flag + scan + compact over the rows.
__global__ void proj_flag_kernel(TrieView t, uint32_t* __restrict__ flag) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < t.rows; e += (uint64_t)gridDim.x * blockDim.x)
    flag[e] = __ldg(t.head_index + t.vals[e]) >= 0 ? 1u : 0u;
}
__global__ void proj_write_kernel(TrieView t, const uint32_t* __restrict__ seg, const uint32_t* __restrict__ pos,
                                  uint32_t* __restrict__ a, uint32_t* __restrict__ b) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < t.rows; e += (uint64_t)gridDim.x * blockDim.x)
    if (__ldg(t.head_index + t.vals[e]) >= 0) {
      a[pos[e]] = t.head[seg[e]];
      b[pos[e]] = t.vals[e];
    }
}
__global__ void seg_of_rows_kernel(const uint64_t* __restrict__ off, uint32_t nh, uint32_t* __restrict__ seg) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = warp; i < nh; i += nwarps)
    for (uint64_t e = off[i] + lane; e < off[i + 1]; e += 32) seg[e] = i;
}

static void query_project_ab(eh_context* ctx, const eh_trie* t, uint32_t* ha, uint32_t* hb, uint64_t cap,
                             uint64_t* n_rows) {
  cudaStream_t s = ctx->stream;
  *n_rows = 0;
  if (!t->rows) return;
  const int grid = num_sms() * 8;
  DevBuf<uint32_t> pos(t->rows, s), seg(t->rows, s), tot(1, s);
  proj_flag_kernel<<<grid, 256, 0, s>>>(t->view(), pos.p);
  EH_CHECK_LAUNCH();
  exclusive_scan<uint32_t>(pos.p, pos.p, t->rows, tot.p, s);
  uint32_t m = 0;
  EH_CUDA(cudaMemcpyAsync(&m, tot.p, 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  *n_rows = m;
  if (!ha || !hb || !m) return;
  EH_REQUIRE(cap >= m, EH_ERR_INVALID, "output columns hold fewer rows than the result");
  DevBuf<uint32_t> da(m, s), db(m, s);
  seg_of_rows_kernel<<<grid, 256, 0, s>>>(t->off.p, t->n_head, seg.p);
  proj_write_kernel<<<grid, 256, 0, s>>>(t->view(), seg.p, pos.p, da.p, db.p);
  EH_CHECK_LAUNCH();
  EH_CUDA(cudaMemcpyAsync(ha, da.p, (size_t)m * 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaMemcpyAsync(hb, db.p, (size_t)m * 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
}

void query_materialize(eh_context* ctx, const eh_trie* t, int query, const eh_exec_config* cfg, int n_cols,
                       uint32_t* ha, uint32_t* hb, uint32_t* hc, uint64_t cap, uint64_t* n_rows) {
  cudaStream_t s = ctx->stream;
  EH_REQUIRE(query == EH_QUERY_TRIANGLE, EH_ERR_UNSUPPORTED, "materialized output is built for the triangle plan");
  EH_REQUIRE(n_cols == 2 || n_cols == 3, EH_ERR_INVALID, "n_cols must be 3 (a,b,c) or 2 (projection on a,b)");
  EH_REQUIRE(t->ctx == ctx, EH_ERR_INVALID, "trie belongs to another context");
  if (n_cols == 2) {
    query_project_ab(ctx, t, ha, hb, cap, n_rows);
    return;
  }
  uint64_t n = 0;
  query_count(ctx, t, EH_QUERY_TRIANGLE, cfg, &n, nullptr);
  *n_rows = n;
  if (n == 0 || !ha || !hb || !hc) return;  // the row count is the triangle count
  EH_REQUIRE(cap >= n, EH_ERR_INVALID, "output columns hold fewer rows than the result");
  EH_REQUIRE(n < (1ull << 32), EH_ERR_UNSUPPORTED, "materialized results hold fewer than 2^32 rows");
  ExecParams ep = exec_params(cfg);
  ep.shard_index = 0;
  ep.shard_count = 1;
  Prepared P;
  const eh_trie* ts[1] = {t};
  prepare(ctx, ts, 1, EH_QUERY_TRIANGLE, ep, false, P);
  set_smem_attr(triangle_kernel<MODE_MAT>, P.smem);
  DevBuf<unsigned long long> counts(P.n_items ? P.n_items : 1, s), offs(P.n_items ? P.n_items : 1, s),
      total(1, s), rows(1, s);
  EH_CUDA(cudaMemsetAsync(total.p, 0, 8, s));
  const uint32_t mult = t->dir == DIR_SYM ? 6u : 1u;
  QueryOut out{0, 1, P.ep.long_row, total.p, nullptr, nullptr, P.q.p};
  out.item_counts = counts.p;
  out.count_mult = mult;
  EH_CUDA(cudaMemsetAsync(P.q.p, 0, 8, s));
  triangle_kernel<MODE_COUNT><<<P.grid, P.threads, P.smem, s>>>(P.dv.p, P.dr.p, P.items.p, P.n_items,
                                                                P.ep.smem_words, out);
  EH_CHECK_LAUNCH();
  exclusive_scan<uint64_t>((const uint64_t*)counts.p, (uint64_t*)offs.p, P.n_items, (uint64_t*)rows.p, s);
  uint64_t nr = 0;
  EH_CUDA(cudaMemcpyAsync(&nr, rows.p, 8, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  EH_REQUIRE(nr == n, EH_ERR_CUDA, "materialize: counting runs disagree");
  DevBuf<uint32_t> ma(n, s), mb(n, s), mc(n, s);
  out.item_counts = nullptr;
  out.item_off = offs.p;
  out.ma = ma.p;
  out.mb = mb.p;
  out.mc = mc.p;
  EH_CUDA(cudaMemsetAsync(P.q.p, 0, 8, s));
  triangle_kernel<MODE_MAT><<<P.grid, P.threads, P.smem, s>>>(P.dv.p, P.dr.p, P.items.p, P.n_items,
                                                              P.ep.smem_words, out);
  EH_CHECK_LAUNCH();
  // order by (a, b, c): stable sort by c, then stable sort by (a, b)
  const int grid = num_sms() * 8;
  const int bb = bits_for(t->n_nodes ? t->n_nodes - 1 : 0);
  DevBuf<uint64_t> k1(n, s), k1t(n, s);
  DevBuf<uint32_t> idx(n, s), idxt(n, s);
  widen_kernel<<<grid, 256, 0, s>>>(mc.p, n, k1.p);
  iota_kernel<<<grid, 256, 0, s>>>(idx.p, n);
  EH_CHECK_LAUNCH();
  radix_sort_kv(k1.p, k1t.p, idx.p, idxt.p, n, bb, s);
  DevBuf<uint64_t> k2(n, s);
  DevBuf<uint32_t> v2(n, s);
  ab_key_kernel<<<grid, 256, 0, s>>>(ma.p, mb.p, idx.p, k1.p, n, bb, k2.p, v2.p);
  EH_CHECK_LAUNCH();
  radix_sort_kv(k2.p, k1t.p, v2.p, idxt.p, n, 2 * bb, s);
  split_ab_kernel<<<grid, 256, 0, s>>>(k2.p, n, bb, ma.p, mb.p);
  EH_CHECK_LAUNCH();
  EH_CUDA(cudaMemcpyAsync(ha, ma.p, n * 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaMemcpyAsync(hb, mb.p, n * 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaMemcpyAsync(hc, v2.p, n * 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
}

// One triangle / 4-clique COUNT of one trie with every piece of device
// scratch (queue, total, views, planner arrays, scan tile sums, work items,
// and the 4-clique's per-warp S buffers when a set is too large for shared
// memory) carved out of `scratch` (256-byte aligned, `bytes` long):
// allocates nothing.  Throws EH_ERR_UNSUPPORTED when the trie needs more
// scratch.  Every check that can fail before the last one is made before
// the first launch; the last (the work plan's size) after a synchronisation,
// so a failing call leaves no work of its own in flight.
static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

void query_count_in_scratch(eh_context* ctx, const eh_trie* t, int query, const eh_exec_config* cfg,
                            unsigned char* scratch, size_t bytes, uint64_t* result) {
  cudaStream_t s = ctx->stream;
  EH_REQUIRE(query == EH_QUERY_TRIANGLE || query == EH_QUERY_CLIQUE4, EH_ERR_UNSUPPORTED,
             "the allocation-free path runs the triangle and 4-clique plans");
  EH_REQUIRE(t->ctx == ctx, EH_ERR_INVALID, "trie belongs to another context");
  ExecParams ep = exec_params(cfg);
  EH_REQUIRE(ep.shard_count == 1, EH_ERR_UNSUPPORTED, "the allocation-free path runs unsharded");
  const bool clique = query == EH_QUERY_CLIQUE4;
  if (clique) {
    size_clique_staging(ep, t->info.max_set);
  }
  // launch shape and shared memory, checked before anything is launched
  const int threads = 32 * ep.warps;
  const size_t smem = (size_t)ep.smem_words * 4 * ep.warps;
  const void* kfn = clique ? (const void*)clique4_kernel : (const void*)triangle_kernel<MODE_COUNT>;
  {
    const size_t room = dynamic_smem_room(kfn);
    EH_REQUIRE(smem <= room, EH_ERR_UNSUPPORTED,
               "shared staging of " + std::to_string(smem) + " bytes per block is above the " + std::to_string(room) +
                   " a block may use");
  }
  if (clique) set_smem_attr(clique4_kernel, smem);
  else set_smem_attr(triangle_kernel<MODE_COUNT>, smem);
  const int per_sm = blocks_per_sm(kfn, threads, smem);
  // carve the scratch
  const uint32_t nh = t->n_head;
  const uint64_t scan_elems = scan_scratch_elems(nh);
  const size_t off_ctrl = 0;  // u32 queue, u32 unused, u64 total
  const size_t off_tv = 256;
  const size_t off_rv = align256(off_tv + sizeof(TrieView));
  const size_t off_nitems = align256(off_rv + sizeof(RevView));
  const size_t off_ipos = align256(off_nitems + 4ull * nh);
  const size_t off_tot = align256(off_ipos + 4ull * nh);
  const size_t off_scan = align256(off_tot + 4);
  const size_t off_items = align256(off_scan + 4ull * scan_elems);
  EH_REQUIRE(off_items <= bytes, EH_ERR_UNSUPPORTED,
             "trie too large for the allocation-free path: its planner needs " + std::to_string(off_items) +
                 " bytes of scratch before the work items, the path holds " + std::to_string(bytes));
  unsigned int* queue = reinterpret_cast<unsigned int*>(scratch + off_ctrl);
  unsigned long long* total = reinterpret_cast<unsigned long long*>(scratch + off_ctrl + 8);
  TrieView* dv = reinterpret_cast<TrieView*>(scratch + off_tv);
  RevView* dr = reinterpret_cast<RevView*>(scratch + off_rv);
  uint32_t* nitems = reinterpret_cast<uint32_t*>(scratch + off_nitems);
  uint32_t* ipos = reinterpret_cast<uint32_t*>(scratch + off_ipos);
  uint32_t* tot = reinterpret_cast<uint32_t*>(scratch + off_tot);
  uint32_t* scan_tmp = reinterpret_cast<uint32_t*>(scratch + off_scan);
  Item* items = reinterpret_cast<Item*>(scratch + off_items);
  // the array keeps the previous call's contents: zero what must start at 0
  EH_CUDA(cudaMemsetAsync(scratch + off_ctrl, 0, 16, s));
  const TrieView hv = t->view();
  const RevView hr = rev_view(t);
  EH_CUDA(cudaMemcpyAsync(dv, &hv, sizeof(TrieView), cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaMemcpyAsync(dr, &hr, sizeof(RevView), cudaMemcpyHostToDevice, s));
  uint32_t n_items = 0;
  const int pgrid = num_sms() * 4;
  if (t->rev_entries) {
    plan_count_kernel<<<pgrid, 256, 0, s>>>(hr, nh, ep.chunk, nitems);
    EH_CHECK_LAUNCH();
    exclusive_scan_scratch<uint32_t>(nitems, ipos, nh, tot, scan_tmp, scan_elems, s);
    EH_CUDA(cudaMemcpyAsync(&n_items, tot, 4, cudaMemcpyDeviceToHost, s));
  }
  EH_CUDA(cudaStreamSynchronize(s));  // nothing of this call is in flight past here
  const size_t items_end = align256(off_items + sizeof(Item) * (size_t)n_items);
  EH_REQUIRE(items_end <= bytes, EH_ERR_UNSUPPORTED,
             "trie too large for the allocation-free path: it needs " + std::to_string(items_end) +
                 " bytes of scratch, the path holds " + std::to_string(bytes));
  int grid = std::max(1, std::min(num_sms() * per_sm, (int)((n_items + ep.warps - 1) / ep.warps)));
  uint32_t* gsbuf = nullptr;
  if (clique && ep.s_cap) {
    // one S buffer of s_cap words per resident warp, after the work items;
    // fewer blocks when the rest of the array holds fewer buffers
    const uint64_t per_block = (uint64_t)ep.warps * ep.s_cap * 4;
    const uint64_t fit = (bytes - items_end) / per_block;
    EH_REQUIRE(fit >= 1, EH_ERR_UNSUPPORTED,
               "4-clique: the largest set (" + std::to_string(t->info.max_set) +
                   " elements) needs S buffers of " + std::to_string(per_block) +
                   " bytes per block, more than the allocation-free path has left");
    grid = (int)std::min<uint64_t>((uint64_t)grid, fit);
    gsbuf = reinterpret_cast<uint32_t*>(scratch + items_end);
  }
  if (n_items) {
    plan_fill_kernel<<<pgrid, 256, 0, s>>>(hr, nh, nitems, ipos, n_items, 0, items);
    EH_CHECK_LAUNCH();
    QueryOut out{0, 1, ep.long_row, total, nullptr, nullptr, queue};
    out.gsbuf = gsbuf;
    out.gcap = ep.s_cap;
    if (clique)
      clique4_kernel<<<grid, threads, smem, s>>>(dv, dr, items, n_items, ep.smem_words, out);
    else
      triangle_kernel<MODE_COUNT><<<grid, threads, smem, s>>>(dv, dr, items, n_items, ep.smem_words, out);
    EH_CHECK_LAUNCH();
  }
  unsigned long long h = 0;
  EH_CUDA(cudaMemcpyAsync(&h, total, 8, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  uint64_t v = h;
  if (t->dir == DIR_SYM) v *= clique ? 24ull : 6ull;
  *result = v;
}

}  // namespace eh

// ------------------------------------------------------------------ batches
// A prepared batch: one queue over every trie's work items and the whole
// step captured once as a CUDA graph (zero results, zero queue, persistent
// kernel, results to pinned host memory).  A run is one graph launch.
struct eh_batch {
  eh_context* ctx = nullptr;
  eh::Prepared P;
  eh::DevBuf<unsigned long long> total;
  unsigned long long* host = nullptr;  // pinned
  std::vector<int> dirs;
  uint32_t n = 0;
  int query = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~eh_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (host) cudaFreeHost(host);
  }
};

namespace eh {

eh_batch* batch_create(eh_context* ctx, const eh_trie* const* tries, uint32_t n, int query,
                       const eh_exec_config* cfg) {
  cudaStream_t s = ctx->stream;
  EH_REQUIRE(n > 0, EH_ERR_INVALID, "no tries");
  EH_REQUIRE(query == EH_QUERY_TRIANGLE || query == EH_QUERY_CLIQUE4, EH_ERR_UNSUPPORTED,
             "batches run the triangle or 4-clique plan");
  ExecParams ep = exec_params(cfg);
  uint32_t mx = 0;
  for (uint32_t g = 0; g < n; g++) {
    EH_REQUIRE(tries[g] && tries[g]->ctx == ctx, EH_ERR_INVALID, "null trie or trie of another context");
    if (query == EH_QUERY_CLIQUE4) {
      mx = std::max(mx, tries[g]->info.max_set);
    }
  }
  if (query == EH_QUERY_CLIQUE4) size_clique_staging(ep, mx);
  auto* b = new eh_batch();
  try {
    b->ctx = ctx;
    b->n = n;
    b->query = query;
    for (uint32_t g = 0; g < n; g++) b->dirs.push_back(tries[g]->dir);
    prepare(ctx, tries, n, query, ep, false, b->P, true);
    b->total.alloc(n, s);
    EH_CUDA(cudaMallocHost((void**)&b->host, n * sizeof(unsigned long long)));
    EH_CUDA(cudaStreamSynchronize(s));
    EH_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t cap = cudaSuccess;
    try {
      EH_CUDA(cudaMemsetAsync(b->total.p, 0, n * 8, s));
      launch(ctx, b->P, b->total.p, nullptr, nullptr);
      EH_CUDA(cudaMemcpyAsync(b->host, b->total.p, n * 8, cudaMemcpyDeviceToHost, s));
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    cap = cudaStreamEndCapture(s, &b->graph);
    EH_CUDA(cap);
    EH_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  } catch (...) {
    delete b;
    throw;
  }
  return b;
}

void batch_run(eh_context* ctx, eh_batch* b, uint64_t* results, eh_query_stats* stats) {
  cudaStream_t s = ctx->stream;
  EH_REQUIRE(b->ctx == ctx, EH_ERR_INVALID, "batch belongs to another context");
  EH_CUDA(cudaEventRecord(ctx->ev0, s));
  EH_CUDA(cudaGraphLaunch(b->exec, s));
  EH_CUDA(cudaEventRecord(ctx->ev2, s));
  EH_CUDA(cudaEventSynchronize(ctx->ev2));
  float ms = 0;
  EH_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev2));
  for (uint32_t g = 0; g < b->n; g++) {
    uint64_t v = b->host[g];
    if (b->dirs[g] == DIR_SYM) v *= b->query == EH_QUERY_CLIQUE4 ? 24ull : 6ull;
    results[g] = v;
  }
  if (stats) {
    stats->query_ms = ms;
    stats->kernel_ms = ms;
    stats->launches = 1;
    stats->work_items = b->P.n_items;
    stats->wedges = b->P.pairs;
    stats->algorithmic_bytes = 0;
  }
}

void batch_free(eh_batch* b) {
  cudaSetDevice(b->ctx->device);
  cudaStream_t s = b->ctx->stream;
  cudaStreamSynchronize(s);
  delete b;
  cudaStreamSynchronize(s);
}

}  // namespace eh
