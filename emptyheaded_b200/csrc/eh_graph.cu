// Input pipeline on the device: seeded edge-sample generators (Erdős–Rényi,
// R-MAT, Chung–Lu) and the preprocessing that turns samples into the
// encoded Edge relation the reference tests load (symmetrise, drop
// self-loops, dedup, relabel by degree, orient or keep both directions).
#include <cmath>
#include <vector>

#include "eh_internal.cuh"

namespace eh {

// ---------------------------------------------------------------- samples
__global__ void gen_er_kernel(uint64_t seedm, uint32_t n, uint64_t m, uint32_t* __restrict__ u,
                              uint32_t* __restrict__ v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t h = rand64(seedm, i);
    u[i] = (uint32_t)(((uint64_t)(uint32_t)h * n) >> 32);
    v[i] = (uint32_t)(((uint64_t)(uint32_t)(h >> 32) * n) >> 32);
  }
}

// R-MAT: per level one 32-bit draw picks a quadrant against fixed-point
// thresholds t0 < t1 < t2 (a, a+b, a+b+c); two levels per 64-bit draw.
__global__ void gen_rmat_kernel(uint64_t seedm, int scale, uint64_t m, uint32_t t0, uint32_t t1, uint32_t t2,
                                uint32_t* __restrict__ u, uint32_t* __restrict__ v) {
  const int words = (scale + 1) / 2;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t x = 0, y = 0;
    for (int w = 0; w < words; w++) {
      const uint64_t h = rand64(seedm, (i << 5) | (uint64_t)w);
#pragma unroll
      for (int half = 0; half < 2; half++) {
        const int level = 2 * w + half;
        if (level < scale) {
          const uint32_t r = half ? (uint32_t)(h >> 32) : (uint32_t)h;
          const uint32_t bit = 1u << (scale - 1 - level);
          if (r >= t0) {
            if (r < t1) y |= bit;
            else if (r < t2) x |= bit;
            else { x |= bit; y |= bit; }
          }
        }
      }
    }
    u[i] = x;
    v[i] = y;
  }
}

__device__ __forceinline__ uint32_t cdf_pick(const uint64_t* __restrict__ cdf, uint32_t n, uint64_t r63) {
  uint32_t lo = 0, hi = n - 1;  // first i with cdf[i] > r63
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (__ldg(cdf + mid) > r63) hi = mid; else lo = mid + 1;
  }
  return lo;
}
__global__ void gen_chunglu_kernel(uint64_t seedm, uint32_t n, uint64_t m, const uint64_t* __restrict__ cdf,
                                   uint32_t* __restrict__ u, uint32_t* __restrict__ v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    u[i] = cdf_pick(cdf, n, rand64(seedm, 2 * i) >> 1);
    v[i] = cdf_pick(cdf, n, rand64(seedm, 2 * i + 1) >> 1);
  }
}

void gen_er(cudaStream_t s, uint64_t seed, uint32_t n, uint64_t m, uint32_t* u, uint32_t* v) {
  EH_REQUIRE(n > 0, EH_ERR_INVALID, "n must be positive");
  if (!m) return;
  gen_er_kernel<<<num_sms() * 8, 256, 0, s>>>(splitmix64(seed), n, m, u, v);
  EH_CHECK_LAUNCH();
}

void rmat_thresholds(double a, double b, double c, uint32_t t[3]) {
  const double sc = 4294967296.0;
  t[0] = (uint32_t)std::floor(a * sc);
  t[1] = (uint32_t)std::floor((a + b) * sc);
  t[2] = (uint32_t)std::floor((a + b + c) * sc);
}

void gen_rmat(cudaStream_t s, uint64_t seed, int scale, uint64_t m, double a, double b, double c, uint32_t* u,
              uint32_t* v) {
  EH_REQUIRE(scale >= 1 && scale <= 31, EH_ERR_INVALID, "R-MAT scale must be in [1, 31]");
  EH_REQUIRE(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0, EH_ERR_INVALID, "bad R-MAT probabilities");
  if (!m) return;
  uint32_t t[3];
  rmat_thresholds(a, b, c, t);
  gen_rmat_kernel<<<num_sms() * 8, 256, 0, s>>>(splitmix64(seed), scale, m, t[0], t[1], t[2], u, v);
  EH_CHECK_LAUNCH();
}

// Weight of node i is (i+1)^(-1/(gamma-1)); the CDF is kept in 63-bit fixed
// point so host and device draw the same endpoints.
void chunglu_cdf(uint32_t n, double gamma, std::vector<uint64_t>& cdf) {
  const double e = -1.0 / (gamma - 1.0);
  double total = 0.0;
  for (uint32_t i = 0; i < n; i++) total += std::pow((double)i + 1.0, e);
  double acc = 0.0;
  const double scale = 9223372036854775808.0 / total;
  cdf.resize(n);
  for (uint32_t i = 0; i < n; i++) {
    acc += std::pow((double)i + 1.0, e);
    const double c = acc * scale;
    cdf[i] = c >= 9223372036854775808.0 ? (1ull << 63) : (uint64_t)c;
  }
  cdf[n - 1] = 1ull << 63;
}

void gen_chunglu(cudaStream_t s, uint64_t seed, uint32_t n, uint64_t m, double gamma, uint32_t* u, uint32_t* v) {
  EH_REQUIRE(n > 0 && gamma > 1.0, EH_ERR_INVALID, "Chung-Lu needs n > 0 and gamma > 1");
  if (!m) return;
  std::vector<uint64_t> h;
  chunglu_cdf(n, gamma, h);
  DevBuf<uint64_t> d(n, s);
  EH_CUDA(cudaMemcpyAsync(d.p, h.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  gen_chunglu_kernel<<<num_sms() * 8, 256, 0, s>>>(splitmix64(seed), n, m, d.p, u, v);
  EH_CHECK_LAUNCH();
  EH_CUDA(cudaStreamSynchronize(s));  // host cdf vector goes out of scope
}

// ----------------------------------------------------------- preprocessing
// A self-loop gets the key with all 2b bits set: lo == hi == 2^b - 1 is
// never a kept edge, and the key sorts last.
__global__ void canon_kernel(const uint32_t* __restrict__ u, const uint32_t* __restrict__ v, uint64_t m, int b,
                             uint64_t* __restrict__ keys) {
  const uint64_t sentinel = (1ull << (2 * b)) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t x = u[i], y = v[i];
    const uint32_t lo = min(x, y), hi = max(x, y);
    keys[i] = (x == y) ? sentinel : (((uint64_t)lo << b) | hi);
  }
}
__global__ void degree_kernel(const uint64_t* __restrict__ keys, uint64_t e, int b, uint32_t* __restrict__ deg) {
  const uint64_t mask = (1ull << b) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < e; i += (uint64_t)gridDim.x * blockDim.x) {
    atomicAdd(&deg[keys[i] >> b], 1u);
    atomicAdd(&deg[keys[i] & mask], 1u);
  }
}
__global__ void nonzero_flag_kernel(const uint32_t* __restrict__ deg, uint64_t n, uint32_t* __restrict__ flag) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    flag[i] = deg[i] ? 1u : 0u;
}
__global__ void degree_key_kernel(const uint32_t* __restrict__ deg, uint64_t n, const uint32_t* __restrict__ pos,
                                  int b, uint64_t* __restrict__ keys) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (deg[i]) keys[pos[i]] = ((uint64_t)deg[i] << b) | i;
}
__global__ void rank_kernel(const uint64_t* __restrict__ keys, uint64_t nn, int b, uint32_t* __restrict__ newid) {
  const uint64_t mask = (1ull << b) - 1;
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nn; r += (uint64_t)gridDim.x * blockDim.x)
    newid[keys[r] & mask] = (uint32_t)r;
}
__global__ void relabel_kernel(const uint64_t* __restrict__ keys, uint64_t e, int b,
                               const uint32_t* __restrict__ newid, int b2, int symmetric,
                               uint64_t* __restrict__ out) {
  const uint64_t mask = (1ull << b) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < e; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t x = newid[keys[i] >> b], y = newid[keys[i] & mask];
    const uint32_t lo = min(x, y), hi = max(x, y);
    if (symmetric) {
      out[2 * i] = ((uint64_t)lo << b2) | hi;
      out[2 * i + 1] = ((uint64_t)hi << b2) | lo;
    } else {
      out[i] = ((uint64_t)lo << b2) | hi;
    }
  }
}
__global__ void split_kernel(const uint64_t* __restrict__ keys, uint64_t n, int b, uint32_t* __restrict__ src,
                             uint32_t* __restrict__ dst) {
  const uint64_t mask = (1ull << b) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    src[i] = (uint32_t)(keys[i] >> b);
    dst[i] = (uint32_t)(keys[i] & mask);
  }
}

void preprocess(cudaStream_t s, const uint32_t* u, const uint32_t* v, uint64_t m, int symmetric, DevBuf<uint32_t>& src,
                DevBuf<uint32_t>& dst, uint64_t* rows_out, uint32_t* nodes_out) {
  const int grid = num_sms() * 8;
  *rows_out = 0;
  *nodes_out = 0;
  if (m == 0) return;
  const uint32_t maxid = std::max(max_u32(u, m, s), max_u32(v, m, s));
  const int b = bits_for(maxid);
  // 1. canonical undirected keys, sorted and deduplicated
  DevBuf<uint64_t> keys(m, s), tmp(m, s);
  canon_kernel<<<grid, 256, 0, s>>>(u, v, m, b, keys.p);
  EH_CHECK_LAUNCH();
  radix_sort_u64(keys.p, tmp.p, m, 2 * b, s);
  uint64_t e = unique_sorted_u64(keys.p, tmp.p, m, s);
  if (e) {  // drop the self-loop key
    uint64_t last = 0;
    EH_CUDA(cudaMemcpyAsync(&last, tmp.p + e - 1, 8, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
    if (last == (1ull << (2 * b)) - 1) e--;
  }
  if (e == 0) return;
  // 2. degrees, 3. relabel nodes of degree > 0 by (degree, id)
  const uint64_t nid = (uint64_t)maxid + 1;
  DevBuf<uint32_t> deg(nid, s), pos(nid, s), nn_dev(1, s);
  EH_CUDA(cudaMemsetAsync(deg.p, 0, nid * 4, s));
  degree_kernel<<<grid, 256, 0, s>>>(tmp.p, e, b, deg.p);
  EH_CHECK_LAUNCH();
  nonzero_flag_kernel<<<grid, 256, 0, s>>>(deg.p, nid, pos.p);
  EH_CHECK_LAUNCH();
  exclusive_scan<uint32_t>(pos.p, pos.p, nid, nn_dev.p, s);
  uint32_t nn = 0;
  EH_CUDA(cudaMemcpyAsync(&nn, nn_dev.p, 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  {
    DevBuf<uint64_t> dk(nn, s), dt(nn, s);
    degree_key_kernel<<<grid, 256, 0, s>>>(deg.p, nid, pos.p, b, dk.p);
    EH_CHECK_LAUNCH();
    const uint32_t maxdeg = max_u32(deg.p, nid, s);
    radix_sort_u64(dk.p, dt.p, nn, b + bits_for(maxdeg), s);
    rank_kernel<<<grid, 256, 0, s>>>(dk.p, nn, b, deg.p /* reused as newid */);
    EH_CHECK_LAUNCH();
  }
  // 4. orient (or symmetrise) in the new ids and sort by (src, dst)
  const int b2 = bits_for(nn ? nn - 1 : 0);
  const uint64_t rows = symmetric ? 2 * e : e;
  DevBuf<uint64_t> ok(rows, s), ot(rows, s);
  relabel_kernel<<<grid, 256, 0, s>>>(tmp.p, e, b, deg.p, b2, symmetric, ok.p);
  EH_CHECK_LAUNCH();
  keys.release();
  tmp.release();
  radix_sort_u64(ok.p, ot.p, rows, 2 * b2, s);
  src.alloc(rows, s);
  dst.alloc(rows, s);
  split_kernel<<<grid, 256, 0, s>>>(ok.p, rows, b2, src.p, dst.p);
  EH_CHECK_LAUNCH();
  EH_CUDA(cudaStreamSynchronize(s));
  *rows_out = rows;
  *nodes_out = nn;
}

}  // namespace eh
