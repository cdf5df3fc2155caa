// Dictionary encoding on the device.
//
// Reference: Encoding<T> (storage_engine/include/Encoding.hpp,
// storage_engine/src/Encoding.cpp:21-48), used by the loader
// (createDB.scala:242-270): build() inserts the distinct values of every
// column that shares the encoding into a std::set and numbers them in
// ascending value order (key 0 = smallest value); encode_column() maps each
// value through value_to_key.at() (an absent value throws); key_to_value
// decodes.  Instantiated there for uint32_t, int, long, float, std::string;
// strings stay on the host, the four numeric types are encoded here.
//
// Device form: every value becomes a 64-bit key whose unsigned order is the
// type's order (sign bit flipped for int/long, the usual sign-magnitude flip
// for float with -0.0 folded into +0.0, which std::set<float> treats as
// equal); the keys of all columns are radix-sorted and de-duplicated into
// the dictionary.  Encoding a column is a lookup per value: a dense map
// (value - min -> key) when the value span is at most a few times the number
// of distinct values, else a binary search in the sorted dictionary.
#include <algorithm>

#include "eh_internal.cuh"

struct eh_encoding {
  eh_context* ctx = nullptr;
  int type = EH_VALUE_UINT32;
  uint64_t n_distinct = 0;
  eh::DevBuf<uint64_t> dict;      // sorted distinct order keys; key k = dict[k]
  eh::DevBuf<uint32_t> dense;     // dense[x - lo] = key of order key x, or kNone
  uint64_t lo = 0, span = 0;      // dense map domain [lo, lo + span)
};

namespace eh {

constexpr uint32_t kNone = 0xffffffffu;

static int value_bytes(int type) { return (type == EH_VALUE_INT64) ? 8 : 4; }

__device__ __forceinline__ uint64_t order_key(const void* col, uint64_t i, int type, unsigned int* bad) {
  switch (type) {
    case EH_VALUE_UINT32:
      return static_cast<const uint32_t*>(col)[i];
    case EH_VALUE_INT32:
      return static_cast<const uint32_t*>(col)[i] ^ 0x80000000u;
    case EH_VALUE_INT64:
      return static_cast<const uint64_t*>(col)[i] ^ 0x8000000000000000ull;
    default: {  // EH_VALUE_FLOAT32
      uint32_t b = static_cast<const uint32_t*>(col)[i];
      if ((b & 0x7fffffffu) > 0x7f800000u) {  // NaN: no order in std::set<float>
        atomicOr(bad, 1u);
        return 0;
      }
      if (b == 0x80000000u) b = 0;  // -0.0 == +0.0
      return (b & 0x80000000u) ? (uint64_t)(~b) : (uint64_t)(b | 0x80000000u);
    }
  }
}

__device__ __forceinline__ void store_value(void* out, uint64_t i, int type, uint64_t k) {
  switch (type) {
    case EH_VALUE_UINT32:
      static_cast<uint32_t*>(out)[i] = (uint32_t)k;
      break;
    case EH_VALUE_INT32:
      static_cast<uint32_t*>(out)[i] = (uint32_t)k ^ 0x80000000u;
      break;
    case EH_VALUE_INT64:
      static_cast<uint64_t*>(out)[i] = k ^ 0x8000000000000000ull;
      break;
    default: {
      const uint32_t b = (uint32_t)k;
      static_cast<uint32_t*>(out)[i] = (b & 0x80000000u) ? (b & 0x7fffffffu) : ~b;
    }
  }
}

__global__ void order_keys_kernel(const void* __restrict__ col, uint64_t n, int type, uint64_t* __restrict__ keys,
                                  unsigned int* __restrict__ bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    keys[i] = order_key(col, i, type, bad);
}

__global__ void minmax_u64_kernel(const uint64_t* __restrict__ a, uint64_t n, unsigned long long* __restrict__ mm) {
  unsigned long long lo = ~0ull, hi = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    lo = min(lo, (unsigned long long)a[i]);
    hi = max(hi, (unsigned long long)a[i]);
  }
  for (int o = 16; o; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(kFull, lo, o));
    hi = max(hi, __shfl_xor_sync(kFull, hi, o));
  }
  if (lane_id() == 0) {
    atomicMin(&mm[0], lo);
    atomicMax(&mm[1], hi);
  }
}

__global__ void dense_fill_kernel(const uint64_t* __restrict__ dict, uint64_t d, uint64_t lo,
                                  uint32_t* __restrict__ dense) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < d; k += (uint64_t)gridDim.x * blockDim.x)
    dense[dict[k] - lo] = (uint32_t)k;
}

// value_to_key.at(): dense map or binary search; an absent value sets *bad
__global__ void encode_kernel(const void* __restrict__ col, uint64_t n, int type, const uint64_t* __restrict__ dict,
                              uint64_t d, const uint32_t* __restrict__ dense, uint64_t lo, uint64_t span,
                              uint32_t* __restrict__ keys, unsigned int* __restrict__ bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t x = order_key(col, i, type, bad + 1);
    uint32_t k = kNone;
    if (dense) {
      if (x >= lo && x - lo < span) k = __ldg(dense + (x - lo));
    } else {
      uint64_t a = 0, b = d;
      while (a < b) {
        const uint64_t m = (a + b) >> 1;
        if (__ldg(dict + m) < x) a = m + 1; else b = m;
      }
      if (a < d && __ldg(dict + a) == x) k = (uint32_t)a;
    }
    if (k == kNone) atomicOr(bad, 1u);
    keys[i] = k;
  }
}

__global__ void decode_kernel(const uint32_t* __restrict__ keys, uint64_t n, int type,
                              const uint64_t* __restrict__ dict, uint64_t d, void* __restrict__ out,
                              unsigned int* __restrict__ bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    if (k >= d) {
      atomicOr(bad, 1u);
      store_value(out, i, type, 0);
      continue;
    }
    store_value(out, i, type, __ldg(dict + k));
  }
}

static void check_type(int type) {
  EH_REQUIRE(type == EH_VALUE_UINT32 || type == EH_VALUE_INT32 || type == EH_VALUE_INT64 ||
                 type == EH_VALUE_FLOAT32,
             EH_ERR_INVALID, "unknown value type");
}

// a device copy of a column given on the host or the device
static const void* device_column(eh_context* ctx, const void* col, uint64_t n, int type, int on_device,
                                 DevBuf<unsigned char>& stage) {
  if (on_device || !n) return col;
  const size_t bytes = n * (size_t)value_bytes(type);
  stage.alloc(bytes, ctx->stream);
  EH_CUDA(cudaMemcpyAsync(stage.p, col, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return stage.p;
}

static int bits_for_u64(uint64_t maxv) {
  int b = 1;
  while (b < 64 && (maxv >> b)) b++;
  return b;
}

eh_encoding* encoding_build(eh_context* ctx, const void* const* cols, const uint64_t* n_rows, uint32_t n_cols,
                            int type, int on_device) {
  check_type(type);
  cudaStream_t s = ctx->stream;
  const int grid = num_sms() * 8;
  uint64_t total = 0;
  for (uint32_t c = 0; c < n_cols; c++) {
    EH_REQUIRE(n_rows[c] == 0 || cols[c] != nullptr, EH_ERR_INVALID, "null column");
    total += n_rows[c];
  }
  auto* e = new eh_encoding();
  e->ctx = ctx;
  e->type = type;
  try {
    if (total) {
      DevBuf<uint64_t> keys(total, s), tmp(total, s);
      DevBuf<unsigned int> bad(1, s);
      EH_CUDA(cudaMemsetAsync(bad.p, 0, 4, s));
      uint64_t o = 0;
      for (uint32_t c = 0; c < n_cols; c++) {
        if (!n_rows[c]) continue;
        DevBuf<unsigned char> stage;
        const void* dc = device_column(ctx, cols[c], n_rows[c], type, on_device, stage);
        order_keys_kernel<<<grid, 256, 0, s>>>(dc, n_rows[c], type, keys.p + o, bad.p);
        EH_CHECK_LAUNCH();
        o += n_rows[c];
      }
      DevBuf<unsigned long long> mm(2, s);
      const unsigned long long init[2] = {~0ull, 0ull};
      EH_CUDA(cudaMemcpyAsync(mm.p, init, 16, cudaMemcpyHostToDevice, s));
      minmax_u64_kernel<<<grid, 256, 0, s>>>(keys.p, total, mm.p);
      EH_CHECK_LAUNCH();
      unsigned long long h[2];
      unsigned int hb = 0;
      EH_CUDA(cudaMemcpyAsync(h, mm.p, 16, cudaMemcpyDeviceToHost, s));
      EH_CUDA(cudaMemcpyAsync(&hb, bad.p, 4, cudaMemcpyDeviceToHost, s));
      EH_CUDA(cudaStreamSynchronize(s));
      EH_REQUIRE(hb == 0, EH_ERR_INVALID, "NaN in a float column (no order to encode it by)");
      const uint64_t lo = h[0], hi = h[1];
      radix_sort_u64(keys.p, tmp.p, total, bits_for_u64(hi), s);
      const uint64_t d = unique_sorted_u64(keys.p, tmp.p, total, s);
      EH_REQUIRE(d <= 0xfffffffeull, EH_ERR_UNSUPPORTED, "more than 2^32 - 2 distinct values");
      e->n_distinct = d;
      e->dict.alloc(d, s);
      EH_CUDA(cudaMemcpyAsync(e->dict.p, tmp.p, d * 8, cudaMemcpyDeviceToDevice, s));
      const uint64_t span = hi - lo + 1;  // hi >= lo; span 0 means the full 2^64 range
      if (span != 0 && span <= 4 * d + (1ull << 20)) {
        e->lo = lo;
        e->span = span;
        e->dense.alloc(span, s);
        EH_CUDA(cudaMemsetAsync(e->dense.p, 0xff, span * 4, s));
        dense_fill_kernel<<<grid, 256, 0, s>>>(e->dict.p, d, lo, e->dense.p);
        EH_CHECK_LAUNCH();
      }
      EH_CUDA(cudaStreamSynchronize(s));
    }
  } catch (...) {
    delete e;
    throw;
  }
  return e;
}

void encoding_encode(eh_context* ctx, const eh_encoding* e, const void* col, uint64_t n, int on_device,
                     uint32_t* keys) {
  cudaStream_t s = ctx->stream;
  if (!n) return;
  DevBuf<unsigned char> stage;
  const void* dc = device_column(ctx, col, n, e->type, on_device, stage);
  DevBuf<uint32_t> kout;
  uint32_t* dk = keys;
  if (!on_device) {
    kout.alloc(n, s);
    dk = kout.p;
  }
  DevBuf<unsigned int> bad(2, s);
  EH_CUDA(cudaMemsetAsync(bad.p, 0, 8, s));
  encode_kernel<<<num_sms() * 8, 256, 0, s>>>(dc, n, e->type, e->dict.p, e->n_distinct, e->dense.p, e->lo, e->span,
                                              dk, bad.p);
  EH_CHECK_LAUNCH();
  unsigned int hb[2];
  EH_CUDA(cudaMemcpyAsync(hb, bad.p, 8, cudaMemcpyDeviceToHost, s));
  if (!on_device) EH_CUDA(cudaMemcpyAsync(keys, dk, n * 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  EH_REQUIRE(hb[1] == 0, EH_ERR_INVALID, "NaN in a float column");
  EH_REQUIRE(hb[0] == 0, EH_ERR_INVALID, "value not in the encoding (value_to_key.at)");
}

void encoding_decode(eh_context* ctx, const eh_encoding* e, const uint32_t* keys, uint64_t n, int on_device,
                     void* values) {
  cudaStream_t s = ctx->stream;
  if (!n) return;
  const size_t vb = (size_t)value_bytes(e->type);
  DevBuf<uint32_t> kin;
  const uint32_t* dk = keys;
  if (!on_device) {
    kin.alloc(n, s);
    EH_CUDA(cudaMemcpyAsync(kin.p, keys, n * 4, cudaMemcpyHostToDevice, s));
    dk = kin.p;
  }
  DevBuf<unsigned char> vout;
  void* dv = values;
  if (!on_device) {
    vout.alloc(n * vb, s);
    dv = vout.p;
  }
  DevBuf<unsigned int> bad(1, s);
  EH_CUDA(cudaMemsetAsync(bad.p, 0, 4, s));
  decode_kernel<<<num_sms() * 8, 256, 0, s>>>(dk, n, e->type, e->dict.p, e->n_distinct, dv, bad.p);
  EH_CHECK_LAUNCH();
  unsigned int hb = 0;
  EH_CUDA(cudaMemcpyAsync(&hb, bad.p, 4, cudaMemcpyDeviceToHost, s));
  if (!on_device) EH_CUDA(cudaMemcpyAsync(values, dv, n * vb, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  EH_REQUIRE(hb == 0, EH_ERR_INVALID, "key out of range (key_to_value)");
}

uint64_t encoding_size(const eh_encoding* e) { return e->n_distinct; }
eh_context* encoding_ctx(const eh_encoding* e) { return e->ctx; }

void encoding_free(eh_encoding* e) {
  cudaSetDevice(e->ctx->device);
  cudaStream_t s = e->ctx->stream;
  delete e;
  cudaStreamSynchronize(s);
}

// key_to_value as host values (the table Encoding::to_binary writes)
__global__ void dict_values_kernel(const uint64_t* __restrict__ dict, uint64_t n, int type, void* __restrict__ out) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
    store_value(out, k, type, dict[k]);
}

void encoding_values(eh_context* ctx, const eh_encoding* e, void* values, uint64_t cap) {
  const uint64_t n = std::min<uint64_t>(cap, e->n_distinct);
  if (!n) return;
  cudaStream_t s = ctx->stream;
  const size_t vb = (size_t)value_bytes(e->type);
  DevBuf<unsigned char> out(n * vb, s);
  dict_values_kernel<<<num_sms() * 4, 256, 0, s>>>(e->dict.p, n, e->type, out.p);
  EH_CHECK_LAUNCH();
  EH_CUDA(cudaMemcpyAsync(values, out.p, n * vb, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
}

}  // namespace eh
