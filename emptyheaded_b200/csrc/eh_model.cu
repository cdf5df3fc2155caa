// Learned layout policy: a small fp32 MLP trained on the device.
//
// The reference picks each set's layout with a density threshold
// (common::is_sparse, utils/common.hpp:60-66; hybrid::get_type,
// layouts/hybrid.hpp:103-111).  Here the engine logs, per work item, the
// device time it spent with each staged set under the layout it had
// (eh_timing_records); a small MLP is trained on those records to predict
// the time of a set under each layout, and EH_POLICY_LEARNED gives every
// set the layout with the lowest predicted time.  The density rule stays
// as the fallback (sets the model cannot place, memory cap) and as the
// point of comparison in the tests.  Layouts change speed only: every layout holds the
// same elements, so counts are identical.
//
// Network: widths d0 -> d1 -> ... -> dL, ReLU between layers, linear
// output; loss = mean over the batch of 0.5 * sum (y_hat - y)^2; plain SGD.
// Sizes are tiny (d <= 64), so the kernels are straightforward fp32 loops:
// there is no dense contraction large enough for tensor cores.
#include <algorithm>
#include <cmath>

#include "eh_internal.cuh"

namespace eh {

constexpr int kFeat = 6;  // features fed to the layout cost model (see model_features)

// ------------------------------------------------------------- kernels
// z[b][o] = bias[o] + sum_i W[o][i] * x[b][i]; a = relu(z) unless last
__global__ void mlp_fwd_kernel(const float* __restrict__ W, const float* __restrict__ bias,
                               const float* __restrict__ x, int din, int dout, int batch, int relu,
                               float* __restrict__ z, float* __restrict__ a) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= batch * dout) return;
  const int b = idx / dout, o = idx % dout;
  float s = bias[o];
  const float* xr = x + (size_t)b * din;
  const float* wr = W + (size_t)o * din;
  for (int i = 0; i < din; i++) s = fmaf(wr[i], xr[i], s);
  z[idx] = s;
  a[idx] = (relu && s < 0.f) ? 0.f : s;
}

// dz[b][o] = (y_hat - y) / batch ; per-sample loss 0.5 * (y_hat - y)^2
__global__ void mlp_loss_kernel(const float* __restrict__ yhat, const float* __restrict__ y, int n, float inv_batch,
                                float* __restrict__ dz, float* __restrict__ loss) {
  float l = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float d = yhat[i] - y[i];
    dz[i] = d * inv_batch;
    l += 0.5f * d * d;
  }
  l = warp_sum(l);
  if (lane_id() == 0) atomicAdd(loss, l * inv_batch);
}

// dW[o][i] = sum_b dz[b][o] * x[b][i]; db[o] = sum_b dz[b][o]
__global__ void mlp_wgrad_kernel(const float* __restrict__ dz, const float* __restrict__ x, int din, int dout,
                                 int batch, float* __restrict__ gW, float* __restrict__ gb) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < dout * din) {
    const int o = idx / din, i = idx % din;
    float s = 0.f;
    for (int b = 0; b < batch; b++) s = fmaf(dz[(size_t)b * dout + o], x[(size_t)b * din + i], s);
    gW[idx] = s;
  } else if (idx < dout * din + dout) {
    const int o = idx - dout * din;
    float s = 0.f;
    for (int b = 0; b < batch; b++) s += dz[(size_t)b * dout + o];
    gb[o] = s;
  }
}

// dx[b][i] = (z_in[b][i] < 0 ? 0 : sum_o W[o][i] * dz[b][o])
__global__ void mlp_xgrad_kernel(const float* __restrict__ W, const float* __restrict__ dz,
                                 const float* __restrict__ zin, int din, int dout, int batch,
                                 float* __restrict__ dx) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= batch * din) return;
  const int b = idx / din, i = idx % din;
  if (zin[idx] < 0.f) { dx[idx] = 0.f; return; }
  float s = 0.f;
  for (int o = 0; o < dout; o++) s = fmaf(W[(size_t)o * din + i], dz[(size_t)b * dout + o], s);
  dx[idx] = s;
}

__global__ void sgd_kernel(float* __restrict__ p, const float* __restrict__ g, size_t n, float lr) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    p[i] -= lr * g[i];
}

// ------------------------------------------------------------- host side
static void check_model(const eh_model* m) {
  EH_REQUIRE(m && m->n_layers > 0, EH_ERR_INVALID, "invalid model");
}

// forward over a device batch; keeps z and a per layer in `ws`
struct Workspace {
  std::vector<DevBuf<float>> z, a;  // layer l output (l = 1..L); a[0] = input
};

static void forward(eh_model* m, const float* dx, int batch, Workspace& ws, cudaStream_t s) {
  const int L = m->n_layers;
  ws.z.resize(L + 1);
  ws.a.resize(L + 1);
  const float* in = dx;
  for (int l = 0; l < L; l++) {
    const int din = m->dims[l], dout = m->dims[l + 1];
    ws.z[l + 1].alloc((size_t)batch * dout, s);
    ws.a[l + 1].alloc((size_t)batch * dout, s);
    const float* W = m->params.p + m->w_off[l];
    const float* b = W + (size_t)dout * din;
    const int n = batch * dout;
    mlp_fwd_kernel<<<(n + 255) / 256, 256, 0, s>>>(W, b, in, din, dout, batch, l + 1 < L ? 1 : 0, ws.z[l + 1].p,
                                                  ws.a[l + 1].p);
    EH_CHECK_LAUNCH();
    in = ws.a[l + 1].p;
  }
}

// loss and gradient into m->grads for a device batch
static float loss_grad(eh_model* m, const float* dx, const float* dy, int batch, cudaStream_t s) {
  const int L = m->n_layers;
  Workspace ws;
  forward(m, dx, batch, ws, s);
  const int dL = m->dims[L];
  DevBuf<float> dz((size_t)batch * dL, s), loss(1, s);
  EH_CUDA(cudaMemsetAsync(loss.p, 0, 4, s));
  mlp_loss_kernel<<<std::max(1, std::min(1024, (batch * dL + 255) / 256)), 256, 0, s>>>(
      ws.a[L].p, dy, batch * dL, 1.f / (float)batch, dz.p, loss.p);
  EH_CHECK_LAUNCH();
  for (int l = L - 1; l >= 0; l--) {
    const int din = m->dims[l], dout = m->dims[l + 1];
    const float* x = l == 0 ? dx : ws.a[l].p;
    float* gW = m->grads.p + m->w_off[l];
    float* gb = gW + (size_t)dout * din;
    const int n = dout * din + dout;
    mlp_wgrad_kernel<<<(n + 255) / 256, 256, 0, s>>>(dz.p, x, din, dout, batch, gW, gb);
    EH_CHECK_LAUNCH();
    if (l > 0) {
      DevBuf<float> dprev((size_t)batch * din, s);
      const float* W = m->params.p + m->w_off[l];
      mlp_xgrad_kernel<<<(batch * din + 255) / 256, 256, 0, s>>>(W, dz.p, ws.z[l].p, din, dout, batch, dprev.p);
      EH_CHECK_LAUNCH();
      dz = std::move(dprev);
    }
  }
  float h = 0.f;
  EH_CUDA(cudaMemcpyAsync(&h, loss.p, 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
  return h;
}

// ------------------------------------------------------ layout chooser
// Features of set b for layout choice (all log-scaled, fp32):
//   log1p(len), log1p(range), density = len / (range + 1),
//   log1p(pairs probed against b by the triangle plan), layout one-hot (2)
// The model predicts log1p(device ns) of staging + probing b's work.
__device__ __forceinline__ void model_features(const TrieView& t, uint32_t b, uint64_t pairs, int layout, float* f) {
  const uint64_t s0 = t.off[b];
  const uint32_t len = (uint32_t)(t.off[b + 1] - s0);
  const uint32_t range = len ? t.vals[s0 + len - 1] - t.vals[s0] : 0;
  f[0] = log1pf((float)len);
  f[1] = log1pf((float)range);
  f[2] = (float)len / ((float)range + 1.f);
  f[3] = log1pf((float)pairs);
  f[4] = layout == EH_LAYOUT_RANGE_BITSET ? 1.f : 0.f;
  f[5] = layout == EH_LAYOUT_BLOCK_BITSET ? 1.f : 0.f;
}

// per set: predicted cost under each candidate layout, pick the minimum.
// A range bitset is admitted only up to 16 words per element plus 64 (and
// the optional absolute per-set cap), which bounds bitset memory to about
// 48x the set's uint bytes in the worst case.
__global__ void choose_kernel(TrieView t, const uint64_t* __restrict__ rev_off, const uint64_t* __restrict__ wpre,
                              const float* __restrict__ params, const int* __restrict__ dims, int L,
                              const int* __restrict__ woff, uint64_t max_words_per_set, float log_keep,
                              uint8_t* __restrict__ layout, float* __restrict__ pred) {
  float buf0[64], buf1[64];
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < t.n_head; b += gridDim.x * blockDim.x) {
    const uint64_t s0 = t.off[b];
    const uint32_t len = (uint32_t)(t.off[b + 1] - s0);
    if (pred) pred[b] = 0.f;
    if (!len) continue;
    const uint64_t pairs = wpre[rev_off[b + 1]] - wpre[rev_off[b]];
    if (!pairs) continue;  // never staged: keep the fallback layout
    const uint32_t words = (t.vals[s0 + len - 1] >> 6) - (t.vals[s0] >> 6) + 1;
    float best = 3.4e38f;
    const int h = layout[b];  // the density rule's layout: the fallback
    int best_l = h;
    float yh = 3.4e38f;
    const int cands[3] = {EH_LAYOUT_UINTEGER, EH_LAYOUT_RANGE_BITSET, EH_LAYOUT_BLOCK_BITSET};
    for (int c = 0; c < 3; c++) {
      const int l = cands[c];
      if (l == EH_LAYOUT_RANGE_BITSET &&
          ((uint64_t)words > 16ull * len + 64 || (max_words_per_set && words > max_words_per_set)))
        continue;
      model_features(t, b, pairs, l, buf0);
      float* in = buf0;
      float* out = buf1;
      for (int k = 0; k < L; k++) {
        const int din = dims[k], dout = dims[k + 1];
        const float* W = params + woff[k];
        const float* bias = W + dout * din;
        for (int o = 0; o < dout; o++) {
          float s = bias[o];
          for (int i = 0; i < din; i++) s = fmaf(W[o * din + i], in[i], s);
          out[o] = (k + 1 < L && s < 0.f) ? 0.f : s;
        }
        float* tmp = in;
        in = out;
        out = tmp;
      }
      if (l == h) yh = in[0];
      if (in[0] < best) {
        best = in[0];
        best_l = l;
      }
    }
    if (best_l != h && !(best < yh + log_keep)) {  // leave the rule only for a predicted gain of min_gain
      best_l = h;
      best = yh;
    }
    layout[b] = (uint8_t)best_l;
    if (pred) pred[b] = fmaxf(expm1f(best), 1.f);  // the model predicts log1p(cycles)
  }
}

// choose_kernel for the default network (6 -> 32 -> 32 -> 1): the weights
// live in shared memory (broadcast reads), the first hidden layer in
// registers, and the second is folded into the output one unit at a time, so
// no activation array touches local memory.
constexpr int kH = 32;
constexpr int kFixedParams = kH * kFeat + kH + kH * kH + kH + kH + 1;

__device__ __forceinline__ float mlp_fixed(const float* __restrict__ P, float f0, float f1, float f2, float f3,
                                           float f4, float f5) {
  const float* W0 = P;
  const float* b0 = W0 + kH * kFeat;
  const float* W1 = b0 + kH;
  const float* b1 = W1 + kH * kH;
  const float* W2 = b1 + kH;
  float h1[kH];
#pragma unroll
  for (int o = 0; o < kH; o++) {
    const float* w = W0 + o * kFeat;
    float z = b0[o];
    z = fmaf(w[0], f0, z);
    z = fmaf(w[1], f1, z);
    z = fmaf(w[2], f2, z);
    z = fmaf(w[3], f3, z);
    z = fmaf(w[4], f4, z);
    z = fmaf(w[5], f5, z);
    h1[o] = fmaxf(z, 0.f);
  }
  float y = W2[kH];
#pragma unroll 2
  for (int o = 0; o < kH; o++) {
    const float* w = W1 + o * kH;
    float z = b1[o];
#pragma unroll
    for (int i = 0; i < kH; i++) z = fmaf(w[i], h1[i], z);
    y = fmaf(W2[o], fmaxf(z, 0.f), y);
  }
  return y;
}

__global__ void __launch_bounds__(128) choose_fixed_kernel(TrieView t, const uint64_t* __restrict__ rev_off,
                                                           const uint64_t* __restrict__ wpre,
                                                           const float* __restrict__ params,
                                                           uint64_t max_words_per_set, float log_keep,
                                                           uint8_t* __restrict__ layout, float* __restrict__ pred) {
  __shared__ float P[kFixedParams];
  for (int i = threadIdx.x; i < kFixedParams; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < t.n_head; b += gridDim.x * blockDim.x) {
    if (pred) pred[b] = 0.f;
    const uint64_t s0 = t.off[b];
    const uint32_t len = (uint32_t)(t.off[b + 1] - s0);
    if (!len) continue;
    const uint64_t pairs = wpre[rev_off[b + 1]] - wpre[rev_off[b]];
    if (!pairs) continue;  // never staged: keep the fallback layout
    const uint32_t first = t.vals[s0], last = t.vals[s0 + len - 1];
    const uint32_t words = (last >> 6) - (first >> 6) + 1;
    const uint32_t range = last - first;
    // the features of model_features; the layout one-hot varies per candidate
    const float f0 = log1pf((float)len), f1 = log1pf((float)range), f2 = (float)len / ((float)range + 1.f),
                f3 = log1pf((float)pairs);
    const int h = layout[b];  // the density rule's layout: the fallback
    const float yu = mlp_fixed(P, f0, f1, f2, f3, 0.f, 0.f);  // uint
    const bool bits_ok = !((uint64_t)words > 16ull * len + 64 || (max_words_per_set && words > max_words_per_set));
    const float yb = bits_ok ? mlp_fixed(P, f0, f1, f2, f3, 1.f, 0.f) : 3.4e38f;  // range bitset
    const float yk = mlp_fixed(P, f0, f1, f2, f3, 0.f, 1.f);                      // block bitset
    float best = yu;
    int best_l = EH_LAYOUT_UINTEGER;
    if (yb < best) {
      best = yb;
      best_l = EH_LAYOUT_RANGE_BITSET;
    }
    if (yk < best) {
      best = yk;
      best_l = EH_LAYOUT_BLOCK_BITSET;
    }
    // leave the rule's layout only for a predicted gain of at least min_gain
    const float yh = h == EH_LAYOUT_RANGE_BITSET ? yb : (h == EH_LAYOUT_BLOCK_BITSET ? yk : yu);
    if (best_l != h && !(best < yh + log_keep)) {
      best_l = h;
      best = yh;
    }
    layout[b] = (uint8_t)best_l;
    if (pred) pred[b] = fmaxf(expm1f(best), 1.f);  // the model predicts log1p(cycles)
  }
}

void model_choose_layouts(eh_context* ctx, const eh_model* m, const eh_trie* t, uint64_t max_bitset_bytes,
                          float min_gain, uint8_t* layout_dev, float* pred_dev) {
  cudaStream_t s = ctx->stream;
  // the model predicts log1p(cycles): a gain g is a difference of log(1 - g)
  const float g = min_gain == 0.f ? 0.1f : std::min(std::max(min_gain, 0.f), 0.99f);
  const float log_keep = logf(1.f - g);
  EH_REQUIRE(m->dims[0] == kFeat && m->dims[m->n_layers] == 1, EH_ERR_INVALID,
             "layout model must map 6 features to 1 output");
  EH_REQUIRE(m->max_dim <= 64, EH_ERR_INVALID, "layout model layers must be at most 64 wide");
  if (!t->n_head || !t->rev_entries) return;
  if (m->n_layers == 3 && m->dims[1] == kH && m->dims[2] == kH && (int)m->n_params == kFixedParams) {
    choose_fixed_kernel<<<num_sms() * 4, 128, 0, s>>>(t->view(), t->rev_off.p, t->rev_wpre.p, m->params.p,
                                                      max_bitset_bytes / 12, log_keep, layout_dev, pred_dev);
    EH_CHECK_LAUNCH();
    EH_CUDA(cudaStreamSynchronize(s));
    return;
  }
  std::vector<int> woff(m->n_layers);
  for (int l = 0; l < m->n_layers; l++) woff[l] = (int)m->w_off[l];
  DevBuf<int> ddims(m->n_layers + 1, s), dwoff(m->n_layers, s);
  EH_CUDA(cudaMemcpyAsync(ddims.p, m->dims.data(), (m->n_layers + 1) * 4, cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaMemcpyAsync(dwoff.p, woff.data(), m->n_layers * 4, cudaMemcpyHostToDevice, s));
  choose_kernel<<<num_sms() * 2, 128, 0, s>>>(t->view(), t->rev_off.p, t->rev_wpre.p, m->params.p, ddims.p,
                                               m->n_layers, dwoff.p, max_bitset_bytes / 12, log_keep, layout_dev,
                                               pred_dev);
  EH_CHECK_LAUNCH();
  EH_CUDA(cudaStreamSynchronize(s));
}

// ------------------------------------------------------------ ABI helpers
eh_model* model_create(eh_context* ctx, int n_layers, const int* dims, uint64_t seed) {
  EH_REQUIRE(n_layers >= 1 && n_layers <= 8, EH_ERR_INVALID, "1..8 layers");
  auto* m = new eh_model();
  m->ctx = ctx;
  m->n_layers = n_layers;
  m->dims.assign(dims, dims + n_layers + 1);
  size_t o = 0;
  for (int l = 0; l < n_layers; l++) {
    EH_REQUIRE(dims[l] > 0 && dims[l + 1] > 0 && dims[l] <= 4096 && dims[l + 1] <= 4096, EH_ERR_INVALID,
               "layer widths must be in 1..4096");
    m->w_off.push_back(o);
    o += (size_t)dims[l + 1] * dims[l] + dims[l + 1];
  }
  for (int l = 0; l <= n_layers; l++) m->max_dim = std::max(m->max_dim, dims[l]);
  m->n_params = o;
  cudaStream_t s = ctx->stream;
  m->params.alloc(o, s);
  m->grads.alloc(o, s);
  // He-uniform init from the counter-based generator, biases zero
  std::vector<float> h(o, 0.f);
  const uint64_t sm = splitmix64(seed);
  for (int l = 0; l < n_layers; l++) {
    const float bound = std::sqrt(6.f / (float)dims[l]);
    for (size_t i = 0; i < (size_t)dims[l + 1] * dims[l]; i++) {
      const uint64_t r = rand64(sm, m->w_off[l] + i);
      const float u = (float)(r >> 40) * (1.f / 16777216.f);  // [0,1)
      h[m->w_off[l] + i] = (2.f * u - 1.f) * bound;
    }
  }
  EH_CUDA(cudaMemcpyAsync(m->params.p, h.data(), o * 4, cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaStreamSynchronize(s));
  return m;
}

float model_train(eh_model* m, const float* x, const float* y, uint32_t batch, float lr, uint32_t steps) {
  check_model(m);
  cudaStream_t s = m->ctx->stream;
  const int d0 = m->dims[0], dL = m->dims[m->n_layers];
  DevBuf<float> dx((size_t)batch * d0, s), dy((size_t)batch * dL, s);
  EH_CUDA(cudaMemcpyAsync(dx.p, x, (size_t)batch * d0 * 4, cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaMemcpyAsync(dy.p, y, (size_t)batch * dL * 4, cudaMemcpyHostToDevice, s));
  float loss = 0.f;
  for (uint32_t it = 0; it < steps; it++) {
    loss = loss_grad(m, dx.p, dy.p, (int)batch, s);
    sgd_kernel<<<std::max<size_t>(1, std::min<size_t>(1024, (m->n_params + 255) / 256)), 256, 0, s>>>(
        m->params.p, m->grads.p, m->n_params, lr);
    EH_CHECK_LAUNCH();
  }
  EH_CUDA(cudaStreamSynchronize(s));
  return loss;
}

float model_loss_grad_host(eh_model* m, const float* x, const float* y, uint32_t batch, float* grad) {
  check_model(m);
  cudaStream_t s = m->ctx->stream;
  const int d0 = m->dims[0], dL = m->dims[m->n_layers];
  DevBuf<float> dx((size_t)batch * d0, s), dy((size_t)batch * dL, s);
  EH_CUDA(cudaMemcpyAsync(dx.p, x, (size_t)batch * d0 * 4, cudaMemcpyHostToDevice, s));
  EH_CUDA(cudaMemcpyAsync(dy.p, y, (size_t)batch * dL * 4, cudaMemcpyHostToDevice, s));
  const float loss = loss_grad(m, dx.p, dy.p, (int)batch, s);
  if (grad) {
    EH_CUDA(cudaMemcpyAsync(grad, m->grads.p, m->n_params * 4, cudaMemcpyDeviceToHost, s));
    EH_CUDA(cudaStreamSynchronize(s));
  }
  return loss;
}

void model_predict(eh_model* m, const float* x, uint32_t batch, float* y) {
  check_model(m);
  cudaStream_t s = m->ctx->stream;
  const int d0 = m->dims[0], dL = m->dims[m->n_layers];
  DevBuf<float> dx((size_t)batch * d0, s);
  EH_CUDA(cudaMemcpyAsync(dx.p, x, (size_t)batch * d0 * 4, cudaMemcpyHostToDevice, s));
  Workspace ws;
  forward(m, dx.p, (int)batch, ws, s);
  EH_CUDA(cudaMemcpyAsync(y, ws.a[m->n_layers].p, (size_t)batch * dL * 4, cudaMemcpyDeviceToHost, s));
  EH_CUDA(cudaStreamSynchronize(s));
}

}  // namespace eh
