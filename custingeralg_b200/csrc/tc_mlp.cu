// Learned scheduler: a 3-layer FP32 MLP (features -> 64 -> 64 -> one predicted cost per
// intersection strategy) with hand-written forward, backward and Adam kernels (sm_100a, SIMT:
// the network is far too small for tensor cores to pay).
//
// Input features per sample (float32): log2(1 + d_a), log2(1 + d_b), d_min / d_max and the bin
// id of the degree cell (scaled to [0, 1]). The label is the measured cost of one strategy on
// that bin (log2 of ns per edge), so the loss is a masked MSE on the strategy's output only.
//
// The model only fills the scheduler's per-cell strategy table (argmin of the predicted costs);
// the counts are exact whatever it predicts.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "tc_internal.cuh"

namespace tc {
namespace {

constexpr int kIn = TC_MLP_IN;
constexpr int kHid = TC_MLP_HIDDEN;
constexpr int kOut = TC_MLP_OUT;
constexpr int kTile = 32;  // samples per CTA

// Parameter layout (floats): W1[kHid][kIn] b1[kHid] W2[kHid][kHid] b2[kHid] W3[kOut][kHid] b3[kOut]
constexpr int oW1 = 0;
constexpr int oB1 = oW1 + kHid * kIn;
constexpr int oW2 = oB1 + kHid;
constexpr int oB2 = oW2 + kHid * kHid;
constexpr int oW3 = oB2 + kHid;
constexpr int oB3 = oW3 + kOut * kHid;
constexpr int kParams = oB3 + kOut;
static_assert(kParams == TC_MLP_PARAMS, "parameter count");

struct MlpSmem {
  float p[kParams];
  float x[kTile][kIn];
  float h1[kTile][kHid];
  float h2[kTile][kHid];
  float y[kTile][kOut];
  float g2[kTile][kHid];
  float g1[kTile][kHid];
  float gy[kTile][kOut];
};

// Forward for a tile of samples; one thread per hidden unit (blockDim = kHid).
__device__ void tile_forward(MlpSmem& s, int ns) {
  const int j = threadIdx.x;
  for (int t = 0; t < ns; ++t) {
    float a = s.p[oB1 + j];
#pragma unroll
    for (int k = 0; k < kIn; ++k) a += s.p[oW1 + j * kIn + k] * s.x[t][k];
    s.h1[t][j] = fmaxf(a, 0.f);
  }
  __syncthreads();
  for (int t = 0; t < ns; ++t) {
    float a = s.p[oB2 + j];
    for (int k = 0; k < kHid; ++k) a += s.p[oW2 + j * kHid + k] * s.h1[t][k];
    s.h2[t][j] = fmaxf(a, 0.f);
  }
  __syncthreads();
  for (int idx = j; idx < ns * kOut; idx += kHid) {
    const int t = idx / kOut, o = idx % kOut;
    float a = s.p[oB3 + o];
    for (int k = 0; k < kHid; ++k) a += s.p[oW3 + o * kHid + k] * s.h2[t][k];
    s.y[t][o] = a;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kHid) k_mlp_forward(const float* __restrict__ params, const float* __restrict__ X,
                                                      const int n, float* __restrict__ Y) {
  extern __shared__ __align__(16) unsigned char raw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(raw);
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) s.p[i] = params[i];
  for (int t0 = blockIdx.x * kTile; t0 < n; t0 += gridDim.x * kTile) {
    const int ns = min(kTile, n - t0);
    __syncthreads();
    for (int i = threadIdx.x; i < ns * kIn; i += blockDim.x) s.x[i / kIn][i % kIn] = X[(int64_t)t0 * kIn + i];
    __syncthreads();
    tile_forward(s, ns);
    for (int i = threadIdx.x; i < ns * kOut; i += blockDim.x) Y[(int64_t)t0 * kOut + i] = s.y[i / kOut][i % kOut];
  }
}

// Forward + backward of the masked MSE: loss = mean over samples of (y[strategy] - label)^2.
// Gradients accumulate into grad[] (zeroed by the caller) and the loss sum into loss[0].
__global__ void __launch_bounds__(kHid) k_mlp_backward(const float* __restrict__ params, const float* __restrict__ X,
                                                       const int32_t* __restrict__ strat,
                                                       const float* __restrict__ label, const int n,
                                                       float* __restrict__ grad, float* __restrict__ loss) {
  extern __shared__ __align__(16) unsigned char raw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(raw);
  const int j = threadIdx.x;
  for (int i = j; i < kParams; i += blockDim.x) s.p[i] = params[i];
  const float inv_n = 1.f / (float)max(n, 1);
  // per-thread gradient accumulators for the rows this thread owns
  float gW1[kIn], gb1 = 0.f, gb2 = 0.f;
  float gW2[kHid];
  float gW3[kOut], gb3 = 0.f;
#pragma unroll
  for (int k = 0; k < kIn; ++k) gW1[k] = 0.f;
  for (int k = 0; k < kHid; ++k) gW2[k] = 0.f;
#pragma unroll
  for (int o = 0; o < kOut; ++o) gW3[o] = 0.f;
  float lsum = 0.f;
  for (int t0 = blockIdx.x * kTile; t0 < n; t0 += gridDim.x * kTile) {
    const int ns = min(kTile, n - t0);
    __syncthreads();
    for (int i = j; i < ns * kIn; i += blockDim.x) s.x[i / kIn][i % kIn] = X[(int64_t)t0 * kIn + i];
    __syncthreads();
    tile_forward(s, ns);
    // dL/dy (only the labelled output)
    for (int idx = j; idx < ns * kOut; idx += kHid) {
      const int t = idx / kOut, o = idx % kOut;
      const int st = strat[t0 + t];
      float g = 0.f;
      if (o == st) {
        const float d = s.y[t][o] - label[t0 + t];
        g = 2.f * d * inv_n;
        lsum += d * d;
      }
      s.gy[t][o] = g;
    }
    __syncthreads();
    // layer 3: thread j owns hidden input k = j of W3 (all outputs); b3 by thread o < kOut
    for (int t = 0; t < ns; ++t) {
#pragma unroll
      for (int o = 0; o < kOut; ++o) gW3[o] += s.gy[t][o] * s.h2[t][j];
    }
    if (j < kOut)
      for (int t = 0; t < ns; ++t) gb3 += s.gy[t][j];
    // dL/dh2 (through ReLU)
    for (int t = 0; t < ns; ++t) {
      float a = 0.f;
#pragma unroll
      for (int o = 0; o < kOut; ++o) a += s.p[oW3 + o * kHid + j] * s.gy[t][o];
      s.g2[t][j] = s.h2[t][j] > 0.f ? a : 0.f;
    }
    __syncthreads();
    // layer 2: thread j owns row j of W2
    for (int t = 0; t < ns; ++t) {
      const float g = s.g2[t][j];
      gb2 += g;
      for (int k = 0; k < kHid; ++k) gW2[k] += g * s.h1[t][k];
    }
    // dL/dh1
    for (int t = 0; t < ns; ++t) {
      float a = 0.f;
      for (int k = 0; k < kHid; ++k) a += s.p[oW2 + k * kHid + j] * s.g2[t][k];
      s.g1[t][j] = s.h1[t][j] > 0.f ? a : 0.f;
    }
    __syncthreads();
    // layer 1: thread j owns row j of W1
    for (int t = 0; t < ns; ++t) {
      const float g = s.g1[t][j];
      gb1 += g;
#pragma unroll
      for (int k = 0; k < kIn; ++k) gW1[k] += g * s.x[t][k];
    }
  }
#pragma unroll
  for (int k = 0; k < kIn; ++k) atomicAdd(&grad[oW1 + j * kIn + k], gW1[k]);
  atomicAdd(&grad[oB1 + j], gb1);
  for (int k = 0; k < kHid; ++k) atomicAdd(&grad[oW2 + j * kHid + k], gW2[k]);
  atomicAdd(&grad[oB2 + j], gb2);
#pragma unroll
  for (int o = 0; o < kOut; ++o) atomicAdd(&grad[oW3 + o * kHid + j], gW3[o]);
  if (j < kOut) atomicAdd(&grad[oB3 + j], gb3);
  // loss: warp sums then one atomic per warp
  __syncwarp();
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(kFull, lsum, o);
  if ((j & 31) == 0) atomicAdd(loss, lsum * inv_n);
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       const int n, const float lr, const float b1, const float b2, const float eps, const float c1,
                       const float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

int mlp_grid(int n) { return std::max(1, std::min((n + kTile - 1) / kTile, device_info().sms * 4)); }

bool configure_mlp() {
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  if (done[dev]) return true;
  if (cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem)) != cudaSuccess)
    return false;
  if (cudaFuncSetAttribute(k_mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem)) !=
      cudaSuccess)
    return false;
  done[dev] = true;
  return true;
}

}  // namespace
}  // namespace tc

using namespace tc;

// The 256 cells' network inputs: the caller's features, or each cell's nominal degrees
// (a = 1.5 * 2^(c/16), b = 1.5 * 2^(c%16)) when there are none.
static void cell_feature_rows(const float* cell_features, float* feat) {
  for (int c = 0; c < 256; ++c) {
    if (cell_features) {
      for (int k = 0; k < kIn; ++k) feat[c * kIn + k] = cell_features[c * kIn + k];
    } else {
      const double a = 1.5 * (double)(1 << (c / 16)), b = 1.5 * (double)(1 << (c % 16));
      feat[c * kIn + 0] = (float)std::log2(1.0 + a);
      feat[c * kIn + 1] = (float)std::log2(1.0 + b);
      feat[c * kIn + 2] = (float)(std::min(a, b) / std::max(a, b));
      feat[c * kIn + 3] = (float)c / 255.f;
    }
  }
}

extern "C" {

tc_status tc_mlp_init(float* params_host, uint64_t seed) {
  if (!params_host) return fail(TC_ERR_INVALID_ARG, "params is NULL");
  // He-uniform initialisation from a counter-based generator; biases zero.
  auto rnd = [&](uint64_t i) {
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + i + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  };
  memset(params_host, 0, sizeof(float) * kParams);
  const double s1 = std::sqrt(6.0 / kIn), s2 = std::sqrt(6.0 / kHid);
  for (int i = 0; i < kHid * kIn; ++i) params_host[oW1 + i] = (float)(s1 * rnd(i));
  for (int i = 0; i < kHid * kHid; ++i) params_host[oW2 + i] = (float)(s2 * rnd(1000 + i));
  for (int i = 0; i < kOut * kHid; ++i) params_host[oW3 + i] = (float)(s2 * 0.1 * rnd(10000 + i));
  return TC_OK;
}

tc_status tc_mlp_forward(const float* d_params, const float* d_x, int32_t n, float* d_y, void* stream) {
  if (!d_params || n < 0 || (n > 0 && (!d_x || !d_y))) return fail(TC_ERR_INVALID_ARG, "invalid MLP arguments");
  if (n == 0) return TC_OK;
  if (!configure_mlp()) return fail(TC_ERR_CUDA, "MLP kernel configuration failed");
  k_mlp_forward<<<mlp_grid(n), kHid, sizeof(MlpSmem), (cudaStream_t)stream>>>(d_params, d_x, n, d_y);
  TC_CUDA_TRY(cudaGetLastError());
  return TC_OK;
}

tc_status tc_mlp_backward(const float* d_params, const float* d_x, const int32_t* d_strategy, const float* d_label,
                          int32_t n, float* d_grad, float* d_loss, void* stream) {
  if (!d_params || !d_grad || !d_loss || n < 0 || (n > 0 && (!d_x || !d_strategy || !d_label)))
    return fail(TC_ERR_INVALID_ARG, "invalid MLP arguments");
  cudaStream_t s = (cudaStream_t)stream;
  TC_CUDA_TRY(cudaMemsetAsync(d_grad, 0, sizeof(float) * kParams, s));
  TC_CUDA_TRY(cudaMemsetAsync(d_loss, 0, sizeof(float), s));
  if (n == 0) return TC_OK;
  if (!configure_mlp()) return fail(TC_ERR_CUDA, "MLP kernel configuration failed");
  k_mlp_backward<<<mlp_grid(n), kHid, sizeof(MlpSmem), s>>>(d_params, d_x, d_strategy, d_label, n, d_grad, d_loss);
  TC_CUDA_TRY(cudaGetLastError());
  return TC_OK;
}

tc_status tc_mlp_adam_step(float* d_params, const float* d_grad, float* d_m, float* d_v, int32_t step, float lr,
                           void* stream) {
  if (!d_params || !d_grad || !d_m || !d_v || step < 1) return fail(TC_ERR_INVALID_ARG, "invalid Adam arguments");
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
  k_adam<<<(kParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_params, d_grad, d_m, d_v, kParams, lr, b1, b2, eps,
                                                                  c1, c2);
  TC_CUDA_TRY(cudaGetLastError());
  return TC_OK;
}

tc_status tc_sched_from_costs(int kind, const float* cell_features, const float* costs, tc_sched* sch) {
  if (!sch || !costs || (kind != 0 && kind != 1)) return fail(TC_ERR_INVALID_ARG, "invalid arguments");
  std::vector<float> feat(256 * kIn);
  cell_feature_rows(cell_features, feat.data());
  // Output ids: static count 0 = the warp streams the list through the hash set, 1 = one lane
  // walks it, 2 = packed walk (the table entry is the output id); streaming 1 = binary search,
  // 2 = merge (table entries 0 and 1). The outputs are predicted log2 costs per edge. A cell
  // departs from the fixed rule (static: lane_max_deg / packed_max_deg; streaming:
  // search_ratio_x16; applied to the cell's mean degrees) only when the network predicts another
  // strategy at least kMargin cheaper; otherwise the rule's choice stays (the fallback).
  constexpr double kMargin = 0.05;
  const float log_keep = (float)std::log2(1.0 - kMargin);
  const long long ratio = std::max(0, sch->search_ratio_x16);
  const long long lane_max = std::max(0, sch->lane_max_deg);
  const long long packed_max = std::max(0, sch->packed_max_deg);
  for (int c = 0; c < 256; ++c) {
    const double a = std::max(1.0, std::exp2((double)feat[c * kIn + 0]) - 1.0);
    const double b = std::max(1.0, std::exp2((double)feat[c * kIn + 1]) - 1.0);
    const long long ai = (long long)std::llround(a), bi = (long long)std::llround(b);
    int lg = 0;
    for (long long t = bi; t > 0; t >>= 1) ++lg;
    // table entries: static 0 = warp, 1 = lane, 2 = packed; streaming 0 = search, 1 = merge
    const int rule = kind == 0 ? (bi <= lane_max ? 1 : bi <= packed_max ? 2 : 0)
                               : (16LL * bi > ratio * ai * lg ? 0 : 1);
    const int nstrat = kind == 0 ? 3 : 2;
    const int out0 = kind == 0 ? 0 : 1;  // network output of table entry 0
    const float c_rule = costs[c * kOut + out0 + rule];
    int pick = rule;
    float c_best = c_rule + log_keep;
    for (int e = 0; e < nstrat; ++e) {
      const float ce = costs[c * kOut + out0 + e];
      if (e != rule && ce < c_best) {
        c_best = ce;
        pick = e;
      }
    }
    sch->table[c / 16][c % 16] = (uint8_t)pick;
  }
  sch->use_table = 1;
  return TC_OK;
}

tc_status tc_sched_learned(const float* d_params, int kind, const float* cell_features, tc_sched* sch, void* stream) {
  if (!d_params || !sch || (kind != 0 && kind != 1)) return fail(TC_ERR_INVALID_ARG, "invalid arguments");
  std::vector<float> feat(256 * kIn);
  cell_feature_rows(cell_features, feat.data());
  cudaStream_t s = (cudaStream_t)stream;
  float *dx = nullptr, *dy = nullptr;
  TC_CUDA_TRY(::tc::dev_malloc(&dx, sizeof(float) * feat.size()));
  TC_CUDA_TRY(::tc::dev_malloc(&dy, sizeof(float) * 256 * kOut));
  std::vector<float> y(256 * kOut);
  tc_status rc = TC_OK;
  if (cudaMemcpyAsync(dx, feat.data(), sizeof(float) * feat.size(), cudaMemcpyHostToDevice, s) != cudaSuccess)
    rc = fail(TC_ERR_CUDA, "copy failed");
  if (rc == TC_OK) rc = tc_mlp_forward(d_params, dx, 256, dy, stream);
  if (rc == TC_OK && (cudaMemcpyAsync(y.data(), dy, sizeof(float) * y.size(), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                      cudaStreamSynchronize(s) != cudaSuccess))
    rc = fail(TC_ERR_CUDA, "copy failed");
  cudaFree(dx);
  cudaFree(dy);
  if (rc != TC_OK) return rc;
  return tc_sched_from_costs(kind, feat.data(), y.data(), sch);
}

tc_status tc_mlp_train(float* d_params, const float* d_x, const int32_t* d_strategy, const float* d_label, int32_t n,
                       int32_t epochs, float lr, float* loss_host, void* stream) {
  if (!d_params || n <= 0 || epochs < 1) return fail(TC_ERR_INVALID_ARG, "invalid training arguments");
  cudaStream_t s = (cudaStream_t)stream;
  float *g = nullptr, *m = nullptr, *v = nullptr, *l = nullptr;
  TC_CUDA_TRY(::tc::dev_malloc(&g, sizeof(float) * kParams));
  TC_CUDA_TRY(::tc::dev_malloc(&m, sizeof(float) * kParams));
  TC_CUDA_TRY(::tc::dev_malloc(&v, sizeof(float) * kParams));
  TC_CUDA_TRY(::tc::dev_malloc(&l, sizeof(float)));
  cudaMemsetAsync(m, 0, sizeof(float) * kParams, s);
  cudaMemsetAsync(v, 0, sizeof(float) * kParams, s);
  tc_status rc = TC_OK;
  for (int e = 1; e <= epochs && rc == TC_OK; ++e) {
    rc = tc_mlp_backward(d_params, d_x, d_strategy, d_label, n, g, l, stream);
    if (rc == TC_OK) rc = tc_mlp_adam_step(d_params, g, m, v, e, lr, stream);
  }
  if (rc == TC_OK && loss_host) {
    // loss of the final parameters
    rc = tc_mlp_backward(d_params, d_x, d_strategy, d_label, n, g, l, stream);
    if (rc == TC_OK && cudaMemcpyAsync(loss_host, l, sizeof(float), cudaMemcpyDeviceToHost, s) != cudaSuccess)
      rc = fail(TC_ERR_CUDA, "loss copy failed");
    if (rc == TC_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(TC_ERR_CUDA, "training failed");
  }
  cudaFree(g);
  cudaFree(m);
  cudaFree(v);
  cudaFree(l);
  return rc;
}

}  // extern "C"
