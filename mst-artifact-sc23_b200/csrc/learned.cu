// Learned schedule for the MST solve: graph features computed on the device,
// and a small MLP (16 -> 64 -> 64 -> 2, ReLU, fp32) with hand-written CUDA
// inference, gradient and training (Adam) kernels. The network maps the
// features to the light-phase filter quantile (output 0, as log2 q relative
// to the reference heuristic's quantile) and the scan's degree split
// (output 1, as log2 split). Only the schedule changes;
// the forest is unique under the (weight, index) order, so the answer does
// not (for non-negative weights). The reference heuristic (ECL_MST.cu:432-440)
// remains the fallback when no weights are loaded.
//
// Parameter blob layout (kMlpParams floats):
//   W1[16][64], b1[64], W2[64][64], b2[64], W3[64][2], b3[2], mean[16], std[16]
// Features are standardised with mean/std before the first layer.
#include <cub/block/block_radix_sort.cuh>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "ecl_mst.h"
#include "internal.h"
#include "mst_kernels.cuh"

namespace {

constexpr int kIn = ECL_MLP_INPUTS, kH = ECL_MLP_HIDDEN, kOut = ECL_MLP_OUTPUTS;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kIn * kH, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH * kOut, kOffMean = kOffB3 + kOut;
constexpr int kOffStd = kOffMean + kIn, kParams = kOffStd + kIn;
static_assert(kParams == ECL_MLP_PARAMS, "parameter blob size");
constexpr int kTrainable = kOffMean;  // W1..b3
constexpr int kMB = 64;               // training minibatch
constexpr int kSample = 4096;         // weight sample for the quantile features
constexpr float kNoFilterLog2Q = -0.32192809f;  // log2(0.8): predicted quantiles above run unfiltered

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return ECL_OK;
  if (e == cudaErrorMemoryAllocation) return ECL_ERR_ALLOC;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return ECL_ERR_NO_DEVICE;
  return ECL_ERR_CUDA;
}
#define ML_TRY(call)                               \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

// ------------------------------------------------------------- features
using ecl::FeatAcc;
using ecl::FeatPart;

constexpr int kFeatThreads = 1024;
constexpr int kFeatKeys = kSample / kFeatThreads;

// The 4096-entry hashed weight sample, sorted (a block radix sort, 4 keys per
// thread) into `sorted`. One CTA of kFeatThreads.
__device__ __forceinline__ void sort_sample(const int* eweight, int m, int* sorted) {
  typedef cub::BlockRadixSort<int, kFeatThreads, kFeatKeys> SampleSort;
  __shared__ typename SampleSort::TempStorage sort_tmp;
  int keys[kFeatKeys];
#pragma unroll
  for (int k = 0; k < kFeatKeys; k++) {
    const int i = threadIdx.x * kFeatKeys + k;
    const uint64_t r = ecl_mix64(0xFEA70000ull + (uint64_t)i);
    keys[k] = m > 0 ? __ldg(eweight + (unsigned)(r % (uint64_t)(unsigned)m)) : 0;
  }
  SampleSort(sort_tmp).Sort(keys);  // blocked: thread t holds ranks t * kFeatKeys ...
#pragma unroll
  for (int k = 0; k < kFeatKeys; k++) sorted[threadIdx.x * kFeatKeys + k] = keys[k];
}

// The solve's share of the feature pass: the sorted weight sample (the
// degree statistics come from k_prep).
__global__ void __launch_bounds__(kFeatThreads) k_sample(const int* eweight, int m, int* sorted) {
  sort_sample(eweight, m, sorted);
}

// The whole feature pass for a graph outside a solve: block 0 sorts the
// weight sample, the other blocks take the degree statistics over all
// vertices (grid-stride) exactly as k_prep does.
__global__ void __launch_bounds__(kFeatThreads) k_feat(const int* nindex, int n, const int* eweight, int m,
                                                        FeatAcc* acc, int* sorted) {
  if (blockIdx.x == 0) {
    sort_sample(eweight, m, sorted);
    return;
  }
  FeatPart fp;
  const int stride = (gridDim.x - 1) * blockDim.x;
  for (int v = (blockIdx.x - 1) * blockDim.x + threadIdx.x; v < n; v += stride) {
    const int b = __ldg(nindex + v), e = __ldg(nindex + v + 1);
    fp.add(e > b ? (unsigned)(e - b) : 0u);
  }
  fp.fold<kFeatThreads>(acc);
}

// Grid of the feature pass: the sorting block plus up to two degree blocks per SM.
int feat_grid(int nodes, int sms) {
  return 1 + std::max(1, std::min(sms * 2, (nodes + kFeatThreads - 1) / kFeatThreads));
}

// The 16 features (one thread), from the degree statistics and the sorted
// weight sample.
__device__ void compute_features(int n, int m, const FeatAcc* acc, const int* sorted, float* out) {
  const double dn = (double)n, dm = (double)m;
  const double mean = dm / dn;
  const double var = fmax(0.0, (double)acc->deg_sq / dn - mean * mean);
  const double wmax = fmax(1.0, (double)sorted[kSample - 1]);
  const float qs[7] = {0.01f, 0.02f, 0.05f, 0.1f, 0.2f, 0.3f, 0.5f};
  out[0] = (float)log2(dn);
  out[1] = (float)log2(fmax(dm, 1.0));
  out[2] = (float)log2(mean + 1.0);
  out[3] = (float)log2((double)acc->max_deg + 1.0);
  out[4] = (float)(sqrt(var) / fmax(mean, 1e-9));
  out[5] = (float)((double)acc->zero / dn);
  out[6] = (float)((double)acc->low / dn);
  out[7] = (float)((double)acc->high / dn);
  out[8] = (float)(3.0 * dn / fmax(dm, 1.0));  // the reference heuristic's "300% of nodes" quantile
  for (int i = 0; i < 7; i++) out[9 + i] = (float)((double)sorted[(int)(qs[i] * (kSample - 1))] / wmax);
}

// The features alone (for training data): one thread.
__global__ void k_feat_finish(int n, int m, const FeatAcc* acc, const int* sorted, float* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) compute_features(n, m, acc, sorted, out);
}

// ------------------------------------------------------------------- MLP
__device__ __forceinline__ float relu(float x) { return x > 0.f ? x : 0.f; }

// Forward pass of one sample held in x[kIn] (already standardised); h1, h2
// and y are written. Serial per thread (the network is tiny).
__device__ void mlp_forward1(const float* p, const float* x, float* h1, float* h2, float* y) {
  for (int j = 0; j < kH; j++) {
    float a = p[kOffB1 + j];
    for (int i = 0; i < kIn; i++) a += x[i] * p[kOffW1 + i * kH + j];
    h1[j] = relu(a);
  }
  for (int k = 0; k < kH; k++) {
    float a = p[kOffB2 + k];
    for (int j = 0; j < kH; j++) a += h1[j] * p[kOffW2 + j * kH + k];
    h2[k] = relu(a);
  }
  for (int o = 0; o < kOut; o++) {
    float a = p[kOffB3 + o];
    for (int k = 0; k < kH; k++) a += h2[k] * p[kOffW3 + k * kOut + o];
    y[o] = a;
  }
}

// Inference for B samples (raw features; standardised here).
__global__ void k_mlp_infer(const float* p, const float* x, int B, float* y) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  float xs[kIn], h1[kH], h2[kH];
  for (int i = 0; i < kIn; i++) xs[i] = (x[b * kIn + i] - p[kOffMean + i]) / p[kOffStd + i];
  mlp_forward1(p, xs, h1, h2, y + b * kOut);
}

// log2 of the weight quantile the reference heuristic filters at
// (ECL_MST.cu:408,432-440): the idx-th of 20 samples sits at quantile
// (idx + 1) / 21 on average; 0 (no filter) when edges/nodes < 4.
__host__ __device__ __forceinline__ float heuristic_log2_quantile(int n, int m) {
  if (n < 1 || m / n < 4) return 0.f;
  const int idx = min(19, (int)(3.0 * n * 20 / m));
  return log2f((float)(idx + 1) / 21.f);
}

// Decode the network output into the solve's control block. Output 0 is the
// log2 quantile relative to the reference heuristic's; output 1 the log2
// degree split.
// One CTA of kH threads: thread j computes hidden unit j of each layer. The
// decoded quantile selects the light-phase threshold from the sorted weight
// sample of the feature pass.
__global__ void k_mlp_apply(const float* pg, const FeatAcc* acc, const int* sorted, int n, int m,
                            ecl::DevState* st, float* feat_out) {
  // the whole parameter blob (21 KB) is staged in shared memory first, so the
  // layers read it at shared-memory latency instead of one global load per
  // multiply-add
  __shared__ float p[kParams];
  __shared__ float fx[kIn], xs[kIn], h1[kH], h2[kH], y[kOut];
  const int j = threadIdx.x;
  for (int i = j; i < kParams; i += blockDim.x) p[i] = __ldg(pg + i);
  if (j == 0) compute_features(n, m, acc, sorted, fx);
  __syncthreads();
  if (j < kIn) {
    feat_out[j] = fx[j];  // kept for ecl_mst_ctx_learned_features
    xs[j] = (fx[j] - p[kOffMean + j]) / p[kOffStd + j];
  }
  __syncthreads();
  if (j < kH) {
    float a = p[kOffB1 + j];
    for (int i = 0; i < kIn; i++) a += xs[i] * p[kOffW1 + i * kH + j];
    h1[j] = relu(a);
  }
  __syncthreads();
  if (j < kH) {
    float a = p[kOffB2 + j];
    for (int i = 0; i < kH; i++) a += h1[i] * p[kOffW2 + i * kH + j];
    h2[j] = relu(a);
  }
  __syncthreads();
  if (j < kOut) {
    float a = p[kOffB3 + j];
    for (int i = 0; i < kH; i++) a += h2[i] * p[kOffW3 + i * kOut + j];
    y[j] = a;
  }
  __syncthreads();
  if (j != 0) return;
  // output 0 (+ the heuristic's log2 quantile) at or above log2(0.8) means
  // "no filter": a light phase holding 80 % of the entries or more is not
  // worth a second phase (measured on the held-out sweeps)
  const float lq = fminf(fmaxf(heuristic_log2_quantile(n, m) + y[0], -10.f), 0.f);
  const float q = lq >= kNoFilterLog2Q ? 1.0f : exp2f(lq);
  st->quantile = q;
  if (q < 1.0f) {
    int idx = (int)(q * (float)(kSample - 1));
    idx = idx < 0 ? 0 : (idx > kSample - 1 ? kSample - 1 : idx);
    st->filtered = 1;
    st->threshold = sorted[idx];
  } else {
    st->filtered = 0;
    st->threshold = 0x7fffffff;
  }
  // output 1: log2 of the degree split, in [1, 6]
  st->learned_split = 1 << (int)lrintf(fminf(fmaxf(y[1], 1.f), 6.f));
  st->split = st->learned_split;  // read by the scans (k_prep leaves it alone in this mode)
}

// Full-batch mean-squared-error loss and gradient of the trainable
// parameters (W1..b3). One CTA; every thread accumulates the gradient of a
// strided subset of samples into shared memory with atomics, in a fixed
// order per thread. grad must hold kTrainable floats.
__device__ void mlp_grad_block(const float* p, const float* x, const float* t, int B, float* g_sm,
                               float* loss_sm) {
  for (int i = threadIdx.x; i < kTrainable; i += blockDim.x) g_sm[i] = 0.f;
  if (threadIdx.x == 0) *loss_sm = 0.f;
  __syncthreads();
  const float inv = 1.f / (float)(B > 0 ? B : 1);
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    float xs[kIn], h1[kH], h2[kH], y[kOut], dy[kOut], d2[kH];
    for (int i = 0; i < kIn; i++) xs[i] = x[b * kIn + i];
    mlp_forward1(p, xs, h1, h2, y);
    float l = 0.f;
    for (int o = 0; o < kOut; o++) {
      const float e = y[o] - t[b * kOut + o];
      l += e * e;
      dy[o] = 2.f * e * inv;
    }
    atomicAdd(loss_sm, l * inv);
    for (int o = 0; o < kOut; o++) atomicAdd(&g_sm[kOffB3 + o], dy[o]);
    for (int k = 0; k < kH; k++) {
      float a = 0.f;
      for (int o = 0; o < kOut; o++) {
        atomicAdd(&g_sm[kOffW3 + k * kOut + o], h2[k] * dy[o]);
        a += dy[o] * p[kOffW3 + k * kOut + o];
      }
      d2[k] = h2[k] > 0.f ? a : 0.f;
      atomicAdd(&g_sm[kOffB2 + k], d2[k]);
    }
    for (int j = 0; j < kH; j++) {
      float a = 0.f;
      for (int k = 0; k < kH; k++) {
        if (d2[k] != 0.f) atomicAdd(&g_sm[kOffW2 + j * kH + k], h1[j] * d2[k]);
        a += d2[k] * p[kOffW2 + j * kH + k];
      }
      const float d1 = h1[j] > 0.f ? a : 0.f;
      if (d1 != 0.f) {
        atomicAdd(&g_sm[kOffB1 + j], d1);
        for (int i = 0; i < kIn; i++) atomicAdd(&g_sm[kOffW1 + i * kH + j], xs[i] * d1);
      }
    }
  }
  __syncthreads();
}

__global__ void k_mlp_grad(const float* p, const float* x, const float* t, int B, float* grad,
                           float* loss) {
  extern __shared__ float smem[];
  float* g_sm = smem;
  float* l_sm = smem + kTrainable;
  mlp_grad_block(p, x, t, B, g_sm, l_sm);
  for (int i = threadIdx.x; i < kTrainable; i += blockDim.x) grad[i] = g_sm[i];
  if (threadIdx.x == 0) *loss = *l_sm;
}

// The whole training run in one launch (one CTA): epochs over minibatches
// of kMB standardised samples, Adam (beta1 0.9, beta2 0.999, eps 1e-8).
// Parameters and the two moment vectors live in global memory; gradients in
// shared memory. loss_hist[e] = mean minibatch loss of epoch e.
__global__ void k_mlp_train(float* p, float* m1, float* m2, const float* x, const float* t, int B,
                            int epochs, float lr, float* loss_hist) {
  extern __shared__ float smem[];
  float* g_sm = smem;
  float* l_sm = smem + kTrainable;
  int step = 0;
  for (int e = 0; e < epochs; e++) {
    float acc = 0.f;
    int nb = 0;
    for (int b0 = 0; b0 < B; b0 += kMB) {
      const int bs = min(kMB, B - b0);
      mlp_grad_block(p, x + (size_t)b0 * kIn, t + (size_t)b0 * kOut, bs, g_sm, l_sm);
      step++;
      const float c1 = 1.f - powf(0.9f, (float)step), c2 = 1.f - powf(0.999f, (float)step);
      for (int i = threadIdx.x; i < kTrainable; i += blockDim.x) {
        const float g = g_sm[i];
        const float a = 0.9f * m1[i] + 0.1f * g;
        const float v = 0.999f * m2[i] + 0.001f * g * g;
        m1[i] = a;
        m2[i] = v;
        p[i] -= lr * (a / c1) / (sqrtf(v / c2) + 1e-8f);
      }
      acc += *l_sm;
      nb++;
      __syncthreads();
    }
    if (threadIdx.x == 0) loss_hist[e] = acc / (float)(nb > 0 ? nb : 1);
    __syncthreads();
  }
}

std::mutex g_w_mu;
std::vector<float> g_weights;  // host copy of the loaded parameter blob
unsigned g_w_version = 0;      // bumped by every load; contexts re-upload on change

}  // namespace

struct ecl_mst_ctx;
int ecl_ctx_learned_buffers(ecl_mst_ctx* c, float** params, float** feat, void** acc, int** sample,
                            unsigned** version, int* sm_count);

extern "C" int ecl_learned_set_weights(const float* params, int count) {
  if (count != kParams || !params) return ECL_ERR_INVALID_ARG;
  for (int i = 0; i < kIn; i++)
    if (!(params[kOffStd + i] > 0.f)) return ECL_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_w_mu);
  g_weights.assign(params, params + count);
  g_w_version++;
  return ECL_OK;
}

extern "C" int ecl_learned_has_weights(void) {
  std::lock_guard<std::mutex> lock(g_w_mu);
  return g_weights.empty() ? 0 : 1;
}

// Version of the loaded weights (bumped by every load); part of the key of a
// captured solve, whose graph does not re-upload them.
unsigned ecl_learned_weights_version() {
  std::lock_guard<std::mutex> lock(g_w_mu);
  return g_w_version;
}

// Upload the loaded weights to the context's parameter buffer if they
// changed since its last upload (synchronous: call it outside any stream
// capture before capturing learned solves).
int ecl_learned_upload(ecl_mst_ctx* c, cudaStream_t s) {
  float *d_params, *d_feat;
  void* d_acc;
  int* d_sample;
  unsigned* version;
  int sms = 0;
  int r = ecl_ctx_learned_buffers(c, &d_params, &d_feat, &d_acc, &d_sample, &version, &sms);
  if (r) return r;
  std::lock_guard<std::mutex> lock(g_w_mu);
  if (g_weights.empty()) return ECL_ERR_UNSUPPORTED;
  if (*version != g_w_version) {
    ML_TRY(cudaMemcpyAsync(d_params, g_weights.data(), kParams * sizeof(float), cudaMemcpyHostToDevice, s));
    ML_TRY(cudaStreamSynchronize(s));
    *version = g_w_version;
  }
  return ECL_OK;
}

// A learned solve's weight sample, sorted on stream s (after uploading the
// loaded weights if they changed since this context's last upload).
int ecl_learned_sample(ecl_mst_ctx* c, const ecl_graph* g, cudaStream_t s) {
  int r = ecl_learned_upload(c, s);
  if (r) return r;
  float *d_params, *d_feat;
  void* d_acc;
  int* d_sample;
  unsigned* version;
  int sms = 0;
  if ((r = ecl_ctx_learned_buffers(c, &d_params, &d_feat, &d_acc, &d_sample, &version, &sms))) return r;
  k_sample<<<1, kFeatThreads, 0, s>>>(g->eweight, g->edges, d_sample);
  ML_TRY(cudaGetLastError());
  return ECL_OK;
}

// The features (sorted sample + k_prep's degree statistics) and the MLP, on
// stream s once both are complete; writes the decoded schedule into the
// solve's control block `st`.
int ecl_learned_apply(ecl_mst_ctx* c, const ecl_graph* g, cudaStream_t s, void* st) {
  float *d_params, *d_feat;
  void* d_acc;
  int* d_sample;
  unsigned* version;
  int sms = 0;
  int r = ecl_ctx_learned_buffers(c, &d_params, &d_feat, &d_acc, &d_sample, &version, &sms);
  if (r) return r;
  k_mlp_apply<<<1, 256, 0, s>>>(d_params, (const FeatAcc*)d_acc, d_sample, g->nodes, g->edges,
                               (ecl::DevState*)st, d_feat);
  ML_TRY(cudaGetLastError());
  return ECL_OK;
}

// Features of a device-resident graph, copied to host out[16].
extern "C" int ecl_graph_features(const ecl_graph* g, float* out) {
  if (!g || !out || g->nodes < 1 || g->edges < 0 || !g->nindex || (g->edges > 0 && !g->eweight))
    return ECL_ERR_INVALID_ARG;
  int dev = 0, sms = 0;
  ML_TRY(cudaGetDevice(&dev));
  ML_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  FeatAcc* acc = nullptr;
  float* f = nullptr;
  int* sorted = nullptr;
  ML_TRY(cudaMalloc(&acc, sizeof(FeatAcc)));
  if (cudaMalloc(&f, kIn * sizeof(float)) != cudaSuccess || cudaMalloc(&sorted, kSample * sizeof(int)) != cudaSuccess) {
    cudaFree(acc);
    cudaFree(f);
    return ECL_ERR_ALLOC;
  }
  cudaMemset(acc, 0, sizeof(FeatAcc));
  k_feat<<<feat_grid(g->nodes, sms), kFeatThreads>>>(g->nindex, g->nodes, g->eweight, g->edges, acc, sorted);
  k_feat_finish<<<1, 32>>>(g->nodes, g->edges, acc, sorted, f);
  cudaError_t e = cudaMemcpy(out, f, kIn * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(acc);
  cudaFree(f);
  cudaFree(sorted);
  return cuda_status(e);
}

namespace {
struct DevBuf {
  float* p = nullptr;
  ~DevBuf() { cudaFree(p); }
  int alloc(size_t n) { return cuda_status(cudaMalloc(&p, n * sizeof(float))); }
};
}  // namespace

extern "C" int ecl_mlp_forward(const float* params, const float* x, int B, float* y) {
  if (!params || !x || !y || B < 0) return ECL_ERR_INVALID_ARG;
  if (B == 0) return ECL_OK;
  DevBuf dp, dx, dy;
  int r;
  if ((r = dp.alloc(kParams)) || (r = dx.alloc((size_t)B * kIn)) || (r = dy.alloc((size_t)B * kOut))) return r;
  ML_TRY(cudaMemcpy(dp.p, params, kParams * sizeof(float), cudaMemcpyHostToDevice));
  ML_TRY(cudaMemcpy(dx.p, x, (size_t)B * kIn * sizeof(float), cudaMemcpyHostToDevice));
  k_mlp_infer<<<(B + 127) / 128, 128>>>(dp.p, dx.p, B, dy.p);
  ML_TRY(cudaGetLastError());
  ML_TRY(cudaMemcpy(y, dy.p, (size_t)B * kOut * sizeof(float), cudaMemcpyDeviceToHost));
  return ECL_OK;
}

extern "C" int ecl_mlp_grad(const float* params, const float* x, const float* t, int B, float* grad,
                            float* loss) {
  if (!params || !x || !t || !grad || !loss || B < 1) return ECL_ERR_INVALID_ARG;
  DevBuf dp, dx, dt, dg, dl;
  int r;
  if ((r = dp.alloc(kParams)) || (r = dx.alloc((size_t)B * kIn)) || (r = dt.alloc((size_t)B * kOut)) ||
      (r = dg.alloc(kTrainable)) || (r = dl.alloc(1)))
    return r;
  ML_TRY(cudaMemcpy(dp.p, params, kParams * sizeof(float), cudaMemcpyHostToDevice));
  ML_TRY(cudaMemcpy(dx.p, x, (size_t)B * kIn * sizeof(float), cudaMemcpyHostToDevice));
  ML_TRY(cudaMemcpy(dt.p, t, (size_t)B * kOut * sizeof(float), cudaMemcpyHostToDevice));
  const size_t smem = (kTrainable + 1) * sizeof(float);
  ML_TRY(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_mlp_grad<<<1, 256, smem>>>(dp.p, dx.p, dt.p, B, dg.p, dl.p);
  ML_TRY(cudaGetLastError());
  ML_TRY(cudaMemcpy(grad, dg.p, kTrainable * sizeof(float), cudaMemcpyDeviceToHost));
  ML_TRY(cudaMemcpy(loss, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
  return ECL_OK;
}

extern "C" int ecl_mlp_train(float* params, const float* x, const float* t, int B, int epochs, float lr,
                             float* loss_hist) {
  if (!params || !x || !t || B < 1 || epochs < 1 || !(lr > 0.f)) return ECL_ERR_INVALID_ARG;
  DevBuf dp, dm1, dm2, dx, dt, dl;
  int r;
  if ((r = dp.alloc(kParams)) || (r = dm1.alloc(kTrainable)) || (r = dm2.alloc(kTrainable)) ||
      (r = dx.alloc((size_t)B * kIn)) || (r = dt.alloc((size_t)B * kOut)) || (r = dl.alloc(epochs)))
    return r;
  ML_TRY(cudaMemcpy(dp.p, params, kParams * sizeof(float), cudaMemcpyHostToDevice));
  ML_TRY(cudaMemset(dm1.p, 0, kTrainable * sizeof(float)));
  ML_TRY(cudaMemset(dm2.p, 0, kTrainable * sizeof(float)));
  ML_TRY(cudaMemcpy(dx.p, x, (size_t)B * kIn * sizeof(float), cudaMemcpyHostToDevice));
  ML_TRY(cudaMemcpy(dt.p, t, (size_t)B * kOut * sizeof(float), cudaMemcpyHostToDevice));
  const size_t smem = (kTrainable + 1) * sizeof(float);
  ML_TRY(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_mlp_train<<<1, 256, smem>>>(dp.p, dm1.p, dm2.p, dx.p, dt.p, B, epochs, lr, dl.p);
  ML_TRY(cudaGetLastError());
  ML_TRY(cudaMemcpy(params, dp.p, kParams * sizeof(float), cudaMemcpyDeviceToHost));
  if (loss_hist) ML_TRY(cudaMemcpy(loss_hist, dl.p, (size_t)epochs * sizeof(float), cudaMemcpyDeviceToHost));
  return ECL_OK;
}
