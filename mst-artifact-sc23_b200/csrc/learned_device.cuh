// Device side of the learned schedule shared by the solve (k_prep) and the
// standalone feature pass (learned.cu): the hashed weight sample and its sort,
// the 16 features, and the network's forward pass with the decoding of its
// two outputs into the solve's control block.
//
// Parameter blob layout (ECL_MLP_PARAMS floats):
//   W1[16][64], b1[64], W2[64][64], b2[64], W3[64][2], b3[2], mean[16], std[16]
// Features are standardised with mean/std before the first layer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ecl_mst.h"
#include "internal.h"
#include "mst_kernels.cuh"

namespace ecl {

constexpr int kMlpIn = ECL_MLP_INPUTS, kMlpH = ECL_MLP_HIDDEN, kMlpOut = ECL_MLP_OUTPUTS;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kMlpIn * kMlpH, kOffW2 = kOffB1 + kMlpH;
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH, kOffW3 = kOffB2 + kMlpH, kOffB3 = kOffW3 + kMlpH * kMlpOut;
constexpr int kOffMean = kOffB3 + kMlpOut, kOffStd = kOffMean + kMlpIn, kMlpParams = kOffStd + kMlpIn;
static_assert(kMlpParams == ECL_MLP_PARAMS, "parameter blob size");
constexpr int kMlpTrainable = kOffMean;  // W1..b3
constexpr int kFeatSample = 4096;        // weight sample for the quantile features and the threshold
constexpr float kNoFilterLog2Q = -0.32192809f;  // log2(0.8): predicted quantiles above run unfiltered

// Weight sample of the learned schedule, sorted ascending into `smem`
// (kFeatSample ints) by the whole CTA: hashed entry positions, then a bitonic
// network in which each thread takes a share of the 2048 compare-exchange
// pairs of every stage. Ends with a CTA barrier.
__device__ __forceinline__ void sort_feat_sample(const int* eweight, int m, int* smem) {
  for (int i = threadIdx.x; i < kFeatSample; i += blockDim.x) {
    const uint64_t r = ecl_mix64(0xFEA70000ull + (uint64_t)i);
    smem[i] = m > 0 ? __ldg(eweight + (unsigned)(r % (uint64_t)(unsigned)m)) : 0;
  }
  __syncthreads();
  for (int k = 2; k <= kFeatSample; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int q = threadIdx.x; q < kFeatSample / 2; q += blockDim.x) {
        const int i = ((q & ~(j - 1)) << 1) | (q & (j - 1)), l = i + j;
        const int x = smem[i], y = smem[l];
        if ((x > y) == ((i & k) == 0)) {
          smem[i] = y;
          smem[l] = x;
        }
      }
      __syncthreads();
    }
  }
}

// The 16 features from the degree statistics and the sorted weight sample:
// log2 n, log2 m, log2(mean degree + 1), log2(max degree + 1), coefficient of
// variation of the degree, shares of degree 0, < 4 and >= 32, 3n/m (the
// reference heuristic's "300 % of nodes" quantile), and seven quantiles of
// the sample over its maximum. The sample is read through L2 (another CTA
// may have written it in the same launch).
__device__ __forceinline__ void compute_features(int n, int m, const FeatAcc& acc, const int* sorted,
                                                 float* out) {
  const double dn = (double)n, dm = (double)m;
  const double mean = dm / dn;
  const double var = fmax(0.0, (double)acc.deg_sq / dn - mean * mean);
  const double wmax = fmax(1.0, (double)__ldcg(sorted + kFeatSample - 1));
  const float qs[7] = {0.01f, 0.02f, 0.05f, 0.1f, 0.2f, 0.3f, 0.5f};
  out[0] = (float)log2(dn);
  out[1] = (float)log2(fmax(dm, 1.0));
  out[2] = (float)log2(mean + 1.0);
  out[3] = (float)log2((double)acc.max_deg + 1.0);
  out[4] = (float)(sqrt(var) / fmax(mean, 1e-9));
  out[5] = (float)((double)acc.zero / dn);
  out[6] = (float)((double)acc.low / dn);
  out[7] = (float)((double)acc.high / dn);
  out[8] = (float)(3.0 * dn / fmax(dm, 1.0));
  for (int i = 0; i < 7; i++)
    out[9 + i] = (float)((double)__ldcg(sorted + (int)(qs[i] * (kFeatSample - 1))) / wmax);
}

__device__ __forceinline__ float relu(float x) { return x > 0.f ? x : 0.f; }

// log2 of the weight quantile the reference heuristic filters at
// (ECL_MST.cu:408,432-440): the idx-th of 20 samples sits at quantile
// (idx + 1) / 21 on average; 0 (no filter) when edges/nodes < 4.
__host__ __device__ __forceinline__ float heuristic_log2_quantile(int n, int m) {
  if (n < 1 || m / n < 4) return 0.f;
  const int idx = min(19, (int)(3.0 * n * 20 / m));
  return log2f((float)(idx + 1) / 21.f);
}

// The network on one graph, run by a whole CTA (at least kMlpH threads): the
// parameter blob is staged in shared memory, thread j computes hidden unit j
// of each layer, and the two outputs are decoded into the control block.
// Output 0 is the log2 filter quantile relative to the reference heuristic's
// (at or above log2(0.8) the solve runs unfiltered: a light phase holding
// 80 % of the entries is not worth a second phase); the threshold is that
// quantile of the sorted sample. Output 1 is the log2 degree split, in
// [1, 6]. The features are also written to feat_out. Every thread of the CTA
// must call this.
__device__ __forceinline__ void mlp_decide(const float* pg, const float* fx_in, const int* sorted, int n,
                                           int m, DevState* st, float* feat_out) {
  __shared__ float p[kMlpParams];
  __shared__ float xs[kMlpIn], h1[kMlpH], h2[kMlpH], y[kMlpOut];
  const int j = threadIdx.x;
  for (int i = j; i < kMlpParams; i += blockDim.x) p[i] = __ldg(pg + i);
  __syncthreads();
  if (j < kMlpIn) {
    feat_out[j] = fx_in[j];
    xs[j] = (fx_in[j] - p[kOffMean + j]) / p[kOffStd + j];
  }
  __syncthreads();
  if (j < kMlpH) {
    float a = p[kOffB1 + j];
    for (int i = 0; i < kMlpIn; i++) a += xs[i] * p[kOffW1 + i * kMlpH + j];
    h1[j] = relu(a);
  }
  __syncthreads();
  if (j < kMlpH) {
    float a = p[kOffB2 + j];
    for (int i = 0; i < kMlpH; i++) a += h1[i] * p[kOffW2 + i * kMlpH + j];
    h2[j] = relu(a);
  }
  __syncthreads();
  if (j < kMlpOut) {
    float a = p[kOffB3 + j];
    for (int i = 0; i < kMlpH; i++) a += h2[i] * p[kOffW3 + i * kMlpOut + j];
    y[j] = a;
  }
  __syncthreads();
  if (j != 0) return;
  const float lq = fminf(fmaxf(heuristic_log2_quantile(n, m) + y[0], -10.f), 0.f);
  const float q = lq >= kNoFilterLog2Q ? 1.0f : exp2f(lq);
  st->quantile = q;
  if (q < 1.0f) {
    int idx = (int)(q * (float)(kFeatSample - 1));
    idx = idx < 0 ? 0 : (idx > kFeatSample - 1 ? kFeatSample - 1 : idx);
    st->filtered = 1;
    st->threshold = __ldcg(sorted + idx);
  } else {
    st->filtered = 0;
    st->threshold = 0x7fffffff;
  }
  st->learned_split = 1 << (int)lrintf(fminf(fmaxf(y[1], 1.f), 6.f));
  st->split = st->learned_split;  // read by the scans
}

}  // namespace ecl
