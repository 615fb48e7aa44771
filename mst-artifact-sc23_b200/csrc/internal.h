// Declarations shared by the host (.cpp) and device (.cu) translation units.
#pragma once
#include <stdint.h>

#include "ecl_mst.h"

#if defined(__CUDACC__)
#define ECL_HD __host__ __device__ __forceinline__
#else
#define ECL_HD inline
#endif

// splitmix64 finalizer (Steele, Lea & Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014): a bijective 64-bit mixer.
ECL_HD uint64_t ecl_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// Counter-based random stream: value number `idx` of stream `stream` under
// `seed`. Host and device produce the same numbers, so a graph generated on
// either side is identical.
ECL_HD uint64_t ecl_rng(uint64_t seed, uint64_t stream, uint64_t idx) {
  return ecl_mix64(ecl_mix64(seed * 0x9E3779B97F4A7C15ULL + stream) ^
                   (idx * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL));
}

enum { ECL_STREAM_WEIGHT = 1, ECL_STREAM_RMAT = 2, ECL_STREAM_ER = 3, ECL_STREAM_RGG = 4 };

// Weight of the undirected edge {u, v}: uniform in [1, wmax], a function of
// the unordered pair only, so both directions carry the same value and
// duplicate samples of one edge agree.
ECL_HD int32_t ecl_edge_weight(uint64_t seed, uint32_t u, uint32_t v, int32_t wmax) {
  const uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
  const uint64_t r = ecl_rng(seed, ECL_STREAM_WEIGHT, ((uint64_t)lo << 32) | hi);
  return 1 + (int32_t)(r % (uint64_t)(wmax < 1 ? 1 : wmax));
}

// Uniform integer in [0, n) from 32 random bits (multiply-high).
ECL_HD uint32_t ecl_below(uint32_t bits, uint32_t n) {
  return (uint32_t)(((uint64_t)bits * n) >> 32);
}

// The reference heuristic's sample hash (ECL_MST.cu:389-395).
uint32_t ecl_sample_hash(uint32_t val);
int ecl_heuristic_threshold_arrays(int32_t nodes, int32_t edges,
                                   const int32_t* eweight, int32_t* threshold,
                                   int32_t* filtered);

// The reference's weight for a weightless input (ECL_MST.cu:410-419):
// 1 + ((i * k) % nodes), made non-negative. i * k wraps modulo 2^32 as int
// arithmetic does on every compiler the artifact targets.
ECL_HD int32_t ecl_synth_weight(int32_t i, int32_t k, int32_t nodes) {
  const int32_t prod = (int32_t)((uint32_t)i * (uint32_t)k);
  int32_t w = 1 + (prod % nodes);
  return w < 0 ? -w : w;
}

// Shared parameters of the synthetic families, so the host generators and the
// device generators (preprocess.cu) draw exactly the same graphs.
struct EclRmatCut {
  uint32_t ta, tab, tabc;  // quadrant thresholds in 16-bit fixed point
};
EclRmatCut ecl_rmat_cut(double a, double b, double c);

struct EclRggGrid {
  uint64_t r2;      // squared radius, 31-bit fixed point units
  int64_t cells;    // cells per side
  uint64_t cell_w;  // cell width
};
EclRggGrid ecl_rgg_grid(int32_t nodes, double avg_degree);

// Family (0 grid, 1 ER, 2 RMAT, 3 RGG2D), vertex count and seed of graph
// `index` of the mixed batch. rows_or_scale is the grid's row count or the
// RMAT scale (unused for the other families).
struct EclBatchPick {
  int family;
  int32_t nodes;
  int32_t rows_or_scale;
  uint64_t seed;
};
EclBatchPick ecl_batch_pick(int32_t index, uint64_t seed0, int32_t nmin, int32_t nmax);

// Families of the mixed batch (besides the grid): ER with average degree 8,
// RMAT (0.57, 0.19, 0.19) with edge factor 8, RGG2D with average degree 3.
constexpr double kBatchErDegree = 8.0;
constexpr int32_t kBatchRmatEdgeFactor = 8;
constexpr double kBatchRmatA = 0.57, kBatchRmatB = 0.19, kBatchRmatC = 0.19;
constexpr double kBatchRggDegree = 3.0;
