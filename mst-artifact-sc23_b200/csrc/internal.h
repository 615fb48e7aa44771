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
