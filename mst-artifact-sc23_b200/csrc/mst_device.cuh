// Kernels of the single-graph B200 ECL-MST engine.
//
// Replaces gpuMST<filter>'s kernels (ECL-MST/ECL_MST.cu): initPM (:147-154),
// initWL<first> (:157-207), kernel1 (:210-226), kernel2 (:229-240),
// kernel3 (:243-251), find (:127-134), join (:137-144). The answer is the
// reference's: the unique minimum spanning forest under the strict order
// (uint32 weight, CSR index j) over the one-direction entries nlist[j] > v,
// built in a light phase (w <= threshold, signed compare as at :172) and a
// heavy phase (w > threshold). Launch sequence of one solve:
//
//   k_prep        initPM + CSR checks + threshold choice + the tile->vertex
//                 table of the edge-balanced scans
//   k_scan<L,E>   initWL<true>: every thread takes E consecutive CSR entries
//                 (128-bit loads); rows shorter than E stay inside one
//                 thread, longer rows are spread over threads, warps and CTAs
//                 (the reference's thread/warp degree split, :167/:185,
//                 becomes the entries-per-thread E). Also zeroes inMST.
//                 Appends are CTA-aggregated: one atomic per tile.
//   k_rounds      all Boruvka rounds of the phase in one cooperative launch
//                 (kernel1, kernel2, kernel3 per round, bounded grid
//                 barriers, no host round trip per round).
//   k_flatten     parent[v] = root(v) once after the light phase
//   k_scan<H,E>   initWL<false>: keeps heavy entries across light trees
//   k_rounds      heavy phase
#pragma once
#include <cuda_pipeline.h>
#include <cuda_runtime.h>
#include <climits>
#include <stdint.h>

#include "ecl_mst.h"
#include "internal.h"
#include "mst_kernels.cuh"

namespace ecl {

constexpr int kThreads = 512;          // threads of the prep, flatten and round kernels
constexpr int kScanThreads = 256;      // threads of a scan CTA
constexpr int kGran = kScanThreads * 4;// entries per tile->vertex table step
constexpr int kSegCap = 4096;          // vertices of a tile's nindex slice kept in smem
#ifndef ECL_ROUND_EPT
#define ECL_ROUND_EPT 1
#endif
#ifndef ECL_ROUND_MIN_BLOCKS
#define ECL_ROUND_MIN_BLOCKS 4
#endif
constexpr int kEPT = ECL_ROUND_EPT;    // worklist entries per thread in a round tile
constexpr int kHotLog = 9;             // hot representative table: 512 slots
constexpr int kHotSlots = 1 << kHotLog;
constexpr int kFindLog = 10;           // find cache: 1024 slots
constexpr int kFindSlots = 1 << kFindLog;
constexpr int kPairLog = 10;           // parallel-edge table: 1024 slots
constexpr int kPairSlots = 1 << kPairLog;
constexpr u64 kNoPair = ~0ull;
constexpr unsigned long long kBarrierTimeoutNs = 5ull * 1000 * 1000 * 1000;

// Entries per thread of the edge-balanced scan for a degree split: rows
// shorter than the split stay inside one thread.
__host__ __device__ __forceinline__ int scan_ept(int split) {
  return split <= 4 ? 4 : (split <= 8 ? 8 : 16);
}

struct PrepArgs {
  int nodes, edges;
  const int* nindex;
  const int* eweight;
  int* parent;
  u64* minv0;
  u64* minv1;
  int* first_v;  // [tiles + 1]: vertex holding entry t * kGran; last = nodes - 1
  int tiles;     // ceil(edges / kGran)
  int mode, explicit_thr, split;
  float quantile;
  DevState* st;
};

struct ScanArgs {
  int nodes, edges;
  const int* nindex;
  const int* nlist;
  const int* eweight;
  const int* first_v;
  int tiles;
  int* parent;
  int4* wl;
  unsigned wl_cap;
  unsigned char* inMST;
  int vec_ok;    // nlist / eweight 16-byte aligned
  int zero_vec;  // inMST 16-byte aligned
  int sm_count;  // host side: sizes the persistent scan launch
  DevState* st;
};

struct RoundArgs {
  int phase;
  int nodes;
  int4* wl0;
  int4* wl1;
  unsigned wl_cap;
  int* parent;
  u64* minv0;
  u64* minv1;
  unsigned char* inMST;
  DevState* st;
  unsigned small_tail;
  int count_atomics;
};

// ------------------------------------------------------------------ prep
// Threshold rule, by mode (run by one CTA). HEURISTIC restates main's rule
// (ECL_MST.cu:408,432-440); QUANTILE takes a quantile of a 4096-entry hashed
// sample; LEARNED keeps the threshold, filter flag and split the MLP kernel
// already wrote into `st` (from its own sorted sample).
__device__ void choose_threshold(const PrepArgs& a, int* samp) {
  DevState* st = a.st;
  const int tid = threadIdx.x;
  int mode = a.mode, split = a.split;
  float quantile = a.quantile;
  if (mode == ECL_THRESH_LEARNED) {
    if (tid == 0) st->split = st->learned_split;
    return;
  }
  const int nodes = a.nodes, edges = a.edges;
  if (tid == 0) st->split = split;
  if (mode == ECL_THRESH_NONE || (mode == ECL_THRESH_QUANTILE && !(quantile < 1.0f))) {
    if (tid == 0) {
      st->filtered = 0;
      st->threshold = INT_MAX;
    }
    return;
  }
  if (mode == ECL_THRESH_EXPLICIT) {
    if (tid == 0) {
      st->filtered = 1;
      st->threshold = a.explicit_thr;
    }
    return;
  }
  if (mode == ECL_THRESH_HEURISTIC) {
    if (tid == 0) {
      if (edges / nodes < 4) {
        st->filtered = 0;
        st->threshold = INT_MAX;
      } else {
        int s[20];
        const int ns = edges < 20 ? edges : 20;
        for (int i = 0; i < ns; i++) {
          unsigned val = (unsigned)i;
          val = ((val >> 16) ^ val) * 0x45d9f3bu;
          val = ((val >> 16) ^ val) * 0x45d9f3bu;
          val = (val >> 16) ^ val;
          s[i] = a.eweight[val % (unsigned)edges];
        }
        for (int i = 1; i < ns; i++) {
          const int x = s[i];
          int k = i - 1;
          while (k >= 0 && s[k] > x) {
            s[k + 1] = s[k];
            k--;
          }
          s[k + 1] = x;
        }
        st->filtered = 1;
        st->threshold = s[min(19, (int)(3.0 * nodes * ns / edges))];
      }
    }
    return;
  }
  const int S = 4096;
  for (int i = tid; i < S; i += blockDim.x) {
    const uint64_t r = ecl_mix64(0x5EED0000ull + (uint64_t)i);
    samp[i] = a.eweight[(unsigned)(r % (uint64_t)(unsigned)edges)];
  }
  __syncthreads();
  for (int k = 2; k <= S; k <<= 1) {  // bitonic sort in shared memory
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < S; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const int x = samp[i], y = samp[ixj];
          if ((x > y) == ((i & k) == 0)) {
            samp[i] = y;
            samp[ixj] = x;
          }
        }
      }
      __syncthreads();
    }
  }
  if (tid == 0) {
    const float q = quantile < 0.f ? 0.f : quantile;
    int idx = (int)(q * (float)(S - 1));
    idx = idx < 0 ? 0 : (idx > S - 1 ? S - 1 : idx);
    st->filtered = 1;
    st->threshold = samp[idx];
  }
}

// Largest v in [0, nodes) with nindex[v] <= e (bounded even on bad input).
__device__ __forceinline__ int vertex_of(const int* nindex, int nodes, long long e) {
  int lo = 0, hi = nodes;  // invariant: nindex[lo] <= e (for a valid CSR), answer in [lo, hi)
  while (hi - lo > 1) {
    const int mid = lo + ((hi - lo) >> 1);
    if ((long long)__ldg(nindex + mid) <= e) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kThreads) k_prep(PrepArgs a) {
  __shared__ int samp[4096];
  DevState* st = a.st;
  if (blockIdx.x == 0) choose_threshold(a, samp);
  const int n = a.nodes, m = a.edges;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (int v = gid; v < n; v += stride) {
    a.parent[v] = v;
    a.minv0[v] = kNoEdge;
    a.minv1[v] = kNoEdge;
    const int b = __ldg(a.nindex + v), e = __ldg(a.nindex + v + 1);
    bad |= b < 0 || e < b || e > m;
  }
  if (gid == 0) bad |= __ldg(a.nindex) != 0 || __ldg(a.nindex + n) != m;
  if (bad) atomicOr(&st->error, kErrFormat);
  for (int t = gid; t <= a.tiles; t += stride)
    a.first_v[t] = t < a.tiles ? vertex_of(a.nindex, n, (long long)t * kGran) : n - 1;
}

// ------------------------------------------------------------------ scans
enum ScanKind { kLight = 0, kHeavy = 1 };

// Edge-balanced CSR scan (initWL, ECL_MST.cu:157-207). Tile = kThreads * EPT
// consecutive entries; thread t owns entries [tile0 + t*EPT, +EPT). The
// vertex of each entry comes from the tile's slice of nindex in shared memory
// (found through first_v), so hub rows and short rows cost the same per
// entry. One-direction entries (nlist[j] > v) with the phase's weight test
// are appended as {rep(v), rep(n), w, j}; the heavy scan additionally drops
// entries whose endpoints share a light-phase tree (parent[] is flat, so a
// rep is one load).
// Asynchronous global -> shared copies (cp.async) of one tile: the thread's
// own EPT entries of nlist and eweight (16-byte copies when aligned), and a
// cooperative copy of the tile's nindex slice when it fits in shared memory.
template <int EPT>
__device__ __forceinline__ void scan_issue_tile(const ScanArgs& a, long long e0, int v_lo, int span,
                                                int* nl_s, int* ew_s, int* sidx) {
  const int m = a.edges;
  const long long j0 = e0 + (long long)threadIdx.x * EPT;
  int* nl_d = nl_s + threadIdx.x * EPT;
  int* ew_d = ew_s + threadIdx.x * EPT;
  if (a.vec_ok && j0 + EPT <= m) {
#pragma unroll
    for (int q = 0; q < EPT; q += 4) {
      __pipeline_memcpy_async(nl_d + q, a.nlist + j0 + q, 16);
      __pipeline_memcpy_async(ew_d + q, a.eweight + j0 + q, 16);
    }
  } else {
    for (int q = 0; q < EPT && j0 + q < m; q++) {
      __pipeline_memcpy_async(nl_d + q, a.nlist + j0 + q, 4);
      __pipeline_memcpy_async(ew_d + q, a.eweight + j0 + q, 4);
    }
  }
  if (span <= kSegCap)
    for (int i = threadIdx.x; i <= span; i += blockDim.x) __pipeline_memcpy_async(sidx + i, a.nindex + v_lo + i, 4);
  __pipeline_commit();
}

// Persistent, double-buffered: while a CTA decides its current tile from
// shared memory, the next tile's entries and nindex slice are already on
// their way (cp.async), and the first_v pair of the tile after that is in
// registers, so the only serial latency per tile is the reservation.
// Dynamic shared memory of a scan CTA: two stages of (nlist, eweight) tiles
// and two nindex slices.
template <int EPT>
constexpr size_t scan_smem_bytes() {
  return 2 * 2 * (size_t)kScanThreads * EPT * sizeof(int) + 2 * (size_t)(kSegCap + 4) * sizeof(int) +
         (size_t)kScanThreads * EPT * sizeof(int);
}

template <int KIND, int EPT>
__global__ void __launch_bounds__(kScanThreads, EPT == 16 ? 2 : 3) k_scan(ScanArgs a) {
  constexpr int kTile = kScanThreads * EPT;
  constexpr int kStep = EPT / 4;  // first_v entries per tile
  extern __shared__ __align__(16) int scan_dyn[];
  int (*nl_s)[kTile] = reinterpret_cast<int (*)[kTile]>(scan_dyn);
  int (*ew_s)[kTile] = reinterpret_cast<int (*)[kTile]>(scan_dyn + 2 * kTile);
  int (*sidx_s)[kSegCap + 4] = reinterpret_cast<int (*)[kSegCap + 4]>(scan_dyn + 4 * kTile);
  // row-start marks of the current tile: (generation << 13) | (span index + 1)
  int* rmark = scan_dyn + 4 * kTile + 2 * (kSegCap + 4);
  __shared__ unsigned warp_off[kScanThreads / 32];
  __shared__ unsigned tile_base;
  DevState* st = a.st;
  if (ld_volatile(&st->error) & kErrFormat) return;  // set by k_prep only
  if (KIND == kHeavy && !st->filtered) return;
  if (scan_ept(st->split) != EPT) return;  // only the variant the split selects runs
  const int thr = st->threshold;
  const int n = a.nodes, m = a.edges;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ntiles = (int)(((long long)m + kTile - 1) / kTile);
  int t = blockIdx.x;
  if (t >= ntiles) return;
  const int stride = gridDim.x;
  auto first_v = [&](int tile) -> int2 {
    const int tb = tile * kStep;
    return make_int2(__ldg(a.first_v + tb), __ldg(a.first_v + min(tb + kStep, a.tiles)));
  };
  int2 fv_cur = first_v(t);
  int2 fv_nxt = t + stride < ntiles ? first_v(t + stride) : make_int2(0, 0);
  scan_issue_tile<EPT>(a, (long long)t * kTile, fv_cur.x, fv_cur.y - fv_cur.x + 1, nl_s[0], ew_s[0], sidx_s[0]);
  for (int q = threadIdx.x; q < kTile; q += blockDim.x) rmark[q] = 0;  // generation 0 never matches
  int gen = 0;
  __pipeline_wait_prior(0);
  __syncthreads();
  for (int buf = 0; t < ntiles; t += stride, buf ^= 1) {
    const int tn = t + stride;
    if (tn < ntiles)
      scan_issue_tile<EPT>(a, (long long)tn * kTile, fv_nxt.x, fv_nxt.y - fv_nxt.x + 1, nl_s[buf ^ 1],
                           ew_s[buf ^ 1], sidx_s[buf ^ 1]);
    const int2 fv_after = tn + stride < ntiles ? first_v(tn + stride) : make_int2(0, 0);
    const long long e0 = (long long)t * kTile;
    const long long j0 = e0 + (long long)threadIdx.x * EPT;
    const int v_lo = fv_cur.x;
    const int span = fv_cur.y - fv_cur.x + 1;  // vertices whose rows may hold this tile's entries
    const bool seg = span <= kSegCap;
    const int* sidx = sidx_s[buf];
    auto row_start = [&](int i) -> int {  // nindex[v_lo + i]
      return seg ? sidx[i] : __ldg(a.nindex + v_lo + i);
    };
    // the thread's own entries, 128 bits at a time from the staged tile
    int nb[EPT], w[EPT];
    if (j0 + EPT <= m) {
#pragma unroll
      for (int q = 0; q < EPT; q += 4) {
        const int4 x = *reinterpret_cast<const int4*>(&nl_s[buf][threadIdx.x * EPT + q]);
        const int4 y = *reinterpret_cast<const int4*>(&ew_s[buf][threadIdx.x * EPT + q]);
        nb[q] = x.x; nb[q + 1] = x.y; nb[q + 2] = x.z; nb[q + 3] = x.w;
        w[q] = y.x; w[q + 1] = y.y; w[q + 2] = y.z; w[q + 3] = y.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < EPT; q++) {
        const bool in = j0 + q < m;
        nb[q] = in ? nl_s[buf][threadIdx.x * EPT + q] : -1;
        w[q] = in ? ew_s[buf][threadIdx.x * EPT + q] : 0;
      }
    }
    if (KIND == kLight && j0 < m) {  // inMST = 0 (the reference memsets it, :306)
      if (a.zero_vec && j0 + EPT <= m) {
        if (EPT == 4) *reinterpret_cast<unsigned*>(a.inMST + j0) = 0u;
        else if (EPT == 8) *reinterpret_cast<uint2*>(a.inMST + j0) = make_uint2(0u, 0u);
        else *reinterpret_cast<uint4*>(a.inMST + j0) = make_uint4(0u, 0u, 0u, 0u);
      } else {
        for (int q = 0; q < EPT && j0 + q < m; q++) a.inMST[j0 + q] = 0;
      }
    }
    // Vertex of every entry without a per-entry walk: each row starting
    // inside the tile marks its start position with its span index (the
    // largest index wins, so a run of zero-degree rows resolves to the row
    // that owns the entries); an entry's vertex is then the largest mark at
    // or before it, seeded with the vertex of the thread's first entry.
    // (Tiles whose vertex range exceeds the shared slice, i.e. long runs of
    // zero-degree vertices, search each entry in global nindex instead.)
    auto last_row_at_or_before = [&](long long j) -> int {
      int lo = 0, hi = span;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (row_start(mid) <= j) lo = mid;
        else hi = mid;
      }
      return lo;
    };
    gen++;
    if (seg)
      for (int r = 1 + threadIdx.x; r < span; r += blockDim.x) {
        const long long p = (long long)sidx[r] - e0;
        if (p > 0 && p < kTile) atomicMax(&rmark[p], (gen << 13) | (r + 1));
      }
    const int i0 = j0 < m ? last_row_at_or_before(j0) : 0;  // vertex of entry j0
    __syncthreads();
    int vi[EPT];
    if (seg) {
      int run = i0;
#pragma unroll
      for (int q = 0; q < EPT; q += 4) {
        const int4 mk = *reinterpret_cast<const int4*>(&rmark[threadIdx.x * EPT + q]);
        const int c[4] = {mk.x, mk.y, mk.z, mk.w};
#pragma unroll
        for (int u = 0; u < 4; u++) {
          if ((c[u] >> 13) == gen) run = max(run, (c[u] & 8191) - 1);
          vi[q + u] = run;
        }
      }
    } else {
#pragma unroll
      for (int q = 0; q < EPT; q++) vi[q] = j0 + q < m ? last_row_at_or_before(j0 + q) : 0;
    }
    int vtx[EPT], nrep[EPT];
    unsigned keep = 0, cnt = 0;
    int cur_v = -1, cur_rep = -1;
#pragma unroll
    for (int q = 0; q < EPT; q++) {
      const long long j = j0 + q;
      vtx[q] = 0;
      nrep[q] = nb[q];
      if (j >= m) continue;
      const int v = v_lo + vi[q];
      if ((unsigned)nb[q] >= (unsigned)n) {
        atomicOr(&st->error, kErrFormat);
        continue;
      }
      if (nb[q] <= v) continue;
      if (KIND == kLight ? !(w[q] <= thr) : !(w[q] > thr)) continue;
      int rv = v;
      if (KIND == kHeavy) {
        if (v != cur_v) {
          cur_v = v;
          cur_rep = __ldg(a.parent + v);
        }
        rv = cur_rep;
        nrep[q] = __ldg(a.parent + nb[q]);
        if (nrep[q] == rv) continue;
      }
      vtx[q] = rv;
      keep |= 1u << q;
      cnt++;
    }
    // Tile reservation. Its two barriers double as the pipeline's: before
    // the first, every thread has finished reading this tile's stage and has
    // waited for its own copies of the next tile, so after it the next stage
    // is complete and this one may be refilled.
    unsigned incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += x;
    }
    if (lane == 31) warp_off[warp] = incl;
    __pipeline_wait_prior(0);
    __syncthreads();
    if (warp == 0) {
      constexpr int nw = kScanThreads / 32;
      const unsigned w0 = lane < nw ? warp_off[lane] : 0u;
      unsigned x0 = w0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned x = __shfl_up_sync(0xffffffffu, x0, o);
        if (lane >= o) x0 += x;
      }
      if (lane < nw) warp_off[lane] = x0 - w0;
      if (lane == 31) tile_base = x0 ? atomicAdd(&st->wl_count[KIND][0], x0) : 0u;
    }
    __syncthreads();
    unsigned pos = tile_base + warp_off[warp] + (incl - cnt);
#pragma unroll
    for (int q = 0; q < EPT; q++) {
      if (!(keep & (1u << q))) continue;
      if (pos < a.wl_cap) a.wl[pos] = make_int4(vtx[q], nrep[q], w[q], (int)(j0 + q));
      else atomicOr(&st->error, kErrOverflow);
      pos++;
    }
    fv_cur = fv_nxt;
    fv_nxt = fv_after;
  }
}

// parent[v] = root(v) for every vertex, once before the heavy scan.
__global__ void __launch_bounds__(kThreads) k_flatten(int* parent, int n, const DevState* st) {
  if (!st->filtered || (ld_volatile(&st->error) & (kErrFormat | kErrTimeout))) return;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    __stcg(parent + v, find_ro(v, parent));
}

// ----------------------------------------------------------------- rounds
// Per-CTA shared-memory state of the round kernel. Representatives shared by
// many worklist entries (a growing giant component) would otherwise put
// every entry's parent read, min-slot guard read, atomicMin and reset on one
// L2 address; these small direct-mapped tables absorb the repeats per CTA.
struct RoundSmem {
  ReserveSmem rs;
  int hot_rep[kHotSlots];    // hot representative -> CTA-local partial minimum
  u64 hot_key[kHotSlots];
  int reset_seen[kHotSlots]; // previous-round slots this CTA already cleared
  u64 find_cache[kFindSlots];// (vertex << 32) | root, valid within one pass
  u64 pair_tag[kPairSlots];  // (lo rep << 32) | hi rep of a tile's cross entry
  u64 pair_min[kPairSlots];  // smallest key of that rep pair within the tile
};

__device__ __forceinline__ unsigned hot_slot(int r) { return ((unsigned)r * 0x9E3779B1u) >> (32 - kHotLog); }
__device__ __forceinline__ unsigned find_slot(int r) { return ((unsigned)r * 0x85EBCA6Bu) >> (32 - kFindLog); }

__device__ __forceinline__ void round_smem_clear(RoundSmem& s) {
  for (int i = threadIdx.x; i < kHotSlots; i += blockDim.x) {
    s.hot_rep[i] = -1;
    s.hot_key[i] = kNoEdge;
    s.reset_seen[i] = -1;
  }
  for (int i = threadIdx.x; i < kFindSlots; i += blockDim.x) s.find_cache[i] = kNoEdge;
  for (int i = threadIdx.x; i < kPairSlots; i += blockDim.x) {
    s.pair_tag[i] = kNoPair;
    s.pair_min[i] = kNoEdge;
  }
}

__device__ __forceinline__ unsigned pair_slot(u64 pk) {
  return (unsigned)((pk * 0x9E3779B97F4A7C15ull) >> (64 - kPairLog));
}

// Parallel-edge elimination in the contracted graph, fused with the tile's
// worklist reservation. Entries of one tile that join the same two trees are
// parallel edges of the contracted graph; only the one with the smallest
// (weight, j) key can be a forest edge (any forest through a heavier one is
// heavier than the same forest through the lightest), so the others are
// dropped for good. Warp groups with equal rep pairs reduce first; group
// minima meet in a per-tile shared table. keep[k] is narrowed to the
// survivors, and *pos receives the first output slot of this thread's
// survivors (one global atomic per CTA tile). Three CTA barriers in all.
// Every thread of the CTA must call this.
template <int E>
__device__ __forceinline__ void drop_parallel_reserve(const int4 (&e)[E], bool (&keep)[E],
                                                      unsigned* ctr, RoundSmem& s, unsigned* pos) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u64 pk[E], gmin[E];
#pragma unroll
  for (int k = 0; k < E; k++) {
    const unsigned lo = (unsigned)min(e[k].x, e[k].y), hi = (unsigned)max(e[k].x, e[k].y);
    pk[k] = keep[k] ? (((u64)lo << 32) | hi) : (0xFFFFFFFF00000000ull | (threadIdx.x * E + k));
    const u64 key = edge_key(e[k].z, e[k].w);
    gmin[k] = key;
#ifndef ECL_NO_DEDUP
    const unsigned g = __match_any_sync(0xffffffffu, pk[k]);
    if (!keep[k]) continue;
    if (g & (g - 1)) {
      const unsigned khi = (unsigned)(key >> 32);
      const unsigned mhi = __reduce_min_sync(g, khi);
      const unsigned mlo = __reduce_min_sync(g, khi == mhi ? (unsigned)key : 0xffffffffu);
      gmin[k] = ((u64)mhi << 32) | mlo;
    }
    if (lane == __ffs(g) - 1) {
      const unsigned slot = pair_slot(pk[k]);
      u64 t = ((volatile u64*)s.pair_tag)[slot];
      if (t == kNoPair) {
        t = atomicCAS(&s.pair_tag[slot], kNoPair, pk[k]);
        if (t == kNoPair) t = pk[k];
      }
      if (t == pk[k] && ((volatile u64*)s.pair_min)[slot] > gmin[k]) atomicMin(&s.pair_min[slot], gmin[k]);
    }
#endif
  }
  __syncthreads();  // S1: the tile's pair table is complete
  unsigned cnt = 0;
#pragma unroll
  for (int k = 0; k < E; k++) {
#ifndef ECL_NO_DEDUP
    if (keep[k]) {
      const unsigned slot = pair_slot(pk[k]);
      const u64 key = edge_key(e[k].z, e[k].w);
      const u64 best = s.pair_tag[slot] == pk[k] ? s.pair_min[slot] : gmin[k];
      keep[k] = key == best;
    }
#endif
    cnt += keep[k];
  }
  unsigned incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) s.rs.warp_off[warp][0] = incl;
  __syncthreads();  // S2: every check done, warp totals written
  for (int i = threadIdx.x; i < kPairSlots; i += blockDim.x) {
    s.pair_tag[i] = kNoPair;
    s.pair_min[i] = kNoEdge;
  }
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    const unsigned w0 = lane < nw ? s.rs.warp_off[lane][0] : 0u;
    unsigned x0 = w0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, x0, o);
      if (lane >= o) x0 += t;
    }
    if (lane < nw) s.rs.warp_off[lane][0] = x0 - w0;
    if (lane == 31) s.rs.base[0] = x0 ? atomicAdd(ctr, x0) : 0u;
  }
  __syncthreads();  // S3: offsets and the tile's base are published
  *pos = s.rs.base[0] + s.rs.warp_off[warp][0] + (incl - cnt);
}

// Roots of the 2*kEPT endpoints a thread holds, all walks advanced in lock
// step so their loads are in flight together. A per-CTA cache of
// (vertex << 32 | root) absorbs repeated endpoints (roots do not change
// during the find/min pass). Path splitting re-points each visited node to
// its grandparent (stays inside the tree; bounds long hook chains).
template <int N>
__device__ __forceinline__ void multi_find(int (&v)[N], const bool (&valid)[N], int* parent,
                                           RoundSmem& s) {
  int par[N];
  unsigned miss = 0;
#pragma unroll
  for (int i = 0; i < N; i++) {
    par[i] = v[i];
    if (!valid[i]) continue;
    const u64 c = ((volatile u64*)s.find_cache)[find_slot(v[i])];
#ifdef ECL_NO_FINDCACHE
    if (false) {
#else
    if ((int)(c >> 32) == v[i] && c != kNoEdge) {
#endif
      v[i] = (int)(unsigned)c;
      par[i] = v[i];
    } else {
      miss |= 1u << i;
      par[i] = __ldcg(parent + v[i]);
    }
  }
  int orig[N];
#pragma unroll
  for (int i = 0; i < N; i++) orig[i] = v[i];
  for (;;) {
    int gp[N];
    bool any = false;
#pragma unroll
    for (int i = 0; i < N; i++) {
      gp[i] = par[i];
      if (par[i] != v[i]) {
        any = true;
        gp[i] = __ldcg(parent + par[i]);
      }
    }
    if (!any) break;
#pragma unroll
    for (int i = 0; i < N; i++) {
      if (par[i] != v[i]) {
#ifndef ECL_NO_SPLIT
        if (gp[i] != par[i]) __stcg(parent + v[i], gp[i]);
#endif
        v[i] = par[i];
        par[i] = gp[i];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < N; i++)
    if (miss & (1u << i))
      ((volatile u64*)s.find_cache)[find_slot(orig[i])] = ((u64)(unsigned)orig[i] << 32) | (unsigned)v[i];
}

// Clear a previous-round min slot once per CTA.
__device__ __forceinline__ void reset_prev(int r, u64* mprev, RoundSmem& s) {
  const unsigned slot = hot_slot(r);
  if (((volatile int*)s.reset_seen)[slot] == r) return;
  ((volatile int*)s.reset_seen)[slot] = r;
  __stcg(mprev + r, kNoEdge);
}

// Offer each of a thread's N (rep, key) pairs to the rep's min slot: the
// guarded atomicMin of ECL_MST.cu:221-223. Lanes of a warp holding the same
// rep first reduce to the group minimum (warp-cooperative for high-degree
// representatives); a group leader then folds it into the CTA's hot table.
// Singletons, and leaders whose table slot belongs to another rep, read the
// global slots together (one round trip for all pairs) and issue
// fire-and-forget atomicMin only where the guard shows an improvement.
// Every lane of the warp must call this.
template <int N>
__device__ __forceinline__ void offer_mins(const int (&rep)[N], const u64 (&key)[N],
                                           const bool (&valid)[N], u64* mcur, RoundSmem& s,
                                           unsigned long long& atomics) {
  const int lane = threadIdx.x & 31;
  bool cold[N];
  u64 val[N];
#pragma unroll
  for (int i = 0; i < N; i++) {
    const unsigned g = __match_any_sync(0xffffffffu, valid[i] ? rep[i] : -2 - lane);
    cold[i] = false;
    val[i] = key[i];
    if (!valid[i]) continue;
#ifdef ECL_NO_HOT
    if (true) {
#else
    if ((g & (g - 1)) == 0) {
#endif
      cold[i] = true;
      continue;
    }
    const unsigned khi = (unsigned)(key[i] >> 32);
    const unsigned hi = __reduce_min_sync(g, khi);
    const unsigned lo = __reduce_min_sync(g, khi == hi ? (unsigned)key[i] : 0xffffffffu);
    if (lane != __ffs(g) - 1) continue;
    const u64 gm = ((u64)hi << 32) | lo;
    const unsigned slot = hot_slot(rep[i]);
    int cur = ((volatile int*)s.hot_rep)[slot];
    if (cur < 0) {
      cur = atomicCAS(&s.hot_rep[slot], -1, rep[i]);
      if (cur < 0) cur = rep[i];
    }
    if (cur == rep[i]) {
      if (((volatile u64*)s.hot_key)[slot] > gm) atomicMin(&s.hot_key[slot], gm);
    } else {
      cold[i] = true;
      val[i] = gm;
    }
  }
  u64 seen[N];
#pragma unroll
  for (int i = 0; i < N; i++) seen[i] = cold[i] ? __ldcg(mcur + rep[i]) : 0ull;
#pragma unroll
  for (int i = 0; i < N; i++) {
    if (cold[i] && seen[i] > val[i]) {
      atomicMin(mcur + rep[i], val[i]);
      atomics++;
    }
  }
}

// kernel1 (ECL_MST.cu:210-226) plus kernel3 of the previous round (:243-251):
// each input entry clears its endpoints' slots in the previous round's min
// array, resolves its endpoints to reps, and if they differ is compacted into
// `out` with the reps (implicit path compression, :218-219) and offers its
// key to both reps' min slots.
__device__ __forceinline__ void round_find_min(const RoundArgs& a, const int4* in, unsigned W,
                                               int4* out, unsigned* out_ctr, u64* mcur, u64* mprev,
                                               bool reset, unsigned start, unsigned stride,
                                               RoundSmem& s) {
  constexpr int N = 2 * kEPT;
  const unsigned tile = blockDim.x * kEPT;
  const unsigned ntiles = (W + tile - 1) / tile;
  unsigned long long atomics = 0;
  for (unsigned t = start; t < ntiles; t += stride) {
    int4 e[kEPT];
    bool in_range[kEPT];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      const unsigned idx = t * tile + k * blockDim.x + threadIdx.x;
      in_range[k] = idx < W;
      e[k] = in_range[k] ? __ldcg(in + idx) : make_int4(0, 0, 0, 0);
    }
    int v[N];
    bool vv[N];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      v[2 * k] = e[k].x;
      v[2 * k + 1] = e[k].y;
      vv[2 * k] = vv[2 * k + 1] = in_range[k];
      if (reset && in_range[k]) {
        reset_prev(e[k].x, mprev, s);
        reset_prev(e[k].y, mprev, s);
      }
    }
    multi_find<N>(v, vv, a.parent, s);
    bool keep[kEPT];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      keep[k] = in_range[k] && v[2 * k] != v[2 * k + 1];
      e[k].x = v[2 * k];
      e[k].y = v[2 * k + 1];
    }
    unsigned pos;
    drop_parallel_reserve<kEPT>(e, keep, out_ctr, s, &pos);
    u64 key[N];
    bool kv[N];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      if (keep[k]) {
        if (pos < a.wl_cap) out[pos] = e[k];
        else atomicOr(&a.st->error, kErrOverflow);
        pos++;
      }
      key[2 * k] = key[2 * k + 1] = edge_key(e[k].z, e[k].w);
      kv[2 * k] = kv[2 * k + 1] = keep[k];
    }
    offer_mins<N>(v, key, kv, mcur, s, atomics);
  }
  __syncthreads();
  // flush the CTA's partial minima of hot representatives
  for (int i = threadIdx.x; i < kHotSlots; i += blockDim.x) {
    const int r = s.hot_rep[i];
    if (r >= 0) {
      const u64 k = s.hot_key[i];
      if (__ldcg(mcur + r) > k) {
        atomicMin(mcur + r, k);
        atomics++;
      }
    }
  }
  if (a.count_atomics && atomics) atomicAdd(&a.st->atomics, atomics);
}

// After the barrier: the hot table's reps now read their final minima.
__device__ __forceinline__ void hot_refresh(const u64* mcur, RoundSmem& s) {
  for (int i = threadIdx.x; i < kHotSlots; i += blockDim.x) {
    const int r = s.hot_rep[i];
    if (r >= 0) s.hot_key[i] = __ldcg(mcur + r);
  }
  __syncthreads();
}

// kernel2 (ECL_MST.cu:229-240): an entry whose key is the minimum of either
// endpoint's slot is a forest edge: union the trees and mark inMST[j].
__device__ __forceinline__ void round_mark(const RoundArgs& a, const int4* wl, unsigned W,
                                           const u64* mcur, unsigned start, unsigned stride,
                                           const RoundSmem& s) {
  const unsigned tile = blockDim.x * kEPT;
  const unsigned ntiles = (W + tile - 1) / tile;
  for (unsigned t = start; t < ntiles; t += stride) {
    int4 e[kEPT];
    bool in_range[kEPT];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      const unsigned idx = t * tile + k * blockDim.x + threadIdx.x;
      in_range[k] = idx < W;
      e[k] = in_range[k] ? __ldcg(wl + idx) : make_int4(0, 0, 0, 0);
    }
    u64 mx[kEPT], my[kEPT];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      mx[k] = my[k] = kNoEdge;
      if (!in_range[k]) continue;
      const unsigned sx = hot_slot(e[k].x), sy = hot_slot(e[k].y);
      mx[k] = s.hot_rep[sx] == e[k].x ? s.hot_key[sx] : __ldcg(mcur + e[k].x);
      my[k] = s.hot_rep[sy] == e[k].y ? s.hot_key[sy] : __ldcg(mcur + e[k].y);
    }
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      if (!in_range[k]) continue;
      const u64 key = edge_key(e[k].z, e[k].w);
      if (key == mx[k] || key == my[k]) {
        cas_union(e[k].x, e[k].y, a.parent);
        a.inMST[e[k].w] = 1;
      }
    }
  }
}

__global__ void __launch_bounds__(kThreads, ECL_ROUND_MIN_BLOCKS) k_rounds(RoundArgs a) {
  __shared__ RoundSmem s;
  DevState* st = a.st;
  const int ph = a.phase;
  if (ph == 1 && !st->filtered) return;
  // Only bits no CTA of this kernel can set, so every CTA takes the same exit.
  if (ld_volatile(&st->error) & (kErrFormat | kErrTimeout)) return;
  round_smem_clear(s);
  __syncthreads();
  bool tail = false;
  int r = 0;
  const bool stamp = blockIdx.x == 0 && threadIdx.x == 0;
  if (stamp) st->t_round_start[ph] = globaltimer_ns();
  for (;;) {
    const unsigned W = min(ld_volatile(&st->wl_count[ph][r]), a.wl_cap);
    if (W == 0) break;
    if (r >= ECL_MAX_ROUNDS) {
      if (stamp) atomicOr(&st->error, kErrRounds);
      break;
    }
    if (!tail && W <= a.small_tail) {
      tail = true;
      if (blockIdx.x != 0) return;
    }
    const unsigned start = tail ? 0u : blockIdx.x, stride = tail ? 1u : gridDim.x;
    const bool odd = (r & 1) != 0;
    const int4* in = odd ? a.wl1 : a.wl0;
    int4* out = odd ? a.wl0 : a.wl1;
    u64* mcur = odd ? a.minv1 : a.minv0;
    u64* mprev = odd ? a.minv0 : a.minv1;
    round_find_min(a, in, W, out, &st->wl_count[ph][r + 1], mcur, mprev, r > 0, start, stride, s);
    if (tail) __syncthreads();
    else if (!grid_barrier(st, kBarrierTimeoutNs)) return;
    if (stamp) st->t_round[ph][2 * r] = globaltimer_ns();
    const unsigned W2 = min(ld_volatile(&st->wl_count[ph][r + 1]), a.wl_cap);
    r++;
    if (W2 == 0) break;
    hot_refresh(mcur, s);
    round_mark(a, out, W2, mcur, start, stride, s);
    __syncthreads();
    round_smem_clear(s);
    if (tail) __syncthreads();
    else if (!grid_barrier(st, kBarrierTimeoutNs)) return;
    if (stamp) st->t_round[ph][2 * r - 1] = globaltimer_ns();
  }
  if (stamp) st->rounds[ph] = r;
}

}  // namespace ecl
