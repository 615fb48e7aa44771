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
//   k_scan<L,E>   initWL<true>: a producer warp stages CSR tiles into shared
//                 memory with bulk asynchronous copies; every consumer lane
//                 takes E consecutive entries, so rows shorter than E stay
//                 inside one lane and longer rows are spread over lanes,
//                 warps and CTAs (the reference's thread/warp degree split,
//                 :167/:185, becomes the entries-per-lane E). Also zeroes
//                 inMST. Appends are warp-aggregated, reserved in chunks.
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

constexpr int kThreads = 512;          // threads of the prep, flatten and batch kernels
constexpr int kGran = 128;             // entries per tile->vertex table step (the smallest scan warp range)
// Round CTAs of 1024 threads, two per SM (measured on RMAT-22: 2.4 % faster
// with the learned schedule and 4.6 % with the heuristic one than 512 x 4;
// 256 x 8 was 11-15 % slower)
#ifndef ECL_ROUND_THREADS
#define ECL_ROUND_THREADS 1024
#endif
#ifndef ECL_ROUND_MIN_BLOCKS
#define ECL_ROUND_MIN_BLOCKS 2
#endif
#ifndef ECL_FIND_LOG
#define ECL_FIND_LOG 10
#endif
#ifndef ECL_PAIR_LOG
#define ECL_PAIR_LOG 10
#endif
constexpr int kRoundThreads = ECL_ROUND_THREADS;  // threads of a round CTA (one worklist entry each per tile)
#ifndef ECL_ROUND_EPT
#define ECL_ROUND_EPT 1
#endif
constexpr int kEPT = ECL_ROUND_EPT;    // worklist entries per thread in a round tile
constexpr int kHotLog = 9;             // hot representative table: 512 slots
constexpr int kHotSlots = 1 << kHotLog;
constexpr int kFindLog = ECL_FIND_LOG; // find cache
constexpr int kFindSlots = 1 << kFindLog;
constexpr int kPairLog = ECL_PAIR_LOG; // parallel-edge table
constexpr int kPairSlots = 1 << kPairLog;
constexpr u64 kNoPair = ~0ull;
constexpr int kSplitAfter = 8;         // find steps before path splitting starts
// Rounds whose worklist holds at least ECL_FLAT_ROUNDS x n entries first
// point every vertex at its root, so their finds are single loads (RMAT-22:
// 11 % faster with the reference heuristic's schedule, 1 % with the learned
// one; flattening from W >= n already was slower than from W >= 2n)
#ifndef ECL_FLAT_ROUNDS
#define ECL_FLAT_ROUNDS 2
#endif
#ifndef ECL_L2_HINTS
#define ECL_L2_HINTS 1                 // evict-first CSR streams, evict-last parent gathers in the scans
#endif
// Entries per lane of the heavy scan: 0 takes the light scan's (the split's),
// 4, 8 or 16 fixes it. Its parent[] gathers make the heavy scan latency-bound,
// and E = 4 runs the most consumer warps per SM (4 CTAs of 8): measured on
// RMAT-25 11.6 % faster than the split's E = 8 (RMAT-22 4.6 %), no slower on
// ER, grid or RGG graphs.
#ifndef ECL_HEAVY_EPT
#define ECL_HEAVY_EPT 4
#endif
constexpr unsigned long long kBarrierTimeoutNs = 5ull * 1000 * 1000 * 1000;

// Entries per thread of the edge-balanced scan for a degree split: rows
// shorter than the split stay inside one thread.
__host__ __device__ __forceinline__ int scan_ept(int split) {
  return split <= 4 ? 4 : (split <= 8 ? 8 : 16);
}

// Entries per lane of the heavy scan (ECL_HEAVY_EPT, else the split's).
__host__ __device__ __forceinline__ int heavy_ept(int split) {
  return ECL_HEAVY_EPT ? ECL_HEAVY_EPT : scan_ept(split);
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
  FeatAcc* feat;  // learned schedule: degree statistics gathered here, else null
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
  unsigned wl_slack;  // host side: wl_cap minus the most entries a scan can keep
  unsigned chunk;     // worklist slots a warp reserves at once (set at launch)
  int ids;            // 1 = append CSR indices (int) instead of tuples (kAblNoTuples)
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
  unsigned abl;  // kAbl* bits: techniques switched off to measure what they buy
  int min_tiles;  // keep one CTA per this many tiles of a round (0 = every CTA)
  // kAblNoTuples: the CSR and the vertex of every entry
  const int* nlist;
  const int* eweight;
  const int* slist;
};

// Ablation switches of the round kernel (mst_opts flags ECL_FLAG_NO_*).
enum : unsigned {
  kAblNoGuards = 1u,     // atomicMin without first reading the slot (ECL_MST.cu:222-223)
  kAblNoCoop = 2u,       // no warp reduction or CTA table for shared reps
  kDedup = 4u,           // parallel-edge elimination on (opt-in: measured slower on RMAT)
  kAblNoFindCache = 8u,  // no per-CTA root cache in the finds
  // The reference's later deoptimization steps, restated so that the forest
  // stays the reference's (one direction is kept):
  kAblNoIPC = 16u,     // NoImplicitPathCompression: compacted entries keep their
                       // endpoints, finds split paths from the first step and
                       // the mark pass finds again
                       // (ECL_MST_..._NoImplicitPathCompression.cu:121-133, 193-216)
  kAblNoTuples = 32u,  // NoTuples: worklists hold CSR indices; endpoints and
                       // weight are gathered every round (..._NoTuples.cu)
  kAblNoDD = 64u,      // NoDataDriven: every round reads the phase's whole list
                       // and nothing is compacted; the rounds end when no entry
                       // joins two trees (..._NoDataDriven.cu:166-180, 263-270)
};
// Switches under which worklist entries keep their endpoints (no rewrite to reps)
constexpr unsigned kAblKeepEnds = kAblNoIPC | kAblNoTuples | kAblNoDD;

// ------------------------------------------------------------------ prep
// Threshold rule, by mode (run by one CTA). HEURISTIC restates main's rule
// (ECL_MST.cu:408,432-440); QUANTILE takes a quantile of a 4096-entry hashed
// sample; LEARNED leaves the threshold, filter flag and split to the MLP
// kernel (k_mlp_apply, which runs beside this kernel on another stream and
// takes them from its own sorted sample).
__device__ void choose_threshold(const PrepArgs& a, int* samp) {
  DevState* st = a.st;
  const int tid = threadIdx.x;
  int mode = a.mode, split = a.split;
  float quantile = a.quantile;
  if (mode == ECL_THRESH_LEARNED) return;
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

__global__ void __launch_bounds__(kThreads) k_prep(PrepArgs a) {
  __shared__ int samp[4096];
  DevState* st = a.st;
  if (blockIdx.x == 0) choose_threshold(a, samp);
  const int n = a.nodes, m = a.edges;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  bool bad = false;
  FeatPart fp;  // degree statistics (learned schedule)
  for (int v = gid; v < n; v += stride) {
    a.parent[v] = v;
    a.minv0[v] = kNoEdge;
    a.minv1[v] = kNoEdge;
    const int b = __ldg(a.nindex + v), e = __ldg(a.nindex + v + 1);
    const bool row_bad = b < 0 || e < b || e > m;
    bad |= row_bad;
    if (a.feat) fp.add(e > b ? (unsigned)(e - b) : 0u);
    // Tile->vertex table (first_v[t] = row of entry t * kGran), first step:
    // the row holding the first step position at or after its start writes
    // itself there (each position has exactly one owner, so no conflicts);
    // the positions further inside long rows stay 0 and are filled by a max
    // scan (k_fill_chunks, k_fill_carry), rows being in increasing order.
    const unsigned t0 = ((unsigned)b + kGran - 1) / kGran, t1 = ((unsigned)e + kGran - 1) / kGran;
    if (!row_bad && t0 < t1) a.first_v[t0] = v;
  }
  if (gid == 0) bad |= __ldg(a.nindex) != 0 || __ldg(a.nindex + n) != m;
  if (bad) atomicOr(&st->error, kErrFormat);
  if (a.feat) fp.fold<kThreads>(a.feat);  // uniform across the grid
}

// Inclusive max scan of the tile->vertex table first_v[0 .. tiles), in
// chunks of kFillChunk entries: each CTA scans its chunk and records the
// chunk's maximum; k_fill_carry then raises every chunk to the maximum of the
// chunks before it and writes the end sentinel first_v[tiles] = nodes - 1.
constexpr int kFillChunk = 8192;  // 1024 threads x 8 entries

__global__ void __launch_bounds__(1024) k_fill_chunks(int* t, int count, int* chunk_max) {
  __shared__ int warp_max[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long base = (long long)blockIdx.x * kFillChunk + threadIdx.x * 8;
  int x[8], run = 0;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    x[q] = base + q < count ? t[base + q] : 0;
    run = max(run, x[q]);
    x[q] = run;
  }
  int incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl = max(incl, y);
  }
  if (lane == 31) warp_max[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = warp_max[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w = max(w, y);
    }
    warp_max[lane] = w;
  }
  __syncthreads();
  int before = __shfl_up_sync(0xffffffffu, incl, 1);
  if (lane == 0) before = 0;
  if (warp > 0) before = max(before, warp_max[warp - 1]);
#pragma unroll
  for (int q = 0; q < 8; q++)
    if (base + q < count) t[base + q] = max(x[q], before);
  if (threadIdx.x == 0) chunk_max[blockIdx.x] = warp_max[31];
}

__global__ void __launch_bounds__(1024) k_fill_carry(int* t, int count, const int* chunk_max, int nodes) {
  __shared__ int carry;
  if (threadIdx.x < 32) {
    int c = 0;
    for (int i = threadIdx.x; i < (int)blockIdx.x; i += 32) c = max(c, chunk_max[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c = max(c, __shfl_xor_sync(0xffffffffu, c, o));
    if (threadIdx.x == 0) carry = c;
  }
  __syncthreads();
  const long long base = (long long)blockIdx.x * kFillChunk;
  if (carry > 0)
    for (int q = threadIdx.x; q < kFillChunk && base + q < count; q += blockDim.x)
      t[base + q] = max(t[base + q], carry);
  if (blockIdx.x == 0 && threadIdx.x == 0) t[count] = nodes - 1;
}

// ------------------------------------------------------------------ scans
enum ScanKind { kLight = 0, kHeavy = 1 };

// Edge-balanced CSR scan (initWL, ECL_MST.cu:157-207), warp-specialised and
// persistent. A tile is kScanWarps * 32 * EPT consecutive CSR entries. One
// producer warp stages each tile's slices of nlist, eweight and nindex into a
// ring of shared-memory stages with bulk asynchronous copies (cp.async.bulk;
// completion counted on the stage's `full` mbarrier) and refills a stage once
// every consumer warp has released it (`empty` mbarrier). Each consumer warp
// takes 32 * EPT consecutive entries of the staged tile, EPT per lane, so hub
// rows and short rows cost the same per entry (the reference's thread / warp
// degree split, :167/:185, becomes the entries-per-lane EPT). A consumer
// finds the vertex of its entries from the staged nindex slice alone: a
// 32-ary search for the row holding the warp's first entry, the rows starting
// inside the warp's range marked in a warp-private array, and a warp max-scan
// over the marks; no step waits on the whole CTA. One-direction entries
// (nlist[j] > v) passing the phase's weight test are appended as
// {rep(v), rep(n), w, j}; the heavy scan also drops entries whose endpoints
// share a light-phase tree (parent[] is flat, so a rep is one load).
// Worklist slots are reserved per warp, `chunk` at a time, from the phase's
// counter; the unused tail of each warp's last chunk is filled with null
// entries (x = -1), which the first round skips.
constexpr int kScanWarps = 8;                        // consumer warps of a scan CTA
constexpr int kScanThreads = (kScanWarps + 1) * 32;  // plus the producer warp
#ifndef ECL_SCAN_SEGCAP
#define ECL_SCAN_SEGCAP 2048
#endif
constexpr int kScanSegCap = ECL_SCAN_SEGCAP;         // longest nindex slice (vertices) staged per tile
constexpr unsigned kScanMaxChunk = 64;               // worklist slots a warp reserves at once

// ring stages and the resident CTAs per SM the launch bounds ask for, per EPT
#ifndef ECL_SCAN_S4
#define ECL_SCAN_S4 2
#endif
#ifndef ECL_SCAN_S8
#define ECL_SCAN_S8 2
#endif
#ifndef ECL_SCAN_S16
#define ECL_SCAN_S16 2
#endif
#ifndef ECL_SCAN_B4
#define ECL_SCAN_B4 4
#endif
#ifndef ECL_SCAN_B8
#define ECL_SCAN_B8 3
#endif
#ifndef ECL_SCAN_B16
#define ECL_SCAN_B16 2
#endif
constexpr int kScanStages[3] = {ECL_SCAN_S4, ECL_SCAN_S8, ECL_SCAN_S16};
constexpr int kScanMinB[3] = {ECL_SCAN_B4, ECL_SCAN_B8, ECL_SCAN_B16};

template <int EPT>
struct ScanCfg {
  static constexpr int kIdx = EPT == 4 ? 0 : (EPT == 8 ? 1 : 2);
  static constexpr int kTile = kScanWarps * 32 * EPT;  // entries per tile
  static constexpr int kStages = kScanStages[kIdx];
  static constexpr int kMinBlocks = kScanMinB[kIdx];
  static constexpr int kSegInts = kScanSegCap + 8;         // slice from a 16-byte boundary
  static constexpr int kStageInts = 2 * kTile + kSegInts;  // nlist, eweight, nindex slice
  static constexpr size_t kHead = 128 + 48 * kStages;      // mbarriers, then stage headers
  // stages, then one row-mark array of 32 * EPT ints per consumer warp
  static constexpr size_t kSmem = kHead + sizeof(int) * ((size_t)kStages * kStageInts + kTile);
};

template <int EPT>
constexpr size_t scan_smem_bytes() {
  return ScanCfg<EPT>::kSmem;
}

struct ScanStage {
  int v_lo;  // vertex holding the tile's first entry
  int span;  // vertices v_lo .. v_lo + span - 1 may own the tile's entries
  int off;   // nindex[v_lo] is at slice index off
  int seg;   // 1 = nindex[v_lo .. v_lo + span] is staged
  int wfirst[kScanWarps];  // vertex holding each consumer warp's first entry
};
static_assert(sizeof(ScanStage) == 48, "stage header size");

// Largest v in [lo, lo + span) with nindex[v] <= e, for an entry e of a tile
// whose rows are v_lo .. v_lo + span - 1 (global binary search; used when the
// tile's slice is too long to stage).
__device__ __forceinline__ int vertex_in(const int* nindex, int lo, int span, long long e) {
  int hi = lo + span;
  while (hi - lo > 1) {
    const int mid = lo + ((hi - lo) >> 1);
    if ((long long)__ldg(nindex + mid) <= e) lo = mid;
    else hi = mid;
  }
  return lo;
}

// The tiles a scan CTA takes, in order: first, first + step, ... < end.
struct TileSeq {
  int first, step, end;
};
__device__ __forceinline__ TileSeq scan_tiles(int ntiles) {
#ifdef ECL_SCAN_CONTIG
  const int g = gridDim.x, b = blockIdx.x, per = ntiles / g, rem = ntiles % g;
  const int first = b * per + min(b, rem);
  return TileSeq{first, 1, first + per + (b < rem ? 1 : 0)};
#else
  return TileSeq{(int)blockIdx.x, (int)gridDim.x, ntiles};
#endif
}

// Producer warp: fills stage i % kStages with the CTA's i-th tile. The
// 16-byte aligned bulk of each slice goes by bulk copy; a ragged end (the
// last tile, the end of nindex) or unaligned arrays go by plain copies of the
// warp's lanes, published by the same mbarrier arrival.
template <int EPT>
__device__ void scan_produce(const ScanArgs& a, unsigned char* smem, int ntiles) {
  using C = ScanCfg<EPT>;
  u64* full = reinterpret_cast<u64*>(smem);
  u64* empty = full + C::kStages;
  ScanStage* hdr = reinterpret_cast<ScanStage*>(smem + 128);
  int* stages = reinterpret_cast<int*>(smem + C::kHead);
  const int lane = threadIdx.x & 31;
  const int n = a.nodes, m = a.edges;
  const bool edge_bulk = a.vec_ok != 0;
  const bool idx_bulk = (((uintptr_t)a.nindex) & 15) == 0;
  const u64 stream_pol = l2_policy_evict_first();  // the CSR is read once per scan
  // Lanes 0..7 read the vertex of each consumer warp's first entry, lane 8
  // the vertex of the next tile's first entry (first_v has one entry per
  // kGran entries), one tile ahead of the copies.
  const TileSeq ts = scan_tiles(ntiles);
  auto first_of = [&](int t) -> int {
    if (lane > kScanWarps || t >= ts.end) return 0;
    const int tb = t * (C::kTile / kGran) + lane * (32 * EPT / kGran);
    return __ldg(a.first_v + min(tb, a.tiles));
  };
  int i = 0;
  int cur = first_of(ts.first);
  for (int t = ts.first; t < ts.end; t += ts.step, i++) {
    const int s = i % C::kStages;
    const int nxt = first_of(t + ts.step);
    // every lane waits; the warp goes on only if all lanes saw the phase end
    if (i >= C::kStages &&
        !__all_sync(0xffffffffu, mbar_wait(&empty[s], ((i / C::kStages) - 1) & 1, kBarrierTimeoutNs))) {
      if (lane == 0) atomicOr(&a.st->error, kErrTimeout);
      break;
    }
    const int v_lo = __shfl_sync(0xffffffffu, cur, 0);
    const int v_hi = __shfl_sync(0xffffffffu, cur, kScanWarps);
    if (lane < kScanWarps) hdr[s].wfirst[lane] = cur;
    cur = nxt;
    const int span = v_hi - v_lo + 1;
    const bool seg = span <= kScanSegCap;
    const long long j0 = (long long)t * C::kTile;
    const int cnt = (int)min((long long)C::kTile, (long long)m - j0);
    int* nl = stages + (size_t)s * C::kStageInts;
    int* ew = nl + C::kTile;
    int* sx = ew + C::kTile;
    const int a0 = v_lo & ~3, off = v_lo - a0;
    const int want = seg ? off + span + 1 : 0;  // slice ints from a0 (a0 + want <= n + 1)
    const int bulk_e = edge_bulk ? (cnt & ~3) : 0;
    const int bulk_x = idx_bulk ? min((want + 3) & ~3, (n + 1 - a0) & ~3) : 0;
    for (int q = bulk_e + lane; q < cnt; q += 32) {
      nl[q] = __ldg(a.nlist + j0 + q);
      ew[q] = __ldg(a.eweight + j0 + q);
    }
    for (int q = bulk_x + lane; q < want; q += 32) sx[q] = __ldg(a.nindex + a0 + q);
    if (lane == 0) {
      hdr[s].v_lo = v_lo;
      hdr[s].span = span;
      hdr[s].off = off;
      hdr[s].seg = seg ? 1 : 0;
    }
    __syncwarp();
    if (lane == 0) {
      fence_proxy_async_smem();
      mbar_arrive_tx(&full[s], 4u * (unsigned)(2 * bulk_e + bulk_x));
      if (bulk_e) {
        if (ECL_L2_HINTS) {
          bulk_g2s_hint(nl, a.nlist + j0, 4u * (unsigned)bulk_e, &full[s], stream_pol);
          bulk_g2s_hint(ew, a.eweight + j0, 4u * (unsigned)bulk_e, &full[s], stream_pol);
        } else {
          bulk_g2s(nl, a.nlist + j0, 4u * (unsigned)bulk_e, &full[s]);
          bulk_g2s(ew, a.eweight + j0, 4u * (unsigned)bulk_e, &full[s]);
        }
      }
      if (bulk_x) bulk_g2s(sx, a.nindex + a0, 4u * (unsigned)bulk_x, &full[s]);
    }
  }
  // Copies still in flight land before the CTA may exit.
  if (lane == 0)
    for (int k = max(0, i - C::kStages); k < i; k++)
      if (!mbar_wait(&full[k % C::kStages], (k / C::kStages) & 1, kBarrierTimeoutNs))
        atomicOr(&a.st->error, kErrTimeout);
}

// One parent[] gather of the heavy scan, through L2 with the evict-last
// policy (L1-allocating loads measured no faster: the gathers rarely repeat
// within an SM).
__device__ __forceinline__ int gather_parent(const int* p, u64 policy) {
  return ECL_L2_HINTS ? ld_cg_hint(p, policy) : __ldg(p);
}

template <int KIND, int EPT>
__global__ void __launch_bounds__(kScanThreads, ScanCfg<EPT>::kMinBlocks) k_scan(ScanArgs a) {
  using C = ScanCfg<EPT>;
  constexpr int kTile = C::kTile, R = 32 * EPT;  // entries per tile / per consumer warp
  extern __shared__ __align__(128) unsigned char scan_dyn[];
  u64* full = reinterpret_cast<u64*>(scan_dyn);
  u64* empty = full + C::kStages;
  const ScanStage* hdr = reinterpret_cast<const ScanStage*>(scan_dyn + 128);
  const int* stages = reinterpret_cast<const int*>(scan_dyn + C::kHead);
  DevState* st = a.st;
  if (ld_volatile(&st->error) & kErrFormat) return;  // set by k_prep only
  if (KIND == kHeavy && !st->filtered) return;
  // only the variant the split selects runs
  if ((KIND == kHeavy ? heavy_ept(st->split) : scan_ept(st->split)) != EPT) return;
  const int n = a.nodes, m = a.edges;
  const int ntiles = (int)(((long long)m + kTile - 1) / kTile);
  if ((int)blockIdx.x >= ntiles) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    for (int s = 0; s < C::kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kScanWarps);
    }
    mbar_fence_init();
  }
  __syncthreads();
  if (warp == kScanWarps) {
    scan_produce<EPT>(a, scan_dyn, ntiles);
    return;
  }
  // Row-start marks of this warp's range: row index minus the warp's first
  // row, 0 = no row starts there. Each lane clears its own slots after use.
  int* rmark = reinterpret_cast<int*>(scan_dyn + C::kHead) + (size_t)C::kStages * C::kStageInts + warp * R;
  for (int q = lane; q < R; q += 32) rmark[q] = 0;
  __syncwarp();
  const int thr = st->threshold;
  const u64 keep_pol = l2_policy_evict_last();  // parent[] is gathered by every consumer warp
  unsigned* ctr = &st->wl_count[KIND][0];
  unsigned wpos = 0, wend = 0, kept = 0;  // this warp's reserved, unused slots [wpos, wend)
  unsigned idmax = 0;                     // largest neighbour id seen, as unsigned
  int i = 0;
  const TileSeq ts = scan_tiles(ntiles);
  for (int t = ts.first; t < ts.end; t += ts.step, i++) {
    const int s = i % C::kStages;
    if (!__all_sync(0xffffffffu, mbar_wait(&full[s], (i / C::kStages) & 1, kBarrierTimeoutNs))) {
      if (lane == 0) atomicOr(&st->error, kErrTimeout);
      break;
    }
    const int* nl = stages + (size_t)s * C::kStageInts;
    const int v_lo = hdr[s].v_lo, span = hdr[s].span;
    const int* sx = nl + 2 * kTile + hdr[s].off;  // sx[i] = nindex[v_lo + i]
    // entry positions fit in 32 bits (edges < 2^31)
    const unsigned jw = (unsigned)t * kTile + warp * R;  // first entry of this warp
    const unsigned jl = jw + lane * EPT;                 // first entry of this lane
    const int lim = jl < (unsigned)m ? min(EPT, m - (int)jl) : 0;  // the lane's valid entries
    const int* nlw = nl + warp * R + lane * EPT;
    const int* eww = nlw + kTile;
    // the lane's entries, 128 bits at a time from the staged tile
    int nb[EPT], w[EPT];
    if (lim == EPT) {
#pragma unroll
      for (int q = 0; q < EPT; q += 4) {
        const int4 x = *reinterpret_cast<const int4*>(nlw + q);
        const int4 y = *reinterpret_cast<const int4*>(eww + q);
        nb[q] = x.x; nb[q + 1] = x.y; nb[q + 2] = x.z; nb[q + 3] = x.w;
        w[q] = y.x; w[q + 1] = y.y; w[q + 2] = y.z; w[q + 3] = y.w;
      }
    } else {
#pragma unroll
      for (int q = 0; q < EPT; q++) {
        nb[q] = q < lim ? nlw[q] : -1;
        w[q] = q < lim ? eww[q] : 0;
      }
    }
    // Vertex of every entry, as an offset from v_lo.
    int vi[EPT];
    if (hdr[s].seg) {
      const int lo = hdr[s].wfirst[warp] - v_lo;  // row holding entry jw
      // Rows starting inside (jw, jw + R) mark their start; of several rows
      // starting at one position (zero-degree rows) the last one owns it.
      if (jw < (unsigned)m)
        for (int kb = lo + 1;; kb += 32) {
          const int k = kb + lane;
          const unsigned sk = k <= span ? (unsigned)sx[k] : jw + R;
          const bool in = sk < jw + R;
          if (in) atomicMax(&rmark[sk - jw], k - lo);
          if (__ballot_sync(0xffffffffu, in) != 0xffffffffu) break;
        }
      __syncwarp();
      // an entry's row is the last mark at or before it (lane-local running
      // maximum, then a warp exclusive max-scan across lanes)
      int run = 0, loc[EPT];
#pragma unroll
      for (int q = 0; q < EPT; q += 4) {
        int4* slot = reinterpret_cast<int4*>(&rmark[lane * EPT + q]);
        const int4 mk = *slot;
        *slot = make_int4(0, 0, 0, 0);
        loc[q] = run = max(run, mk.x);
        loc[q + 1] = run = max(run, mk.y);
        loc[q + 2] = run = max(run, mk.z);
        loc[q + 3] = run = max(run, mk.w);
      }
      int incl = run;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl = max(incl, x);
      }
      int prev = __shfl_up_sync(0xffffffffu, incl, 1);
      if (lane == 0) prev = 0;
#pragma unroll
      for (int q = 0; q < EPT; q++) vi[q] = lo + max(prev, loc[q]);
    } else {
      // slice too long to stage (long runs of zero-degree vertices)
#pragma unroll
      for (int q = 0; q < EPT; q++) vi[q] = q < lim ? vertex_in(a.nindex, v_lo, span, jl + q) - v_lo : 0;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);  // this warp reads nothing more of the stage
    if (KIND == kLight && lim > 0) {  // inMST = 0 (the reference memsets it, :306)
      if (a.zero_vec && lim == EPT) {
        if (EPT == 4) *reinterpret_cast<unsigned*>(a.inMST + jl) = 0u;
        else if (EPT == 8) *reinterpret_cast<uint2*>(a.inMST + jl) = make_uint2(0u, 0u);
        else *reinterpret_cast<uint4*>(a.inMST + jl) = make_uint4(0u, 0u, 0u, 0u);
      } else {
        for (int q = 0; q < lim; q++) a.inMST[jl + q] = 0;
      }
    }
    // filter: one direction with a valid id (v < nb < n, as one unsigned
    // compare), then the phase's weight test
    unsigned cand = 0;
    int vtx[EPT], nrep[EPT];
#pragma unroll
    for (int q = 0; q < EPT; q++) {
      const int v = v_lo + vi[q];
      if (q < lim) idmax = max(idmax, (unsigned)nb[q]);
      const bool pass = q < lim && (unsigned)nb[q] - (unsigned)v - 1u < (unsigned)(n - v - 1) &&
                        (KIND == kLight ? w[q] <= thr : w[q] > thr);
      cand |= (unsigned)pass << q;
      vtx[q] = v;
      nrep[q] = nb[q];
    }
    if (KIND == kHeavy) {  // light-tree reps of both endpoints, all loads in flight together
      // A lane's entries run in CSR order, so consecutive ones mostly share
      // their row: its rep is loaded once per row, not once per entry.
      int rv = -1, rrep = 0;
#pragma unroll
      for (int q = 0; q < EPT; q++)
        if (cand & (1u << q)) {
          if (vtx[q] != rv) {
            rv = vtx[q];
            rrep = gather_parent(a.parent + rv, keep_pol);
          }
          vtx[q] = rrep;
          nrep[q] = gather_parent(a.parent + nb[q], keep_pol);
        }
#pragma unroll
      for (int q = 0; q < EPT; q++)
        if (vtx[q] == nrep[q]) cand &= ~(1u << q);
    }
    const unsigned cnt = __popc(cand);
    // warp reservation: slots from this warp's chunk, then a fresh chunk
    unsigned incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += x;
    }
    const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
    if (total) {
      const unsigned avail = wend - wpos;
      unsigned fresh = 0, take = 0;
      if (total > avail) {
        take = max(total - avail, a.chunk);
        if (lane == 0) fresh = atomicAdd(ctr, take);
        fresh = __shfl_sync(0xffffffffu, fresh, 0);
      }
      unsigned p = incl - cnt;
#pragma unroll
      for (int q = 0; q < EPT; q++) {
        if (!(cand & (1u << q))) continue;
        const unsigned slot = p < avail ? wpos + p : fresh + (p - avail);
        if (slot >= a.wl_cap) atomicOr(&st->error, kErrOverflow);
        else if (a.ids) reinterpret_cast<int*>(a.wl)[slot] = (int)(jl + q);
        else a.wl[slot] = make_int4(vtx[q], nrep[q], w[q], (int)(jl + q));
        p++;
      }
      if (total > avail) {
        wpos = fresh + (total - avail);
        wend = fresh + take;
      } else {
        wpos += total;
      }
      kept += cnt;
    }
  }
  if (idmax >= (unsigned)n) atomicOr(&st->error, kErrFormat);  // a neighbour id outside [0, n)
  for (unsigned p = wpos + lane; p < wend; p += 32)  // null entries in the unused slots
    if (p < a.wl_cap) {
      if (a.ids) reinterpret_cast<int*>(a.wl)[p] = -1;
      else a.wl[p] = make_int4(-1, -1, 0, 0);
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
  if (lane == 0 && kept) atomicAdd(&st->scan_kept[KIND], kept);
}

// parent[v] = root(v) for every vertex, once before the heavy scan.
// A per-CTA set of roots already found ends a walk as soon as it reaches one:
// every walk through a giant light tree would otherwise read that tree's
// root entry, one L2 line hammered by millions of threads. Roots do not
// change during the pass (other threads only shorten paths).
__global__ void __launch_bounds__(kThreads) k_flatten(int* parent, int n, const DevState* st) {
  constexpr int kRootSlots = 1024;
  __shared__ int roots[kRootSlots];
  if (!st->filtered || (ld_volatile(&st->error) & (kErrFormat | kErrTimeout))) return;
  for (int i = threadIdx.x; i < kRootSlots; i += blockDim.x) roots[i] = -1;
  __syncthreads();
  volatile int* known = roots;
  auto slot = [](int x) { return ((unsigned)x * 0x85EBCA6Bu) >> 22; };  // 10 bits
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    int x = v, p = __ldcg(parent + v);
    while (p != x) {
      x = p;
      if (known[slot(x)] == x) break;
      p = __ldcg(parent + x);
    }
    known[slot(x)] = x;
    if (x != v) __stcg(parent + v, x);
  }
}

// ----------------------------------------------------------------- rounds
// Per-CTA shared-memory state of the round kernel. Representatives shared by
// many worklist entries (a growing giant component) would otherwise put
// every entry's parent read, min-slot guard read, atomicMin and reset on one
// L2 address; these small direct-mapped tables absorb the repeats per CTA.
struct RoundSmem {
  ReserveSmem rs;            // the batch kernel's CTA scans
  unsigned cursor;           // entries this CTA kept so far in the current find/min pass
  int seg_n;                 // segments of the list the passes read (1 = dense from seg_off[0])
  unsigned seg_q[kMaxRoundCtas + 1];  // entries in the segments before b (seg_q[seg_n] = all)
  unsigned seg_off[kMaxRoundCtas];    // first position of segment b
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
  if (threadIdx.x == 0) s.cursor = 0;
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

// ---- segmented round worklists
// A find/min pass compacts its kept entries without any global reservation:
// the CTA that runs tile share b of the pass (tiles b, b + stride, ...) owns
// the output positions [region_b, region_b + share_b), where share_b counts
// the logical input entries of its tiles, and its warps take positions from a
// shared-memory cursor. The pass's output is therefore one dense segment per
// CTA (seg_cnt[b] kept entries from region_b). The next passes address that
// list by logical index through a prefix table of the segment counts, so a
// pass needs neither a global atomic per tile nor a CTA barrier per tile.

// The list read next is dense: entries [0, count) from position 0.
__device__ __forceinline__ void seg_set_dense(RoundSmem& s, unsigned count) {
  if (threadIdx.x == 0) {
    s.seg_n = 1;
    s.seg_off[0] = 0;
    s.seg_q[0] = 0;
    s.seg_q[1] = count;
  }
}

// The list read next is the one the grid's find/min pass just wrote (`nseg`
// segments, published in the control block before the grid barrier). The
// whole CTA builds the prefix table: thread t loads kSegPer consecutive
// segment counts, one warp scan and one pass over the warp totals give the
// prefixes. Every thread of the CTA must call this; the caller synchronises
// the CTA before the table is used.
constexpr int kSegPer = (kMaxRoundCtas + kRoundThreads - 1) / kRoundThreads;
__device__ __forceinline__ void seg_load(RoundSmem& s, const DevState* st, int nseg) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int b0 = kSegPer * t;
  unsigned c[kSegPer], mine = 0;
#pragma unroll
  for (int k = 0; k < kSegPer; k++) {
    const int b = b0 + k;
    c[k] = b < nseg ? __ldcg(&st->seg_cnt[b]) : 0u;
    if (b < nseg) s.seg_off[b] = __ldcg(&st->seg_off[b]);
    mine += c[k];
  }
  unsigned incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned x = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += x;
  }
  if (lane == 31) s.rs.warp_off[warp][0] = incl;
  __syncthreads();
  unsigned q = incl - mine;
  for (int w = 0; w < warp; w++) q += s.rs.warp_off[w][0];
#pragma unroll
  for (int k = 0; k < kSegPer; k++) {
    const int b = b0 + k;
    if (b < nseg) s.seg_q[b] = q;
    q += c[k];
    if (b == nseg - 1) s.seg_q[nseg] = q;  // the thread holding the last segment
  }
  if (t == 0) s.seg_n = nseg;
}

// Position of logical entry i of the list described by the prefix table.
__device__ __forceinline__ unsigned seg_at(const RoundSmem& s, unsigned i) {
  const int nseg = s.seg_n;
  if (nseg == 1) return s.seg_off[0] + i;
  int lo = 0, hi = nseg;  // largest b with seg_q[b] <= i (seg_q[nseg] > i)
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (s.seg_q[mid] <= i) lo = mid;
    else hi = mid;
  }
  return s.seg_off[lo] + (i - s.seg_q[lo]);
}

// First output position of tile share `b` of a pass over W logical entries
// in tiles of `tile`, shares strided by `stride`: the logical entries of the
// tiles of all shares before b (the last tile may be partial).
__device__ __forceinline__ unsigned share_region(unsigned W, unsigned tile, unsigned b, unsigned stride) {
  const unsigned ntiles = (W + tile - 1) / tile;
  const unsigned q = ntiles / stride, rr = ntiles % stride;
  const unsigned long long full = (unsigned long long)tile * ((unsigned long long)q * b + min(b, rr));
  const unsigned last_owner = ntiles ? (ntiles - 1) % stride : 0u;
  const unsigned short_by = (unsigned)((unsigned long long)ntiles * tile - W);
  return (unsigned)(full - (ntiles && b > last_owner ? short_by : 0u));
}

// Parallel-edge elimination within a tile (opt-in through ECL_FLAG_DEDUP).
// Entries of one tile that join the same two trees are parallel edges of the
// contracted graph; only the one with the smallest (weight, j) key can be a
// forest edge (any forest through a heavier one is heavier than the same
// forest through the lightest), so the others may be dropped for good. Warp
// groups with equal rep pairs reduce first; group minima meet in a per-tile
// shared table. Measured on RMAT scale 22 the elimination costs more (two CTA
// barriers and the table per tile) than the smaller worklists save, so it is
// off by default. keep[k] is narrowed to the survivors. Every thread of the
// CTA must call this (it synchronises the CTA).
template <int E>
__device__ __forceinline__ void drop_parallel(const int4 (&e)[E], bool (&keep)[E], RoundSmem& s) {
  const int lane = threadIdx.x & 31;
  u64 pk[E], gmin[E];
#pragma unroll
  for (int k = 0; k < E; k++) {
    const unsigned lo = (unsigned)min(e[k].x, e[k].y), hi = (unsigned)max(e[k].x, e[k].y);
    pk[k] = keep[k] ? (((u64)lo << 32) | hi) : (0xFFFFFFFF00000000ull | (threadIdx.x * E + k));
    const u64 key = edge_key(e[k].z, e[k].w);
    gmin[k] = key;
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
  }
  __syncthreads();  // the tile's pair table is complete
#pragma unroll
  for (int k = 0; k < E; k++) {
    if (keep[k]) {
      const unsigned slot = pair_slot(pk[k]);
      const u64 key = edge_key(e[k].z, e[k].w);
      const u64 best = s.pair_tag[slot] == pk[k] ? s.pair_min[slot] : gmin[k];
      keep[k] = key == best;
    }
  }
  __syncthreads();  // every check done before the table is cleared
  for (int i = threadIdx.x; i < kPairSlots; i += blockDim.x) {
    s.pair_tag[i] = kNoPair;
    s.pair_min[i] = kNoEdge;
  }
}

// Output positions for this thread's kept entries: one shared-memory atomic
// per warp on the CTA's cursor, no barrier. Returns the position of the
// thread's first kept entry (the rest follow) inside the CTA's segment that
// starts at `region`. Every lane of the warp must call this.
template <int E>
__device__ __forceinline__ unsigned warp_reserve(const bool (&keep)[E], RoundSmem& s, unsigned region) {
  const int lane = threadIdx.x & 31;
  unsigned cnt = 0;
#pragma unroll
  for (int k = 0; k < E; k++) cnt += keep[k];
  unsigned excl, total;
  if (E == 1) {
    const unsigned mask = __ballot_sync(0xffffffffu, cnt != 0);
    excl = __popc(mask & ((1u << lane) - 1u));
    total = __popc(mask);
  } else {
    unsigned incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    excl = incl - cnt;
    total = __shfl_sync(0xffffffffu, incl, 31);
  }
  unsigned base = 0;
  if (lane == 0 && total) base = atomicAdd(&s.cursor, total);
  base = __shfl_sync(0xffffffffu, base, 0);
  return region + base + excl;
}

// Roots of the 2*kEPT endpoints a thread holds, all walks advanced in lock
// step so their loads are in flight together. A per-CTA cache of
// (vertex << 32 | root) is consulted at every step (roots do not change
// during the find/min pass): after a walk it holds the start vertex, its
// parent and the root, so the nodes near the top of a large tree, which
// every walk through that tree would otherwise read from the same L2 lines,
// are read once per CTA. Hooking by random priority keeps trees shallow, so
// a walk only starts path splitting (re-pointing each visited node to its
// grandparent, which stays inside the tree) once it is kSplitAfter steps
// deep: the writes bound pathological chains, while splitting every walk
// would have the many walkers that share a start vertex all store to the
// same parent entries.
__device__ __forceinline__ int find_cached(const RoundSmem& s, int x) {
  const u64 c = ((const volatile u64*)s.find_cache)[find_slot(x)];
  return (int)(c >> 32) == x ? (int)(unsigned)c : -1;  // -1: not cached (x >= 0)
}

template <int N>
__device__ __forceinline__ void multi_find(int (&v)[N], const bool (&valid)[N], int* parent,
                                           RoundSmem& s, bool use_cache = true,
                                           int split_after = kSplitAfter) {
  int par[N], orig[N], first[N];  // first: the start vertex's parent
  unsigned miss = 0;
#pragma unroll
  for (int i = 0; i < N; i++) {
    orig[i] = v[i];
    par[i] = v[i];
    first[i] = v[i];
    if (!valid[i]) continue;
    const int r = use_cache ? find_cached(s, v[i]) : -1;
    if (r >= 0) {
      v[i] = par[i] = r;
    } else {
      miss |= 1u << i;
      par[i] = first[i] = __ldcg(parent + v[i]);
    }
  }
  for (int step = 0;; step++) {
    int gp[N];
    bool any = false;
#pragma unroll
    for (int i = 0; i < N; i++) {
      gp[i] = par[i];
      if (par[i] != v[i]) {
        const int r = use_cache ? find_cached(s, par[i]) : -1;
        if (r >= 0) {  // the rest of the walk is known
          v[i] = par[i] = gp[i] = r;
          continue;
        }
        any = true;
        gp[i] = __ldcg(parent + par[i]);
      }
    }
    if (!any) break;
#pragma unroll
    for (int i = 0; i < N; i++) {
      if (par[i] != v[i]) {
        if (step >= split_after && gp[i] != par[i]) __stcg(parent + v[i], gp[i]);
        v[i] = par[i];
        par[i] = gp[i];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < N; i++)
    if (use_cache && (miss & (1u << i))) {
      volatile u64* fc = (volatile u64*)s.find_cache;
      const u64 root = (unsigned)v[i];
      fc[find_slot(orig[i])] = ((u64)(unsigned)orig[i] << 32) | root;
      if (first[i] != v[i]) fc[find_slot(first[i])] = ((u64)(unsigned)first[i] << 32) | root;
      if (orig[i] != v[i]) fc[find_slot(v[i])] = (root << 32) | root;
    }
}

// How a find/min pass clears the previous round's min slots: not at all
// (first round), slot by slot for its entries' reps (deduplicated per CTA),
// or the whole array with coalesced stores when the entries outnumber the
// vertices enough that the scattered stores would cost more.
enum : int { kResetNone = 0, kResetSparse = 1, kResetDense = 2 };

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
// A lone entry of a rep already in the table folds into it as well, so a
// giant component's rep costs no global traffic. The rest (lone entries of
// other reps, leaders whose table slot belongs to another rep) read the
// global slots together (one round trip for all pairs) and issue
// fire-and-forget atomicMin only where the guard shows an improvement.
// Every lane of the warp must call this.
template <int N>
__device__ __forceinline__ void offer_mins(const int (&rep)[N], const u64 (&key)[N],
                                           const bool (&valid)[N], u64* mcur, RoundSmem& s,
                                           unsigned long long& atomics, bool coop = true,
                                           bool guard = true) {
  const int lane = threadIdx.x & 31;
  bool cold[N];
  u64 val[N];
#pragma unroll
  for (int i = 0; i < N; i++) {
    cold[i] = valid[i];
    val[i] = key[i];
    if (!coop) continue;  // uniform: every valid pair goes straight to its global slot
    cold[i] = false;
    const unsigned g = __match_any_sync(0xffffffffu, valid[i] ? rep[i] : -2 - lane);
    if (!valid[i]) continue;
    if ((g & (g - 1)) == 0) {
      // a lone entry of a rep already in the hot table folds into it too
      const unsigned slot = hot_slot(rep[i]);
      if (((volatile int*)s.hot_rep)[slot] == rep[i]) {
        if (((volatile u64*)s.hot_key)[slot] > key[i]) atomicMin(&s.hot_key[slot], key[i]);
      } else {
        cold[i] = true;
      }
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
  for (int i = 0; i < N; i++) seen[i] = cold[i] && guard ? __ldcg(mcur + rep[i]) : kNoEdge;
#pragma unroll
  for (int i = 0; i < N; i++) {
    if (cold[i] && seen[i] > val[i]) {
      atomicMin(mcur + rep[i], val[i]);
      atomics++;
    }
  }
}

// Worklist entry at position `pos`: a tuple {rep a, rep b, w, j}, or under
// kAblNoTuples a CSR index whose endpoints and weight are gathered (x = -1
// marks a null entry either way).
__device__ __forceinline__ int4 load_entry(const RoundArgs& a, const int4* list, unsigned pos) {
  if (a.abl & kAblNoTuples) {
    const int j = __ldcg(reinterpret_cast<const int*>(list) + pos);
    if (j < 0) return make_int4(-1, -1, 0, 0);
    return make_int4(__ldg(a.slist + j), __ldg(a.nlist + j), __ldg(a.eweight + j), j);
  }
  return __ldcg(list + pos);
}

__device__ __forceinline__ void store_entry(const RoundArgs& a, int4* list, unsigned pos, const int4& e) {
  if (a.abl & kAblNoTuples) reinterpret_cast<int*>(list)[pos] = e.w;
  else list[pos] = e;
}

// kernel1 (ECL_MST.cu:210-226) plus kernel3 of the previous round (:243-251):
// each input entry clears its endpoints' slots in the previous round's min
// array, resolves its endpoints to reps, and if they differ is compacted into
// `out` with the reps (implicit path compression, :218-219) and offers its
// key to both reps' min slots. The input is the list the prefix table in `s`
// describes (W logical entries); the kept entries go to this CTA's segment of
// `out` (share `start` of `stride`), whose size is left in s.cursor and
// added to *out_ctr and *kept_ctr.
//
// `fresh` marks the first round of a phase: its entries come straight from
// the scan, so both endpoints are roots (parent[v] = v before the light
// phase, the flattened light-tree roots before the heavy one) and differ.
// That round needs no find and keeps every entry: it only offers keys, and
// the scan's list serves as its output unchanged (no copy).
__device__ __forceinline__ void round_find_min(const RoundArgs& a, const int4* in, unsigned W,
                                               int4* out, unsigned* out_ctr, unsigned* kept_ctr,
                                               u64* mcur, u64* mprev, int reset, bool fresh,
                                               unsigned start, unsigned stride, RoundSmem& s,
                                               bool flat = false) {
  constexpr int N = 2 * kEPT;
  const unsigned tile = blockDim.x * kEPT;
  const unsigned ntiles = (W + tile - 1) / tile;
  const unsigned region = share_region(W, tile, start, stride);
  const bool dedup = (a.abl & kDedup) != 0;
  const bool keep_ends = (a.abl & kAblKeepEnds) != 0;  // entries are not rewritten to reps
  const bool count_only = (a.abl & kAblNoDD) != 0;     // nothing is compacted
  unsigned long long atomics = 0;
  if (reset == kResetDense)  // every slot of the previous round's array, coalesced
    for (unsigned i = start * blockDim.x + threadIdx.x; i < (unsigned)a.nodes; i += stride * blockDim.x)
      __stcg(mprev + i, kNoEdge);
  for (unsigned t = start; t < ntiles; t += stride) {
    int4 e[kEPT];
    bool in_range[kEPT];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      const unsigned idx = t * tile + k * blockDim.x + threadIdx.x;
      in_range[k] = idx < W;
      e[k] = in_range[k] ? load_entry(a, in, seg_at(s, idx)) : make_int4(0, 0, 0, 0);
      if (e[k].x < 0) in_range[k] = false;  // null entry (unused scan slot)
    }
    int4 orig[kEPT];
#pragma unroll
    for (int k = 0; k < kEPT; k++) orig[k] = e[k];
    int v[N];
    bool vv[N];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      v[2 * k] = e[k].x;
      v[2 * k + 1] = e[k].y;
      vv[2 * k] = vv[2 * k + 1] = in_range[k];
      if (reset == kResetSparse && in_range[k]) {
        reset_prev(e[k].x, mprev, s);
        reset_prev(e[k].y, mprev, s);
      }
    }
    bool keep[kEPT];
    if (fresh) {
#pragma unroll
      for (int k = 0; k < kEPT; k++) keep[k] = in_range[k];
    } else {
      if (flat) {  // parent[] was just flattened: one load names the root
#pragma unroll
        for (int i = 0; i < N; i++) v[i] = vv[i] ? __ldcg(a.parent + v[i]) : v[i];
      } else {
        multi_find<N>(v, vv, a.parent, s, !(a.abl & kAblNoFindCache), keep_ends ? 0 : kSplitAfter);
      }
#pragma unroll
      for (int k = 0; k < kEPT; k++) {
        keep[k] = in_range[k] && v[2 * k] != v[2 * k + 1];
        e[k].x = v[2 * k];
        e[k].y = v[2 * k + 1];
      }
      if (dedup) drop_parallel<kEPT>(e, keep, s);  // uniform across the CTA
      unsigned pos = warp_reserve<kEPT>(keep, s, region);
      if (!count_only) {
#pragma unroll
        for (int k = 0; k < kEPT; k++) {
          if (keep[k]) {
            if (pos < a.wl_cap) store_entry(a, out, pos, keep_ends ? orig[k] : e[k]);
            else atomicOr(&a.st->error, kErrOverflow);
            pos++;
          }
        }
      }
    }
    u64 key[N];
    bool kv[N];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      key[2 * k] = key[2 * k + 1] = edge_key(e[k].z, e[k].w);
      kv[2 * k] = kv[2 * k + 1] = keep[k];
    }
    offer_mins<N>(v, key, kv, mcur, s, atomics, !(a.abl & kAblNoCoop), !(a.abl & kAblNoGuards));
  }
  __syncthreads();
  if (threadIdx.x == 0 && s.cursor) {
    atomicAdd(out_ctr, s.cursor);
    atomicAdd(kept_ctr, s.cursor);
  }
  // flush the CTA's partial minima of hot representatives
  for (int i = threadIdx.x; i < kHotSlots; i += blockDim.x) {
    const int r = s.hot_rep[i];
    if (r >= 0) {
      const u64 k = s.hot_key[i];
      if ((a.abl & kAblNoGuards) || __ldcg(mcur + r) > k) {
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
// endpoint's slot is a forest edge: union the trees and mark inMST[j]. The
// list is the one the prefix table in `s` describes (W logical entries).
__device__ __forceinline__ void round_mark(const RoundArgs& a, const int4* wl, unsigned W,
                                           const u64* mcur, unsigned start, unsigned stride,
                                           RoundSmem& s) {
  constexpr int N = 2 * kEPT;
  const unsigned tile = blockDim.x * kEPT;
  const unsigned ntiles = (W + tile - 1) / tile;
  const bool keep_ends = (a.abl & kAblKeepEnds) != 0;
  for (unsigned t = start; t < ntiles; t += stride) {
    int4 e[kEPT];
    bool in_range[kEPT];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      const unsigned idx = t * tile + k * blockDim.x + threadIdx.x;
      in_range[k] = idx < W;
      e[k] = in_range[k] ? load_entry(a, wl, seg_at(s, idx)) : make_int4(0, 0, 0, 0);
      if (e[k].x < 0) in_range[k] = false;  // null entry (unused scan slot)
    }
    if (keep_ends) {
      // Entries hold their endpoints, not reps: find them again. Unions of
      // this pass may already have moved a root; a key then meets the slot of
      // the tree it joined, which can only defer an edge to a later round:
      // every edge marked is still the lightest edge leaving a tree of the
      // find/min pass (the reference's kernel2 finds the same way, :198-216).
      int v[N];
      bool vv[N];
#pragma unroll
      for (int k = 0; k < kEPT; k++) {
        v[2 * k] = e[k].x;
        v[2 * k + 1] = e[k].y;
        vv[2 * k] = vv[2 * k + 1] = in_range[k];
      }
      multi_find<N>(v, vv, a.parent, s, false, 0);
#pragma unroll
      for (int k = 0; k < kEPT; k++) {
        e[k].x = v[2 * k];
        e[k].y = v[2 * k + 1];
        if (e[k].x == e[k].y) in_range[k] = false;
      }
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

__global__ void __launch_bounds__(kRoundThreads, ECL_ROUND_MIN_BLOCKS) k_rounds(RoundArgs a) {
  __shared__ RoundSmem s;
  DevState* st = a.st;
  const int ph = a.phase;
  if (ph == 1 && !st->filtered) return;
  // Only bits no CTA of this kernel can set, so every CTA takes the same exit.
  if (ld_volatile(&st->error) & (kErrFormat | kErrTimeout)) return;
  round_smem_clear(s);
  seg_set_dense(s, 0);  // round 0 reads the scan's list as it is
  __syncthreads();
  unsigned active = gridDim.x;  // CTAs still in the launch
  bool tail = active == 1;      // one CTA: CTA barriers stand for the grid's
  int r = 0;
  const bool stamp = blockIdx.x == 0 && threadIdx.x == 0;
  // Round 0 offers straight from the scan's list, whose endpoints are roots
  // (not so under kAblNoTuples: those lists hold CSR indices, whose
  // endpoints are gathered as they are).
  const bool fresh0 = !(a.abl & kAblNoTuples);
  const bool ndd = (a.abl & kAblNoDD) != 0;
  if (stamp) st->t_round_start[ph] = globaltimer_ns();
  for (;;) {
    unsigned W = min(ld_volatile(&st->wl_count[ph][r]), a.wl_cap);
    if (W == 0) break;  // (kAblNoDD: no entry joined two trees last round)
    if (ndd) W = min(ld_volatile(&st->wl_count[ph][0]), a.wl_cap);  // the phase's whole list, every round
    if (r >= ECL_MAX_ROUNDS) {
      if (stamp) atomicOr(&st->error, kErrRounds);
      break;
    }
    // CTAs the round keeps: one per min_tiles tiles of its worklist (the
    // rest leave for good; worklists never grow), or one CTA alone at the
    // small tail, which then syncs with CTA barriers only
    unsigned want = active;
    if (a.min_tiles > 0) {
      const unsigned per = (unsigned)a.min_tiles * blockDim.x * kEPT;
      want = min(want, max(1u, (W + per - 1) / per));
    }
    if (W <= a.small_tail) want = 1;
    if (want < active) {
      active = want;
      if (blockIdx.x >= active) return;
      tail = active == 1;
    }
    const unsigned start = blockIdx.x, stride = active;
    // A fresh round 0 reads the scan's list (wl0) and keeps it as its
    // output; the compacting rounds after it alternate between the lists.
    // The min-slot arrays alternate per round.
    const bool fresh = fresh0 && r == 0;
    const int k = fresh0 ? r - 1 : r;  // index among the compacting rounds
    const bool in1 = !fresh && !ndd && (k & 1) != 0;
    const int4* in = in1 ? a.wl1 : a.wl0;
    int4* out = in1 ? a.wl0 : a.wl1;
    const bool odd = (r & 1) != 0;
    u64* mcur = odd ? a.minv1 : a.minv0;
    u64* mprev = odd ? a.minv0 : a.minv1;
    // entries that keep their endpoints cannot name the previous round's
    // reps: those rounds clear the whole previous array
    const bool dense = (a.abl & kAblKeepEnds) || (!tail && 4ull * W >= (unsigned long long)a.nodes);
    const int reset = r == 0 ? kResetNone : (dense ? kResetDense : kResetSparse);
    // A round whose entries outnumber the vertices ECL_FLAT_ROUNDS times first
    // points every vertex at its root (one grid-stride pass; roots do not
    // change between passes), so each of its finds is a single load.
    const bool flat = ECL_FLAT_ROUNDS > 0 && !fresh && !tail && !(a.abl & kAblKeepEnds) &&
                      (unsigned long long)W >= (unsigned long long)ECL_FLAT_ROUNDS * (unsigned)a.nodes;
    if (flat) {
      for (int v = (int)(start * blockDim.x + threadIdx.x); v < a.nodes; v += (int)(stride * blockDim.x)) {
        const int rt = find_ro(v, a.parent);
        if (rt != v) __stcg(a.parent + v, rt);
      }
      if (!grid_barrier(st, kBarrierTimeoutNs, active)) return;
    }
    round_find_min(a, in, W, out, &st->wl_count[ph][r + 1], &st->wl_kept[ph][r + 1], mcur, mprev, reset,
                   fresh, start, stride, s, flat);
    if (fresh && blockIdx.x == 0 && threadIdx.x == 0) {  // the scan's list is round 0's output
      st->wl_count[ph][1] = W;
      st->wl_kept[ph][1] = st->scan_kept[ph];
    }
    if (!fresh && !tail && !ndd && threadIdx.x == 0) {  // this CTA's segment of the output list
      st->seg_cnt[blockIdx.x] = s.cursor;
      st->seg_off[blockIdx.x] = share_region(W, blockDim.x * kEPT, start, stride);
    }
    if (tail) __syncthreads();
    else if (!grid_barrier(st, kBarrierTimeoutNs, active)) return;
    if (stamp) st->t_round[ph][2 * r] = globaltimer_ns();
    const unsigned W2 = min(ld_volatile(&st->wl_count[ph][r + 1]), a.wl_cap);
    r++;
    if (W2 == 0) break;
    // the list the mark pass and the next round read: the scan's list (round
    // 0), the tail CTA's single segment, or the grid's per-CTA segments
    if (!fresh && !ndd) {
      if (tail) seg_set_dense(s, s.cursor);
      else seg_load(s, st, (int)active);
    }
    hot_refresh(mcur, s);
    round_mark(a, fresh || ndd ? in : out, ndd ? W : W2, mcur, start, stride, s);
    __syncthreads();
    round_smem_clear(s);
    if (tail) __syncthreads();
    else if (!grid_barrier(st, kBarrierTimeoutNs, active)) return;
    if (stamp) st->t_round[ph][2 * r - 1] = globaltimer_ns();
  }
  if (stamp) st->rounds[ph] = r;
}

// ------------------------------------------------ reference ablation steps
// kAblNoTuples: the vertex of every CSR entry (the reference's NoTuples
// variant keeps such an slist, Deoptimizations/..._NoTuples.cu:163-169),
// filled entry-parallel from the scans' tile->vertex table (the row holding
// entry t * kGran), then a short walk along nindex.
__global__ void __launch_bounds__(kThreads) k_slist(const int* nindex, const int* first_v, int* slist,
                                                    int edges, const DevState* st) {
  if (ld_volatile(&st->error) & kErrFormat) return;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < edges; j += gridDim.x * blockDim.x) {
    int v = __ldg(first_v + j / kGran);
    while (__ldg(nindex + v + 1) <= j) v++;
    slist[j] = v;
  }
}

// NoEdgeBased (Deoptimizations/..._NoEdgeBased.cu:152-195): all Boruvka
// rounds of a phase as vertex-centric passes over the CSR, one thread per
// vertex walking its row, in one cooperative launch: (A) every one-direction
// entry of the phase's weight class whose endpoints lie in different trees
// offers its key to both roots, (B) an entry holding the minimum of either
// root's slot joins the trees and is marked, (C) the slots are cleared. The
// rounds end when pass A finds no entry across two trees (the reference's
// go_again). Pass B finds while other threads join; an entry it marks is
// still the lightest edge leaving a tree of pass A, so the forest is the
// reference's (an edge missed in one round is found in a later one).
__global__ void __launch_bounds__(kRoundThreads, ECL_ROUND_MIN_BLOCKS) k_rounds_vertex(RoundArgs a,
                                                                                       const int* nindex) {
  DevState* st = a.st;
  const int ph = a.phase;
  if (ph == 1 && !st->filtered) return;
  if (ld_volatile(&st->error) & (kErrFormat | kErrTimeout)) return;
  const int n = a.nodes, thr = st->threshold;
  const bool filtered = st->filtered != 0, guard = !(a.abl & kAblNoGuards);
  const int gid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  u64* mv = a.minv0;
  const bool stamp = blockIdx.x == 0 && threadIdx.x == 0;
  if (stamp) st->t_round_start[ph] = globaltimer_ns();
  auto in_phase = [&](int w) { return !filtered || (ph == 0 ? w <= thr : w > thr); };
  int r = 0;
  for (;; r++) {
    if (r >= ECL_MAX_ROUNDS) {
      if (stamp) atomicOr(&st->error, kErrRounds);
      break;
    }
    unsigned live = 0;
    for (int v = gid; v < n; v += gstride) {  // pass A
      const int beg = __ldg(nindex + v), end = __ldg(nindex + v + 1);
      int rv = -1;
      for (int j = beg; j < end; j++) {
        const int nb = __ldg(a.nlist + j);
        if (nb <= v) continue;  // one direction
        const int w = __ldg(a.eweight + j);
        if (!in_phase(w)) continue;
        if (rv < 0) rv = find_halve(v, a.parent);
        const int rn = find_halve(nb, a.parent);
        if (rv == rn) continue;
        live++;
        const u64 key = edge_key(w, j);
        if (!guard || __ldcg(mv + rv) > key) atomicMin(mv + rv, key);
        if (!guard || __ldcg(mv + rn) > key) atomicMin(mv + rn, key);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) live += __shfl_xor_sync(0xffffffffu, live, o);
    if (lane == 0 && live) atomicAdd(&st->wl_count[ph][r + 1], live);
    if (!grid_barrier(st, kBarrierTimeoutNs, gridDim.x)) return;
    if (stamp) st->t_round[ph][2 * r] = globaltimer_ns();
    if (ld_volatile(&st->wl_count[ph][r + 1]) == 0) break;
    for (int v = gid; v < n; v += gstride) {  // pass B
      const int beg = __ldg(nindex + v), end = __ldg(nindex + v + 1);
      for (int j = beg; j < end; j++) {
        const int nb = __ldg(a.nlist + j);
        if (nb <= v) continue;
        const int w = __ldg(a.eweight + j);
        if (!in_phase(w)) continue;
        const int rv = find_ro(v, a.parent), rn = find_ro(nb, a.parent);
        if (rv == rn) continue;
        const u64 key = edge_key(w, j);
        if (key == __ldcg(mv + rv) || key == __ldcg(mv + rn)) {
          cas_union(rv, rn, a.parent);
          a.inMST[j] = 1;
        }
      }
    }
    if (!grid_barrier(st, kBarrierTimeoutNs, gridDim.x)) return;
    for (int v = gid; v < n; v += gstride) __stcg(mv + v, kNoEdge);  // pass C
    if (!grid_barrier(st, kBarrierTimeoutNs, gridDim.x)) return;
    if (stamp) st->t_round[ph][2 * r + 1] = globaltimer_ns();
  }
  if (stamp) {
    st->rounds[ph] = r;
    st->wl_count[ph][0] = st->wl_count[ph][1];
  }
}

}  // namespace ecl
