// B200 (sm_100a) engine of the ECL-MST minimum spanning forest.
//
// Replaces gpuMST<filter> (ECL-MST/ECL_MST.cu:265-362) and its kernels
// initPM (:147-154), initWL<first> (:157-207), kernel1 (:210-226),
// kernel2 (:229-240), kernel3 (:243-251), find (:127-134) and join (:137-144).
//
// The answer is the reference's: the unique minimum spanning forest under the
// strict order (uint32 weight, CSR index j) over the one-direction entries
// nlist[j] > v, computed in a light phase (w <= threshold, signed compare as
// at :172) and a heavy phase (w > threshold) when filtered. Only the schedule
// differs:
//   k_threshold      threshold on the device (reference heuristic :432-440,
//                    explicit, sampled quantile, or learned)
//   k_scan<LIGHT>    fused initPM + initWL<true>: rows shorter than the degree
//                    split are scanned by one thread, longer rows are cut into
//                    aligned 128-entry chunks that whole warps read with
//                    128-bit loads; appends are CTA-aggregated (one atomic per
//                    CTA tile instead of one per edge, :175,:200)
//   k_rounds         all Boruvka rounds of a phase in one cooperative launch:
//                    per round a find/compact/guarded-atomicMin pass (kernel1)
//                    and a mark/union pass (kernel2), separated by bounded
//                    grid barriers; kernel3's min-slot reset is folded into
//                    the next round's first pass via two alternating min
//                    arrays. No host round trip per round (:312,:318).
//                    Small worklists are finished by one CTA alone.
//   k_scan<HEAVY>    flattens parent[] once, then initWL<false> with the same
//                    two-tier schedule (reps are one load away after flatten)
#include <cuda_runtime.h>
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include "ecl_mst.h"
#include "internal.h"
#include "mst_kernels.cuh"

using namespace ecl;

namespace ecl {

constexpr int kScanThreads = 512;
constexpr int kRoundThreads = 512;
constexpr int kEPT = 4;  // worklist entries per thread per round tile
constexpr int kDefaultSplit = 32;
constexpr unsigned kDefaultSmallTail = 4096;
constexpr unsigned long long kBarrierTimeoutNs = 5ull * 1000 * 1000 * 1000;

struct ScanArgs {
  int nodes;
  int edges;
  const int* nindex;
  const int* nlist;
  const int* eweight;
  int* parent;
  u64* minv0;
  u64* minv1;
  int4* wl;
  unsigned wl_cap;
  int2* desc;
  unsigned desc_cap;
  DevState* st;
  int vec_ok;  // nlist/eweight 16-byte aligned: chunk tier may use int4 loads
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

// --------------------------------------------------------------- threshold
__global__ void k_threshold(const int* __restrict__ eweight, int nodes, int edges, int mode,
                            int explicit_thr, float quantile, int split, DevState* st) {
  __shared__ int samp[4096];
  const int tid = threadIdx.x;
  if (mode == ECL_THRESH_LEARNED) {
    // The MLP kernel has written quantile / split into the control block.
    quantile = st->quantile;
    split = st->learned_split;
    mode = ECL_THRESH_QUANTILE;
  }
  if (tid == 0) st->split = split;
  if (mode == ECL_THRESH_NONE || edges == 0) {
    if (tid == 0) {
      st->filtered = 0;
      st->threshold = INT_MAX;
    }
    return;
  }
  if (mode == ECL_THRESH_EXPLICIT) {
    if (tid == 0) {
      st->filtered = 1;
      st->threshold = explicit_thr;
    }
    return;
  }
  if (mode == ECL_THRESH_HEURISTIC) {
    // ECL_MST.cu:408,432-440: filter iff edges/nodes >= 4; threshold is the
    // min(19, int(3.0*n*20/m))-th of 20 weights sampled at hash(i) % m.
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
          s[i] = eweight[val % (unsigned)edges];
        }
        for (int i = 1; i < ns; i++) {  // insertion sort of <= 20 values
          const int x = s[i];
          int k = i - 1;
          while (k >= 0 && s[k] > x) {
            s[k + 1] = s[k];
            k--;
          }
          s[k + 1] = x;
        }
        const int idx = min(19, (int)(3.0 * nodes * ns / edges));
        st->filtered = 1;
        st->threshold = s[idx];
      }
    }
    return;
  }
  // ECL_THRESH_QUANTILE: quantile of a 4096-entry hashed sample.
  if (!(quantile < 1.0f)) {
    if (tid == 0) {
      st->filtered = 0;
      st->threshold = INT_MAX;
    }
    return;
  }
  const int S = 4096;
  for (int i = tid; i < S; i += blockDim.x) {
    const uint64_t r = ecl_mix64(0x5EED0000ull + (uint64_t)i);
    samp[i] = eweight[(unsigned)(r % (uint64_t)(unsigned)edges)];
  }
  __syncthreads();
  // Bitonic sort of the 4096 samples in shared memory.
  for (int k = 2; k <= S; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < S; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const int a = samp[i], b = samp[ixj];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            samp[i] = b;
            samp[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  if (tid == 0) {
    float q = quantile < 0.f ? 0.f : quantile;
    int idx = (int)(q * (float)(S - 1));
    idx = idx < 0 ? 0 : (idx > S - 1 ? S - 1 : idx);
    st->filtered = 1;
    st->threshold = samp[idx];
  }
}

// --------------------------------------------------------------- scans
enum ScanKind { kLight = 0, kHeavy = 1 };

template <int KIND>
__device__ __forceinline__ bool keep_entry(int v, int n, int w, int thr) {
  return n > v && (KIND == kLight ? (w <= thr) : (w > thr));
}

// Row-or-chunk scan of the CSR (a cooperative launch). LIGHT also performs
// initPM for its vertices; HEAVY first flattens parent[] so that each rep is
// a single load, then keeps only entries whose endpoints are in different
// light-phase trees.
template <int KIND>
__global__ void __launch_bounds__(kScanThreads) k_scan(ScanArgs a) {
  __shared__ ReserveSmem sm;
  DevState* st = a.st;
  if (KIND == kHeavy && !st->filtered) return;
  const int thr = st->threshold;
  const int split = st->split;
  const int n = a.nodes, m = a.edges;
  unsigned* wl_ctr = &st->wl_count[KIND][0];

  if (KIND == kHeavy) {
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
      __stcg(a.parent + v, find_ro(v, a.parent));
    if (!grid_barrier(st, kBarrierTimeoutNs)) return;
  }

  // Pass 1: one thread per vertex.
  const unsigned tiles = (unsigned)((n + blockDim.x - 1) / blockDim.x);
  for (unsigned t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int v = (int)(t * blockDim.x + threadIdx.x);
    unsigned cnt = 0, ndesc = 0;
    int beg = 0, end = 0, rv = v;
    bool thread_row = false;
    if (v < n) {
      if (KIND == kLight) {
        a.parent[v] = v;
        a.minv0[v] = kNoEdge;
        a.minv1[v] = kNoEdge;
      }
      beg = __ldg(a.nindex + v);
      end = __ldg(a.nindex + v + 1);
      if (beg < 0 || end < beg || end > m) {
        atomicOr(&st->error, kErrFormat);
        beg = end = 0;
      }
      if (KIND == kHeavy) rv = __ldcg(a.parent + v);
      if (end - beg < split) {
        thread_row = true;
        for (int j = beg; j < end; j++) {
          const int nb = __ldg(a.nlist + j);
          if ((unsigned)nb >= (unsigned)n) {
            atomicOr(&st->error, kErrFormat);
            continue;
          }
          if (nb > v) {
            const int w = __ldg(a.eweight + j);
            if (keep_entry<KIND>(v, nb, w, thr)) {
              if (KIND == kLight || __ldcg(a.parent + nb) != rv) cnt++;
            }
          }
        }
      } else {
        ndesc = (unsigned)(((end - 1) >> kChunkLog) - (beg >> kChunkLog) + 1);
      }
    }
    unsigned pos, dpos;
    cta_reserve2(cnt, ndesc, wl_ctr, &st->desc_count, sm, pos, dpos);
    if (thread_row && cnt) {
      for (int j = beg; j < end; j++) {
        const int nb = __ldg(a.nlist + j);
        if ((unsigned)nb >= (unsigned)n || nb <= v) continue;
        const int w = __ldg(a.eweight + j);
        if (!keep_entry<KIND>(v, nb, w, thr)) continue;
        int rn = nb;
        if (KIND == kHeavy) {
          rn = __ldcg(a.parent + nb);
          if (rn == rv) continue;
        }
        if (pos < a.wl_cap) a.wl[pos] = make_int4(rv, rn, w, j);
        else atomicOr(&st->error, kErrOverflow);
        pos++;
      }
    }
    if (ndesc) {
      const int b0 = beg >> kChunkLog;
      for (unsigned k = 0; k < ndesc; k++) {
        if (dpos + k < a.desc_cap) a.desc[dpos + k] = make_int2(v, b0 + (int)k);
        else atomicOr(&st->error, kErrOverflow);
      }
    }
  }
  if (!grid_barrier(st, kBarrierTimeoutNs)) return;

  // Pass 2: one warp per 128-entry chunk of a long row, 4 entries per lane.
  const unsigned D = min(ld_volatile(&st->desc_count), a.desc_cap);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned wpc = blockDim.x >> 5;
  for (unsigned base = blockIdx.x * wpc; base < D; base += gridDim.x * wpc) {
    const unsigned d = base + warp;
    unsigned cnt = 0, mask = 0;
    int4 item[4];
    if (d < D) {
      const int2 ds = __ldcg(a.desc + d);
      const int v = ds.x;
      const int beg = __ldg(a.nindex + v), end = __ldg(a.nindex + v + 1);
      const int j0 = (ds.y << kChunkLog) + lane * 4;
      int nb[4], w[4];
      if (a.vec_ok && j0 + 3 < m) {
        const int4 q = __ldg(reinterpret_cast<const int4*>(a.nlist + j0));
        const int4 r = __ldg(reinterpret_cast<const int4*>(a.eweight + j0));
        nb[0] = q.x; nb[1] = q.y; nb[2] = q.z; nb[3] = q.w;
        w[0] = r.x; w[1] = r.y; w[2] = r.z; w[3] = r.w;
      } else {
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int j = j0 + q;
          const bool in = j >= beg && j < end;
          nb[q] = in ? __ldg(a.nlist + j) : -1;
          w[q] = in ? __ldg(a.eweight + j) : 0;
        }
      }
      const int rv = KIND == kHeavy ? __ldcg(a.parent + v) : v;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int j = j0 + q;
        item[q] = make_int4(rv, nb[q], w[q], j);
        if (j < beg || j >= end) continue;
        if ((unsigned)nb[q] >= (unsigned)n) {
          atomicOr(&st->error, kErrFormat);
          continue;
        }
        if (!keep_entry<KIND>(v, nb[q], w[q], thr)) continue;
        if (KIND == kHeavy) {
          item[q].y = __ldcg(a.parent + nb[q]);
          if (item[q].y == rv) continue;
        }
        mask |= 1u << q;
        cnt++;
      }
    }
    unsigned pos, unused;
    cta_reserve2(cnt, 0u, wl_ctr, nullptr, sm, pos, unused);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (!(mask & (1u << q))) continue;
      if (pos < a.wl_cap) a.wl[pos] = item[q];
      else atomicOr(&st->error, kErrOverflow);
      pos++;
    }
  }
}

// --------------------------------------------------------------- rounds
// kernel1 of one round (ECL_MST.cu:210-226) plus kernel3 of the previous
// round (:243-251): every input entry first clears its endpoints' slots in the
// previous round's min array, then resolves its endpoints to reps; entries
// still crossing two trees are compacted into `out` with their reps
// (implicit path compression, :218-219) and offer their key to both reps'
// slots with a guarded atomicMin (:221-223).
__device__ __forceinline__ void round_find_min(const RoundArgs& a, const int4* in, unsigned W,
                                               int4* out, unsigned* out_ctr, u64* mcur, u64* mprev,
                                               bool reset, unsigned start, unsigned stride,
                                               ReserveSmem& sm) {
  const unsigned tile = blockDim.x * kEPT;
  const unsigned ntiles = (W + tile - 1) / tile;
  unsigned long long atomics = 0;
  for (unsigned t = start; t < ntiles; t += stride) {
    int4 e[kEPT];
    bool keep[kEPT];
    unsigned cnt = 0;
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      const unsigned idx = t * tile + k * blockDim.x + threadIdx.x;
      keep[k] = false;
      if (idx < W) e[k] = __ldcg(in + idx);
    }
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      const unsigned idx = t * tile + k * blockDim.x + threadIdx.x;
      if (idx < W) {
        if (reset) {
          __stcg(mprev + e[k].x, kNoEdge);
          __stcg(mprev + e[k].y, kNoEdge);
        }
        const int ra = find_halve(e[k].x, a.parent);
        const int rb = find_halve(e[k].y, a.parent);
        keep[k] = ra != rb;
        e[k].x = ra;
        e[k].y = rb;
        cnt += keep[k];
      }
    }
    unsigned pos, unused;
    cta_reserve2(cnt, 0u, out_ctr, nullptr, sm, pos, unused);
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      if (!keep[k]) continue;
      if (pos < a.wl_cap) out[pos] = e[k];
      else atomicOr(&a.st->error, kErrOverflow);
      pos++;
      const u64 key = edge_key(e[k].z, e[k].w);
      if (__ldcg(mcur + e[k].x) > key) {
        atomicMin(mcur + e[k].x, key);
        atomics++;
      }
      if (__ldcg(mcur + e[k].y) > key) {
        atomicMin(mcur + e[k].y, key);
        atomics++;
      }
    }
  }
  if (a.count_atomics && atomics) atomicAdd(&a.st->atomics, atomics);
}

// kernel2 (ECL_MST.cu:229-240): an entry whose key is the minimum of either
// endpoint's slot is a forest edge; union the two trees and mark inMST[j].
__device__ __forceinline__ void round_mark(const RoundArgs& a, const int4* wl, unsigned W,
                                           const u64* mcur, unsigned start, unsigned stride) {
  const unsigned tile = blockDim.x * kEPT;
  const unsigned ntiles = (W + tile - 1) / tile;
  for (unsigned t = start; t < ntiles; t += stride) {
    int4 e[kEPT];
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      const unsigned idx = t * tile + k * blockDim.x + threadIdx.x;
      if (idx < W) e[k] = __ldcg(wl + idx);
    }
#pragma unroll
    for (int k = 0; k < kEPT; k++) {
      const unsigned idx = t * tile + k * blockDim.x + threadIdx.x;
      if (idx >= W) continue;
      const u64 key = edge_key(e[k].z, e[k].w);
      if (key == __ldcg(mcur + e[k].x) || key == __ldcg(mcur + e[k].y)) {
        cas_union(e[k].x, e[k].y, a.parent);
        a.inMST[e[k].w] = 1;
      }
    }
  }
}

__global__ void __launch_bounds__(kRoundThreads) k_rounds(RoundArgs a) {
  __shared__ ReserveSmem sm;
  DevState* st = a.st;
  const int ph = a.phase;
  if (ph == 1 && !st->filtered) return;
  // Only bits no CTA of this kernel can set, so every CTA takes the same exit.
  if (ld_volatile(&st->error) & (kErrFormat | kErrTimeout)) return;
  bool tail = false;
  int r = 0;
  for (;;) {
    const unsigned W = min(ld_volatile(&st->wl_count[ph][r]), a.wl_cap);
    if (W == 0) break;
    if (r >= ECL_MAX_ROUNDS) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&st->error, kErrRounds);
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
    round_find_min(a, in, W, out, &st->wl_count[ph][r + 1], mcur, mprev, r > 0, start, stride, sm);
    if (tail) __syncthreads();
    else if (!grid_barrier(st, kBarrierTimeoutNs)) return;
    const unsigned W2 = min(ld_volatile(&st->wl_count[ph][r + 1]), a.wl_cap);
    r++;
    if (W2 == 0) break;
    round_mark(a, out, W2, mcur, start, stride);
    if (tail) __syncthreads();
    else if (!grid_barrier(st, kBarrierTimeoutNs)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->rounds[ph] = r;
}

}  // namespace ecl

// =================================================================== host
struct ecl_mst_ctx {
  int device = 0;
  int sm_count = 0;
  int64_t max_nodes = 0, max_edges = 0;
  cudaStream_t stream = nullptr;
  // [minv0 | minv1 | parent] in one allocation (one L2 access-policy window)
  void* slots = nullptr;
  int* parent = nullptr;
  u64* minv0 = nullptr;
  u64* minv1 = nullptr;
  int4* wl[2] = {nullptr, nullptr};
  unsigned wl_cap = 0;
  int2* desc = nullptr;
  unsigned desc_cap = 0;
  DevState* st = nullptr;
  DevState* st_host = nullptr;  // pinned
  int scan_grid = 0, round_grid = 0;
  // device CSR + output for host-buffer runs (allocated on first use)
  int* d_nindex = nullptr;
  int* d_nlist = nullptr;
  int* d_eweight = nullptr;
  unsigned char* d_inMST = nullptr;
  cudaEvent_t ev[5] = {};
};

namespace {

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return ECL_OK;
  if (e == cudaErrorMemoryAllocation) return ECL_ERR_ALLOC;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return ECL_ERR_NO_DEVICE;
  return ECL_ERR_CUDA;
}

#define ECL_CUDA_TRY(call)                         \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

int device_error_status(unsigned err) {
  if (err & kErrTimeout) return ECL_ERR_TIMEOUT;
  if (err & kErrFormat) return ECL_ERR_FORMAT;
  if (err & kErrOverflow) return ECL_ERR_OVERFLOW;
  if (err & kErrRounds) return ECL_ERR_OVERFLOW;
  return ECL_OK;
}

int coop_grid(const void* fn, int threads, int sm_count) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0) != cudaSuccess)
    return 0;
  return per_sm * sm_count;
}

}  // namespace

extern "C" void ecl_default_opts(mst_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->threshold_mode = ECL_THRESH_HEURISTIC;
  o->quantile = 1.0f;
}

extern "C" int ecl_mst_ctx_create(int device, int64_t max_nodes, int64_t max_edges,
                                  ecl_mst_ctx** out) {
  if (!out || max_nodes < 1 || max_edges < 0 || max_nodes > INT32_MAX || max_edges > INT32_MAX)
    return ECL_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return ECL_ERR_NO_DEVICE;
  if (device < 0 || device >= ndev) return ECL_ERR_INVALID_ARG;
  ECL_CUDA_TRY(cudaSetDevice(device));
  ecl_mst_ctx* c = new (std::nothrow) ecl_mst_ctx();
  if (!c) return ECL_ERR_ALLOC;
  c->device = device;
  c->max_nodes = max_nodes;
  c->max_edges = max_edges;
  int st = ECL_OK;
  auto fail = [&](int s) {
    ecl_mst_ctx_destroy(c);
    return s;
  };
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return fail(ECL_ERR_CUDA);
  if (!prop.cooperativeLaunch) return fail(ECL_ERR_UNSUPPORTED);
  c->sm_count = prop.multiProcessorCount;
  if ((st = cuda_status(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)))) return fail(st);
  const size_t slot_bytes = (size_t)max_nodes * (2 * sizeof(u64) + sizeof(int));
  if ((st = cuda_status(cudaMalloc(&c->slots, slot_bytes)))) return fail(st);
  c->minv0 = (u64*)c->slots;
  c->minv1 = c->minv0 + max_nodes;
  c->parent = (int*)(c->minv1 + max_nodes);
  // A phase's worklist holds at most one entry per one-direction CSR entry,
  // i.e. at most `edges` (the reference sizes it edges/2, :279, which only
  // holds for symmetric inputs).
  c->wl_cap = (unsigned)std::max<int64_t>(max_edges, 1);
  for (int i = 0; i < 2; i++)
    if ((st = cuda_status(cudaMalloc(&c->wl[i], (size_t)c->wl_cap * sizeof(int4))))) return fail(st);
  // Chunk descriptors: a row of degree d >= 1 spans at most d/128 + 2 chunks.
  const int64_t dcap = max_edges / kChunk + 2 * std::min<int64_t>(max_nodes, max_edges) + 16;
  c->desc_cap = (unsigned)std::min<int64_t>(dcap, UINT_MAX);
  if ((st = cuda_status(cudaMalloc(&c->desc, (size_t)c->desc_cap * sizeof(int2))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->st, sizeof(DevState))))) return fail(st);
  if ((st = cuda_status(cudaHostAlloc(&c->st_host, sizeof(DevState), cudaHostAllocDefault))))
    return fail(st);
  for (auto& e : c->ev)
    if ((st = cuda_status(cudaEventCreate(&e)))) return fail(st);
  c->scan_grid = coop_grid((const void*)k_scan<kLight>, kScanThreads, c->sm_count);
  const int hg = coop_grid((const void*)k_scan<kHeavy>, kScanThreads, c->sm_count);
  c->scan_grid = std::min(c->scan_grid, hg);
  c->round_grid = coop_grid((const void*)k_rounds, kRoundThreads, c->sm_count);
  if (c->scan_grid <= 0 || c->round_grid <= 0) return fail(ECL_ERR_CUDA);
  *out = c;
  return ECL_OK;
}

extern "C" void ecl_mst_ctx_destroy(ecl_mst_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->slots);
  cudaFree(c->wl[0]);
  cudaFree(c->wl[1]);
  cudaFree(c->desc);
  cudaFree(c->st);
  cudaFreeHost(c->st_host);
  cudaFree(c->d_nindex);
  cudaFree(c->d_nlist);
  cudaFree(c->d_eweight);
  cudaFree(c->d_inMST);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" void* ecl_mst_ctx_stream(ecl_mst_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" int ecl_mst_ctx_sync(ecl_mst_ctx* c) {
  if (!c) return ECL_ERR_INVALID_ARG;
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  ECL_CUDA_TRY(cudaStreamSynchronize(c->stream));
  unsigned err = 0;
  ECL_CUDA_TRY(cudaMemcpy(&err, &c->st->error, sizeof(unsigned), cudaMemcpyDeviceToHost));
  return device_error_status(err);
}

namespace {

int launch_coop(const void* fn, int grid, int threads, void* arg, cudaStream_t s) {
  void* args[] = {arg};
  return cuda_status(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(threads), args, 0, s));
}

int enqueue_solve(ecl_mst_ctx* c, const ecl_graph* g, unsigned char* d_inMST, const mst_opts* o,
                  cudaStream_t s, bool timed) {
  const int n = g->nodes, m = g->edges;
  ECL_CUDA_TRY(cudaMemsetAsync(d_inMST, 0, (size_t)m, s));
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  int split = o->degree_split > 0 ? o->degree_split : kDefaultSplit;
  k_threshold<<<1, 1024, 0, s>>>(g->eweight, n, m, o->threshold_mode, o->threshold, o->quantile,
                                 split, c->st);
  ECL_CUDA_TRY(cudaGetLastError());
  ScanArgs sa;
  sa.nodes = n;
  sa.edges = m;
  sa.nindex = g->nindex;
  sa.nlist = g->nlist;
  sa.eweight = g->eweight;
  sa.parent = c->parent;
  sa.minv0 = c->minv0;
  sa.minv1 = c->minv1;
  sa.wl = c->wl[0];
  sa.wl_cap = c->wl_cap;
  sa.desc = c->desc;
  sa.desc_cap = c->desc_cap;
  sa.st = c->st;
  sa.vec_ok = ((((uintptr_t)g->nlist) | ((uintptr_t)g->eweight)) & 15) == 0;
  RoundArgs ra;
  ra.nodes = n;
  ra.wl0 = c->wl[0];
  ra.wl1 = c->wl[1];
  ra.wl_cap = c->wl_cap;
  ra.parent = c->parent;
  ra.minv0 = c->minv0;
  ra.minv1 = c->minv1;
  ra.inMST = d_inMST;
  ra.st = c->st;
  ra.small_tail = o->small_tail < 0 ? 0u : (o->small_tail == 0 ? kDefaultSmallTail : (unsigned)o->small_tail);
  if (o->flags & ECL_FLAG_NO_SMALL_TAIL) ra.small_tail = 0;
  ra.count_atomics = (o->flags & ECL_FLAG_STATS) ? 1 : 0;
  const int sgrid = std::max(1, std::min(c->scan_grid, (n + kScanThreads - 1) / kScanThreads + (m / kChunk) / 16 + 1));
  const int rgrid = std::max(1, std::min(c->round_grid, (m / 2 + kRoundThreads * kEPT - 1) / (kRoundThreads * kEPT) + 1));
  int st;
  if ((st = launch_coop((const void*)k_scan<kLight>, sgrid, kScanThreads, &sa, s))) return st;
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  ra.phase = 0;
  if ((st = launch_coop((const void*)k_rounds, rgrid, kRoundThreads, &ra, s))) return st;
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[2], s));
  ScanArgs sh = sa;
  if ((st = launch_coop((const void*)k_scan<kHeavy>, sgrid, kScanThreads, &sh, s))) return st;
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[3], s));
  ra.phase = 1;
  if ((st = launch_coop((const void*)k_rounds, rgrid, kRoundThreads, &ra, s))) return st;
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[4], s));
  return ECL_OK;
}

int fill_stats(ecl_mst_ctx* c, ecl_mst_stats* stats, bool timed) {
  ECL_CUDA_TRY(cudaMemcpyAsync(c->st_host, c->st, sizeof(DevState), cudaMemcpyDeviceToHost, c->stream));
  ECL_CUDA_TRY(cudaStreamSynchronize(c->stream));
  const DevState& h = *c->st_host;
  memset(stats, 0, sizeof(*stats));
  stats->threshold = h.threshold;
  stats->filtered = h.filtered;
  stats->degree_split = h.split;
  stats->rounds[0] = h.rounds[0];
  stats->rounds[1] = h.rounds[1];
  stats->status = (int32_t)h.error;
  for (int p = 0; p < 2; p++) {
    stats->scan_kept[p] = h.wl_count[p][0];
    for (int r = 0; r < ECL_MAX_ROUNDS; r++) stats->wl_in[p][r] = h.wl_count[p][r];
  }
  stats->atomics = (int64_t)h.atomics;
  if (timed) {
    float t01, t12, t23, t34, t04;
    cudaEventElapsedTime(&t01, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&t12, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&t23, c->ev[2], c->ev[3]);
    cudaEventElapsedTime(&t34, c->ev[3], c->ev[4]);
    cudaEventElapsedTime(&t04, c->ev[0], c->ev[4]);
    stats->ms_scan = t01 + t23;
    stats->ms_rounds = t12 + t34;
    stats->ms_total = t04;
  }
  return device_error_status(h.error);
}

int check_graph_args(const ecl_mst_ctx* c, const ecl_graph* g, const void* inMST) {
  if (!c || !g || !inMST) return ECL_ERR_INVALID_ARG;
  if (g->nodes < 1 || g->edges < 0) return ECL_ERR_INVALID_ARG;
  if (g->nodes > c->max_nodes || g->edges > c->max_edges) return ECL_ERR_TOO_LARGE;
  if (!g->nindex || (g->edges > 0 && (!g->nlist || !g->eweight))) return ECL_ERR_INVALID_ARG;
  return ECL_OK;
}

int check_opts(const mst_opts* o) {
  if (o->threshold_mode < ECL_THRESH_HEURISTIC || o->threshold_mode > ECL_THRESH_LEARNED)
    return ECL_ERR_INVALID_ARG;
  if (o->degree_split < 0 || o->degree_split > (1 << 20)) return ECL_ERR_INVALID_ARG;
  if (o->threshold_mode == ECL_THRESH_QUANTILE && !(o->quantile >= 0.0f)) return ECL_ERR_INVALID_ARG;
  return ECL_OK;
}

}  // namespace

// Learned threshold/split: extracts graph features on the device and runs the
// trained MLP, writing DevState::quantile and DevState::learned_split.
int ecl_learned_prepare(ecl_mst_ctx* c, const ecl_graph* d_graph, cudaStream_t s, void* st);

extern "C" int ecl_mst_run_device(ecl_mst_ctx* c, const ecl_graph* g, uint8_t* d_inMST,
                                  const mst_opts* opts, void* stream, ecl_mst_stats* stats) {
  int st = check_graph_args(c, g, d_inMST);
  if (st) return st;
  mst_opts o;
  if (opts) o = *opts;
  else ecl_default_opts(&o);
  if ((st = check_opts(&o))) return st;
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  if (g->edges == 0) {
    if (stats) {
      memset(stats, 0, sizeof(*stats));
      stats->threshold = INT_MAX;
    }
    return ECL_OK;
  }
  ECL_CUDA_TRY(cudaMemsetAsync(c->st, 0, sizeof(DevState), s));
  if (o.threshold_mode == ECL_THRESH_LEARNED) {
    if ((st = ecl_learned_prepare(c, g, s, c->st))) return st;
  }
  if ((st = enqueue_solve(c, g, d_inMST, &o, s, stats != nullptr))) return st;
  if (stats) {
    if (s != c->stream) {
      ECL_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return fill_stats(c, stats, true);
  }
  return ECL_OK;
}

extern "C" int ecl_mst_ctx_run_host(ecl_mst_ctx* c, const ecl_graph* g, uint8_t* inMST,
                                    const mst_opts* opts, ecl_mst_stats* stats) {
  int st = check_graph_args(c, g, inMST);
  if (st) return st;
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  const size_t nb = ((size_t)c->max_nodes + 1) * 4, eb = (size_t)std::max<int64_t>(c->max_edges, 1) * 4;
  if (!c->d_nindex) {
    ECL_CUDA_TRY(cudaMalloc(&c->d_nindex, nb));
    ECL_CUDA_TRY(cudaMalloc(&c->d_nlist, eb));
    ECL_CUDA_TRY(cudaMalloc(&c->d_eweight, eb));
    ECL_CUDA_TRY(cudaMalloc(&c->d_inMST, eb / 4));
  }
  const int n = g->nodes, m = g->edges;
  ECL_CUDA_TRY(cudaMemcpyAsync(c->d_nindex, g->nindex, ((size_t)n + 1) * 4, cudaMemcpyHostToDevice, c->stream));
  if (m > 0) {
    ECL_CUDA_TRY(cudaMemcpyAsync(c->d_nlist, g->nlist, (size_t)m * 4, cudaMemcpyHostToDevice, c->stream));
    ECL_CUDA_TRY(cudaMemcpyAsync(c->d_eweight, g->eweight, (size_t)m * 4, cudaMemcpyHostToDevice, c->stream));
  }
  ecl_graph dg = {n, m, c->d_nindex, c->d_nlist, c->d_eweight};
  if ((st = ecl_mst_run_device(c, &dg, c->d_inMST, opts, c->stream, stats))) return st;
  if (m > 0)
    ECL_CUDA_TRY(cudaMemcpyAsync(inMST, c->d_inMST, (size_t)m, cudaMemcpyDeviceToHost, c->stream));
  if ((st = ecl_mst_ctx_sync(c))) return st;
  if (stats) {
    int64_t fe = 0;
    uint64_t fw = 0;
    for (int j = 0; j < m; j++)
      if (inMST[j]) {
        fe++;
        fw += (uint64_t)(int64_t)g->eweight[j];
      }
    stats->forest_edges = fe;
    stats->forest_weight = fw;
  }
  return ECL_OK;
}

extern "C" int ecl_mst_run(const ecl_graph* g, uint8_t* inMST, const mst_opts* opts,
                           ecl_mst_stats* stats) {
  if (!g || !inMST || g->nodes < 1 || g->edges < 0) return ECL_ERR_INVALID_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ECL_ERR_NO_DEVICE;
  ecl_mst_ctx* c = nullptr;
  int st = ecl_mst_ctx_create(dev, g->nodes, g->edges, &c);
  if (st) return st;
  st = ecl_mst_ctx_run_host(c, g, inMST, opts, stats);
  ecl_mst_ctx_destroy(c);
  return st;
}

extern "C" int ecl_host_alloc_pinned(size_t bytes, void** out) {
  if (!out) return ECL_ERR_INVALID_ARG;
  *out = nullptr;
  ECL_CUDA_TRY(cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault));
  return ECL_OK;
}

extern "C" void ecl_host_free_pinned(void* p) {
  if (p) cudaFreeHost(p);
}
