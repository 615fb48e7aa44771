// Device building blocks of the B200 ECL-MST engine: coherent loads, the
// bounded grid barrier, CTA-aggregated worklist reservation, find with path
// halving and the CAS union. Shared by the single-graph engine (ecl_mst.cu)
// and the batched engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ecl_mst.h"

namespace ecl {

typedef unsigned long long u64;

// Device error word bits (DevState::error).
enum : unsigned {
  kErrFormat = 1u,    // nindex not monotone / out of range, or nlist id >= nodes
  kErrOverflow = 2u,  // a worklist or descriptor buffer ran out of room
  kErrTimeout = 4u,   // a grid barrier waited past its limit
  kErrRounds = 8u     // more Boruvka rounds than ECL_MAX_ROUNDS
};

// Most CTAs a round-kernel launch may have: each CTA of a find/min pass
// writes its kept entries as one segment of the round's output list.
constexpr int kMaxRoundCtas = 1024;

constexpr int kChunkLog = 7;  // long rows are scanned in aligned 128-entry chunks
constexpr int kChunk = 1 << kChunkLog;
constexpr u64 kNoEdge = ~0ull;

// Degree statistics of the learned schedule's features, summed over all
// vertices (row degree = nindex[v + 1] - nindex[v]).
struct FeatAcc {
  unsigned long long deg_sum, deg_sq, zero, low, high;  // sum d, sum d^2, #d = 0, #d < 4, #d >= 32
  unsigned max_deg;
};

// One thread's part of the degree statistics.
struct FeatPart {
  unsigned long long d1 = 0, d2 = 0, z = 0, lo = 0, hi = 0;
  unsigned mx = 0;
  __device__ __forceinline__ void add(unsigned d) {
    d1 += d;
    d2 += (unsigned long long)d * d;
    z += d == 0;
    lo += d < 4;
    hi += d >= 32;
    mx = max(mx, d);
  }
  // Fold the CTA's parts into `acc`: warp shuffles, one shared-memory pass,
  // one atomic per counter per CTA. Every thread of the CTA (kBlock threads)
  // must call this.
  template <int kBlock>
  __device__ __forceinline__ void fold(FeatAcc* acc) {
    __shared__ unsigned long long part[5][kBlock / 32];
    __shared__ unsigned pmax[kBlock / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      d1 += __shfl_down_sync(0xffffffffu, d1, o);
      d2 += __shfl_down_sync(0xffffffffu, d2, o);
      z += __shfl_down_sync(0xffffffffu, z, o);
      lo += __shfl_down_sync(0xffffffffu, lo, o);
      hi += __shfl_down_sync(0xffffffffu, hi, o);
      mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
      part[0][w] = d1;
      part[1][w] = d2;
      part[2][w] = z;
      part[3][w] = lo;
      part[4][w] = hi;
      pmax[w] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int i = 1; i < kBlock / 32; i++) {
        for (int k = 0; k < 5; k++) part[k][0] += part[k][i];
        pmax[0] = max(pmax[0], pmax[i]);
      }
      atomicAdd(&acc->deg_sum, part[0][0]);
      atomicAdd(&acc->deg_sq, part[1][0]);
      atomicAdd(&acc->zero, part[2][0]);
      atomicAdd(&acc->low, part[3][0]);
      atomicAdd(&acc->high, part[4][0]);
      atomicMax(&acc->max_deg, pmax[0]);
    }
  }
};

// Control block of one solve, zeroed before every solve.
struct DevState {
  int threshold;       // light phase keeps w <= threshold
  int filtered;        // 1 = light + heavy phase, 0 = one unfiltered phase
  int split;           // degree split between the thread and the chunk tier
  unsigned error;      // kErr* bits
  unsigned bar_count;  // grid barrier: CTAs arrived in the current generation
  unsigned bar_gen;    // grid barrier: generation counter
  int rounds[2];       // Boruvka rounds per phase
  unsigned desc_count; // long-row chunk descriptors emitted by the current scan
  unsigned pad;
  float quantile;      // learned / quantile modes: filter quantile in [0,1]
  int learned_split;   // learned mode: predicted degree split
  u64 atomics;         // guarded atomicMin issued (stats mode)
  unsigned wl_count[2][ECL_MAX_ROUNDS + 1];  // [phase][r] = entries entering round r
  // globaltimer stamps taken by CTA 0 at phase boundaries (diagnostics):
  // [phase][2r] after round r's find/min pass, [phase][2r+1] after its mark pass
  u64 t_round_start[2];
  u64 t_round[2][2 * ECL_MAX_ROUNDS];
  unsigned scan_kept[2];  // entries each scan kept (wl_count[p][0] also counts padding)
  unsigned wl_kept[2][ECL_MAX_ROUNDS + 1];  // [phase][r + 1] = entries round r kept (no padding)
  // The last find/min pass's output list, one segment per CTA: CTA b wrote
  // seg_cnt[b] entries from position seg_off[b] (written before the grid
  // barrier that ends the pass, read after it).
  unsigned seg_cnt[kMaxRoundCtas];
  unsigned seg_off[kMaxRoundCtas];
};

__device__ __forceinline__ u64 globaltimer_ns() {
  u64 t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_volatile(const unsigned* p) {
  return *(const volatile unsigned*)p;
}

// Grid-wide barrier for cooperative launches among the `expected` CTAs
// still in the launch (the others have left for good). Every wait is bounded
// by `timeout_ns`; on expiry the kErrTimeout bit is set and all later
// barriers return at once, so a stuck CTA turns into an error status instead
// of a hang. Returns false once the timeout bit is set.
__device__ __forceinline__ bool grid_barrier(DevState* st, u64 timeout_ns, unsigned expected) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned gen = ld_volatile(&st->bar_gen);
    __threadfence();
    const unsigned arrived = atomicAdd(&st->bar_count, 1u);
    if (arrived == expected - 1) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      const u64 t0 = globaltimer_ns();
      unsigned ns = 32;
      while (ld_volatile(&st->bar_gen) == gen) {
        if (ld_volatile(&st->error) & kErrTimeout) break;
        if (globaltimer_ns() - t0 > timeout_ns) {
          atomicOr(&st->error, kErrTimeout);
          break;
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
      }
    }
    __threadfence();
  }
  __syncthreads();
  return (ld_volatile(&st->error) & kErrTimeout) == 0;
}

// ---- mbarriers and bulk asynchronous copies (cp.async.bulk, no multicast)
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(u64* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the asynchronous copy unit.
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(u64* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Arrive and add `bytes` to the transaction count the phase waits for.
__device__ __forceinline__ void mbar_arrive_tx(u64* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Test for the phase's completion; if it is not complete the thread is
// suspended until it completes or about 20 us pass (no busy spinning).
__device__ __forceinline__ bool mbar_try_wait(u64* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"(20000u)
      : "memory");
  return ok != 0;
}

// Wait for the phase of the given parity to complete, for at most
// `timeout_ns`; false on expiry.
__device__ __forceinline__ bool mbar_wait(u64* bar, unsigned parity, u64 timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const u64 t0 = globaltimer_ns();
  while (!mbar_try_wait(bar, parity))
    if (globaltimer_ns() - t0 > timeout_ns) return false;
  return true;
}

// Orders this thread's generic-proxy shared-memory accesses before later
// asynchronous-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Global -> shared bulk copy of `bytes` (multiple of 16, both addresses
// 16-byte aligned); completion is counted on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, u64* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// ---- L2 eviction priorities (createpolicy + .L2::cache_hint, sm_80 and
// later). Streams read once (the CSR in the scans) are marked evict-first so
// they do not push out the small arrays every thread gathers from (parent[],
// the min slots), which are marked evict-last where they are read.
__device__ __forceinline__ u64 l2_policy_evict_first() {
  u64 p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ u64 l2_policy_evict_last() {
  u64 p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// Global -> shared bulk copy as bulk_g2s, with an L2 cache policy.
__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, unsigned bytes, u64* bar, u64 policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// 32-bit global load through L2 (no L1 allocation) with an L2 cache policy.
__device__ __forceinline__ int ld_cg_hint(const int* p, u64 policy) {
  int v;
  asm volatile("ld.global.cg.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(policy));
  return v;
}

// Shared memory of one CTA-wide two-counter reservation.
struct ReserveSmem {
  unsigned warp_off[32][2];
  unsigned base[2];
};

// CTA-aggregated reservation of c0 slots in counter ctr0 and c1 slots in
// counter ctr1 (ctr1 may be null when every c1 is 0): one warp-shuffle scan,
// one scan over warp totals and at most one global atomic per counter per CTA.
// Every thread of the CTA must call it (it contains __syncthreads).
__device__ __forceinline__ void cta_reserve2(unsigned c0, unsigned c1, unsigned* ctr0,
                                             unsigned* ctr1, ReserveSmem& sm, unsigned& pos0,
                                             unsigned& pos1) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned s0 = c0, s1 = c1;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t0 = __shfl_up_sync(0xffffffffu, s0, o);
    const unsigned t1 = __shfl_up_sync(0xffffffffu, s1, o);
    if (lane >= o) {
      s0 += t0;
      s1 += t1;
    }
  }
  if (lane == 31) {
    sm.warp_off[warp][0] = s0;
    sm.warp_off[warp][1] = s1;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    const unsigned w0 = lane < nw ? sm.warp_off[lane][0] : 0u;
    const unsigned w1 = lane < nw ? sm.warp_off[lane][1] : 0u;
    unsigned x0 = w0, x1 = w1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t0 = __shfl_up_sync(0xffffffffu, x0, o);
      const unsigned t1 = __shfl_up_sync(0xffffffffu, x1, o);
      if (lane >= o) {
        x0 += t0;
        x1 += t1;
      }
    }
    if (lane < nw) {
      sm.warp_off[lane][0] = x0 - w0;
      sm.warp_off[lane][1] = x1 - w1;
    }
    if (lane == 31) {
      sm.base[0] = x0 ? atomicAdd(ctr0, x0) : 0u;
      sm.base[1] = x1 ? atomicAdd(ctr1, x1) : 0u;
    }
  }
  __syncthreads();
  pos0 = sm.base[0] + sm.warp_off[warp][0] + (s0 - c0);
  pos1 = sm.base[1] + sm.warp_off[warp][1] + (s1 - c1);
  __syncthreads();
}

// Union-find order. A root is hooked under a root of higher priority, where
// the priority is a fixed bijective 32-bit mix of the vertex id (the
// MurmurHash3 finalizer): parent pointers therefore always lead to strictly
// higher priority, so every walk ends and no cycle can form, and because the
// priorities are a random permutation of the ids, the chains built when many
// components merge in one round stay short in expectation (hooking by id, as
// the reference join does with max -> min at ECL_MST.cu:137-144, builds a
// chain as long as any id-monotone path of merging components).
__device__ __forceinline__ unsigned uf_prio(int v) {
  unsigned h = (unsigned)v;
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

// Root of v. Path splitting (each visited node is re-pointed to its
// grandparent) is applied on the way: it only shortcuts inside one tree, so
// concurrent finds still reach the same root. Must not run concurrently with
// unions.
__device__ __forceinline__ int find_halve(int v, int* parent) {
  int p = __ldcg(parent + v);
  while (p != v) {
    const int gp = __ldcg(parent + p);
    if (gp != p) __stcg(parent + v, gp);
    v = p;
    p = gp;
  }
  return v;
}

// Read-only root walk (no writes); safe next to unions.
__device__ __forceinline__ int find_ro(int v, const int* parent) {
  int p = __ldcg(parent + v);
  while (p != v) {
    v = p;
    p = __ldcg(parent + v);
  }
  return v;
}

// Union of the trees holding a and b (ECL_MST.cu:137-144): CAS-hook the
// lower-priority node under the higher-priority one if it is still a root;
// a failed CAS returns its current parent, which has higher priority, so the
// lower priority of the pair strictly increases and the loop ends.
__device__ __forceinline__ void cas_union(int a, int b, int* parent) {
  while (a != b) {
    if (uf_prio(a) > uf_prio(b)) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicCAS(parent + a, a, b);
    if (old == a) return;
    a = old;
  }
}

// Tuple key of an edge: (uint32 weight, edge index), as ((ull)w << 32) | j.
__device__ __forceinline__ u64 edge_key(int w, int j) {
  return ((u64)(unsigned)w << 32) | (u64)(unsigned)j;
}

}  // namespace ecl
