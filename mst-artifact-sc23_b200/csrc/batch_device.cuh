// Batched engine: thousands of graphs of uneven sizes in one persistent
// launch. Each CTA takes the next graph from a device work queue and runs the
// whole reference algorithm on it (initPM, initWL<true>, rounds, initWL<false>,
// rounds: ECL_MST.cu:305-340) with CTA barriers only, so every graph ends its
// own rounds when its worklist empties. Graphs too large for one CTA's
// scratch go through the grid-wide single-graph engine instead.
#pragma once
#include "mst_device.cuh"

namespace ecl {

struct BatchArgs {
  int num_small;
  const int* small_list;        // graph ids taken by the persistent kernel, largest first
  const long long* node_off;    // [graphs + 1]
  const long long* edge_off;    // [graphs + 1]
  const int* nindex;            // graph g's nindex (n_g + 1 local offsets) at node_off[g] + g
  const int* nlist;             // local neighbour ids at edge_off[g]
  const int* eweight;
  unsigned char* inMST;         // at edge_off[g]
  int* parent_pool;             // per CTA: cap_n
  u64* minv_pool;               // per CTA: 2 * cap_n
  int4* wl_pool;                // per CTA: 2 * cap_m
  int cap_n, cap_m;
  unsigned* queue;              // work queue head
  DevState* st;                 // shared error word / atomics counter
  int mode, explicit_thr;
  float quantile;
  int count_atomics;
  unsigned abl;                 // round-kernel ablation switches (kAbl*)
};

// Threshold of one graph by the chosen rule (the reference heuristic per
// input graph, as its main applies it, ECL_MST.cu:408,432-440). One thread.
__device__ __forceinline__ void batch_threshold(const BatchArgs& b, const int* ew, int n, int m,
                                                int* thr, int* filtered) {
  if (b.mode == ECL_THRESH_NONE || m == 0) {
    *filtered = 0;
    *thr = INT_MAX;
    return;
  }
  if (b.mode == ECL_THRESH_EXPLICIT) {
    *filtered = 1;
    *thr = b.explicit_thr;
    return;
  }
  if (b.mode == ECL_THRESH_QUANTILE) {
    if (!(b.quantile < 1.0f)) {
      *filtered = 0;
      *thr = INT_MAX;
      return;
    }
    // quantile of 64 hashed samples (insertion sort), enough for a schedule hint
    int s[64];
    const int ns = m < 64 ? m : 64;
    for (int i = 0; i < ns; i++) {
      const uint64_t r = ecl_mix64(0x5EED0000ull + (uint64_t)i);
      const int x = ew[(unsigned)(r % (uint64_t)(unsigned)m)];
      int k = i - 1;
      while (k >= 0 && s[k] > x) {
        s[k + 1] = s[k];
        k--;
      }
      s[k + 1] = x;
    }
    int idx = (int)(b.quantile * (float)(ns - 1));
    idx = idx < 0 ? 0 : (idx > ns - 1 ? ns - 1 : idx);
    *filtered = 1;
    *thr = s[idx];
    return;
  }
  if (m / n < 4) {
    *filtered = 0;
    *thr = INT_MAX;
    return;
  }
  int s[20];
  const int ns = m < 20 ? m : 20;
  for (int i = 0; i < ns; i++) {
    unsigned val = (unsigned)i;
    val = ((val >> 16) ^ val) * 0x45d9f3bu;
    val = ((val >> 16) ^ val) * 0x45d9f3bu;
    val = (val >> 16) ^ val;
    const int x = ew[val % (unsigned)m];
    int k = i - 1;
    while (k >= 0 && s[k] > x) {
      s[k + 1] = s[k];
      k--;
    }
    s[k + 1] = x;
  }
  *filtered = 1;
  *thr = s[min(19, (int)(3.0 * n * ns / m))];
}

// CTA-wide scan of one graph's CSR (initWL, ECL_MST.cu:157-207): each thread
// takes 4 consecutive entries, finds their vertex by binary search over the
// graph's nindex (small, cache resident) and appends one-direction entries of
// the phase with one smem-counter reservation per tile.
template <int KIND>
__device__ void cta_scan(const int* ni, const int* nl, const int* ew, int n, int m, int thr,
                         int* parent, int4* wl, unsigned cap, unsigned* ctr, unsigned char* out,
                         DevState* st, ReserveSmem& rs) {
  constexpr int E = 4;
  const int tile = blockDim.x * E;
  for (int base = 0; base < m; base += tile) {
    const int j0 = base + threadIdx.x * E;
    int nb[E], w[E], vtx[E], nrep[E];
    unsigned keep = 0, cnt = 0;
#pragma unroll
    for (int q = 0; q < E; q++) {
      const bool in = j0 + q < m;
      nb[q] = in ? __ldg(nl + j0 + q) : -1;
      w[q] = in ? __ldg(ew + j0 + q) : 0;
      if (KIND == kLight && in) out[j0 + q] = 0;
    }
    if (j0 < m) {
      int lo = 0, hi = n;  // last vertex with nindex <= j0
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(ni + mid) <= j0) lo = mid;
        else hi = mid;
      }
      int v = lo, row_end = __ldg(ni + v + 1);
      int cur_v = -1, cur_rep = -1;
#pragma unroll
      for (int q = 0; q < E; q++) {
        const int j = j0 + q;
        vtx[q] = 0;
        nrep[q] = nb[q];
        if (j >= m) continue;
        while (j >= row_end && v < n - 1) row_end = __ldg(ni + (++v) + 1);
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
            cur_rep = __ldcg(parent + v);
          }
          rv = cur_rep;
          nrep[q] = __ldcg(parent + nb[q]);
          if (nrep[q] == rv) continue;
        }
        vtx[q] = rv;
        keep |= 1u << q;
        cnt++;
      }
    }
    unsigned pos, unused;
    cta_reserve2(cnt, 0u, ctr, nullptr, rs, pos, unused);
#pragma unroll
    for (int q = 0; q < E; q++) {
      if (!(keep & (1u << q))) continue;
      if (pos < cap) wl[pos] = make_int4(vtx[q], nrep[q], w[q], j0 + q);
      else atomicOr(&st->error, kErrOverflow);
      pos++;
    }
  }
}

// All Boruvka rounds of one phase of one graph inside the CTA.
__device__ void cta_rounds(RoundArgs& ra, unsigned* cnt, RoundSmem& s) {
  int r = 0;
  for (;;) {
    const unsigned W = min(((volatile unsigned*)cnt)[r], ra.wl_cap);
    if (W == 0) break;
    if (r >= ECL_MAX_ROUNDS) {
      if (threadIdx.x == 0) atomicOr(&ra.st->error, kErrRounds);
      break;
    }
    const bool odd = (r & 1) != 0;
    const int4* in = odd ? ra.wl1 : ra.wl0;
    int4* out = odd ? ra.wl0 : ra.wl1;
    u64* mcur = odd ? ra.minv1 : ra.minv0;
    u64* mprev = odd ? ra.minv0 : ra.minv1;
    round_find_min(ra, in, W, out, &cnt[r + 1], &cnt[ECL_MAX_ROUNDS + 1], mcur, mprev,
                   r > 0 ? kResetSparse : kResetNone, false, 0u, 1u, s);
    __syncthreads();
    const unsigned W2 = min(((volatile unsigned*)cnt)[r + 1], ra.wl_cap);
    r++;
    if (W2 == 0) break;
    hot_refresh(mcur, s);
    round_mark(ra, out, W2, mcur, 0u, 1u, s);
    __syncthreads();
    round_smem_clear(s);
    __syncthreads();
  }
  __syncthreads();
  round_smem_clear(s);
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads, 2) k_batch_small(BatchArgs b) {
  __shared__ RoundSmem s;
  __shared__ unsigned cnt[ECL_MAX_ROUNDS + 2];  // per-round entry counts, then a kept-count sink
  __shared__ int sh_g, sh_thr, sh_filtered;
  int* parent = b.parent_pool + (size_t)blockIdx.x * b.cap_n;
  u64* minv0 = b.minv_pool + (size_t)blockIdx.x * 2 * b.cap_n;
  u64* minv1 = minv0 + b.cap_n;
  int4* wl0 = b.wl_pool + (size_t)blockIdx.x * 2 * b.cap_m;
  int4* wl1 = wl0 + b.cap_m;
  round_smem_clear(s);
  seg_set_dense(s, 0);  // one CTA per graph: every round list is dense from 0
  __syncthreads();
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned gi = atomicAdd(b.queue, 1u);
      sh_g = gi < (unsigned)b.num_small ? b.small_list[gi] : -1;
    }
    __syncthreads();
    const int g = sh_g;
    if (g < 0) break;
    const long long n0 = b.node_off[g], e0 = b.edge_off[g];
    const int n = (int)(b.node_off[g + 1] - n0), m = (int)(b.edge_off[g + 1] - e0);
    const int* ni = b.nindex + n0 + g;
    const int* nl = b.nlist + e0;
    const int* ew = b.eweight + e0;
    unsigned char* out = b.inMST + e0;
    if (threadIdx.x == 0) {
      int t, f;
      batch_threshold(b, ew, n, m, &t, &f);
      sh_thr = t;
      sh_filtered = f;
    }
    for (int i = threadIdx.x; i <= ECL_MAX_ROUNDS; i += blockDim.x) cnt[i] = 0;
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
      parent[v] = v;
      minv0[v] = kNoEdge;
      minv1[v] = kNoEdge;
    }
    __syncthreads();
    const int thr = sh_thr, filtered = sh_filtered;
    RoundArgs ra{};
    ra.phase = 0;
    ra.nodes = n;
    ra.wl0 = wl0;
    ra.wl1 = wl1;
    ra.wl_cap = (unsigned)b.cap_m;
    ra.parent = parent;
    ra.minv0 = minv0;
    ra.minv1 = minv1;
    ra.inMST = out;
    ra.st = b.st;
    ra.small_tail = 0;
    ra.count_atomics = b.count_atomics;
    ra.abl = b.abl;
    cta_scan<kLight>(ni, nl, ew, n, m, thr, parent, wl0, ra.wl_cap, &cnt[0], out, b.st, s.rs);
    __syncthreads();
    cta_rounds(ra, cnt, s);
    if (filtered) {
      for (int v = threadIdx.x; v < n; v += blockDim.x) __stcg(parent + v, find_ro(v, parent));
      for (int i = threadIdx.x; i <= ECL_MAX_ROUNDS; i += blockDim.x) cnt[i] = 0;
      __syncthreads();
      cta_scan<kHeavy>(ni, nl, ew, n, m, thr, parent, wl0, ra.wl_cap, &cnt[0], out, b.st, s.rs);
      __syncthreads();
      cta_rounds(ra, cnt, s);
    }
  }
}

}  // namespace ecl
