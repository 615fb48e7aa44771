// GPU-side graph preprocessing.
//
//   ecl_csr_from_pairs_device   undirected pair list -> symmetric,
//                               deduplicated, self-loop-free ECLgraph CSR
//   ecl_gen_*_device            the four synthetic families drawn on the
//                               device, identical to the host generators
//                               (generators.cpp) entry for entry
//   ecl_gen_batch_device        the mixed batch packed into one ecl_batch
//
// The reference prepares its inputs on the host: the benchmark graphs are
// downloaded .egr files (Inputs/download_inputs.sh), and its converters
// (PBBS_CPU/inputs/ecl2pbbs_genweights.cpp, cuGraph_GPU/inputs/
// ecl2mtx_genweights_cugraph.cpp) walk the CSR serially. Here a CSR is built
// by one radix sort of (row, neighbour) keys, a scan of run-head flags and
// one emit pass that writes nlist, eweight and the row offsets. All of it is
// HBM-bound integer work; the sort and the scan are CUB's device primitives.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "ecl_mst.h"
#include "internal.h"

namespace {

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return ECL_OK;
  if (e == cudaErrorMemoryAllocation) return ECL_ERR_ALLOC;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return ECL_ERR_NO_DEVICE;
  return ECL_ERR_CUDA;
}

#define PP_TRY(call)                               \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

#define PP_CHECK(expr)       \
  do {                       \
    const int st_ = (expr);  \
    if (st_) return st_;     \
  } while (0)

constexpr int kPT = 256;  // threads per block of every kernel in this file

int sm_count() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) return 148;
  return sms;
}

// Grid-stride launches: at most 8 blocks of 256 threads per SM.
int blocks_for(int64_t items) {
  const int64_t want = (std::max<int64_t>(items, 1) + kPT - 1) / kPT;
  return (int)std::min<int64_t>(want, (int64_t)sm_count() * 8);
}

// Bits of a vertex id: the smallest b >= 1 with 2^b >= nodes.
int id_bits(int64_t nodes) {
  int b = 1;
  while ((1ll << b) < nodes) b++;
  return b;
}

// Scratch comes from a private stream-ordered pool per device that keeps its
// memory between calls (a batch of thousands of graphs reuses one reservation
// instead of calling cudaMalloc per graph). Each public call trims it when it
// returns.
cudaMemPool_t scratch_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

struct Scratch {
  cudaStream_t s;
  cudaMemPool_t pool;
  std::vector<void*> held;
  explicit Scratch(cudaStream_t st) : s(st), pool(scratch_pool()) {}
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
  ~Scratch() { release(); }
  void release() {
    for (void* p : held) cudaFreeAsync(p, s);
    held.clear();
  }
  template <class T>
  int get(T** p, size_t count) {
    if (!pool) return ECL_ERR_CUDA;
    void* q = nullptr;
    PP_TRY(cudaMallocFromPoolAsync(&q, std::max<size_t>(count, 1) * sizeof(T), pool, s));
    held.push_back(q);
    *p = static_cast<T*>(q);
    return ECL_OK;
  }
};

// Releases the pool's memory when a public call returns.
struct TrimOnExit {
  cudaStream_t s;
  ~TrimOnExit() {
    cudaStreamSynchronize(s);
    if (cudaMemPool_t p = scratch_pool()) cudaMemPoolTrimTo(p, 0);
  }
};

__device__ __forceinline__ int64_t gtid() { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int64_t gstride() { return (int64_t)gridDim.x * blockDim.x; }

// Sum over the block, added once to *total.
__device__ void block_add(unsigned long long mine, unsigned long long* total) {
  __shared__ unsigned long long part[kPT / 32];
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = mine;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < kPT / 32; w++) t += part[w];
    if (t) atomicAdd(total, t);
  }
}

// Both directions of every pair as (row << bits | neighbour) keys. Self-loops
// and out-of-range ids become the all-ones key, which sorts after every real
// key (a real key has row != neighbour); out-of-range ids also set *bad.
__global__ void __launch_bounds__(kPT) k_pair_keys(int64_t pairs, const int32_t* __restrict__ u,
                                                   const int32_t* __restrict__ v, const int32_t* __restrict__ w,
                                                   uint32_t nodes, int bits, ulonglong2* __restrict__ keys,
                                                   uint2* __restrict__ vals, unsigned long long* dropped,
                                                   unsigned* bad) {
  const uint64_t none = (1ull << (2 * bits)) - 1;
  unsigned long long mine = 0;
  bool oob_seen = false;
  for (int64_t i = gtid(); i < pairs; i += gstride()) {
    const uint32_t a = (uint32_t)u[i], b = (uint32_t)v[i];
    const bool oob = a >= nodes || b >= nodes;
    oob_seen |= oob;
    ulonglong2 k = make_ulonglong2(none, none);
    if (!oob && a != b) {
      k.x = ((uint64_t)a << bits) | b;
      k.y = ((uint64_t)b << bits) | a;
    } else {
      mine += 2;
    }
    keys[i] = k;
    if (vals) {
      const uint32_t x = (uint32_t)w[i];
      vals[i] = make_uint2(x, x);
    }
  }
  if (oob_seen) atomicOr(bad, 1u);
  block_add(mine, dropped);
}

// flags[i] = 1 where sorted key i starts a run of equal keys (i < valid);
// flags[valid] = 0, so the exclusive scan's last entry is the run count.
__global__ void __launch_bounds__(kPT) k_run_heads(int64_t valid, const uint64_t* __restrict__ keys,
                                                   uint32_t* __restrict__ flags) {
  for (int64_t i = gtid(); i <= valid; i += gstride())
    flags[i] = (i < valid && (i == 0 || keys[i] != keys[i - 1])) ? 1u : 0u;
}

// One entry per run: nlist, the weight by `rule`, and the row offsets. The
// head of the first run of row a writes nindex[r] for every r after the
// previous run's row up to a (rows without entries in between start there
// too); the last key writes the offsets after its row. With the given-weight
// rule every key of a run folds its weight into the run's entry with an
// unsigned atomicMin (eweight preset to all ones), so duplicate pairs keep
// the weight the MST order (uint32 weight, then entry) prefers.
__global__ void __launch_bounds__(kPT) k_emit_csr(int64_t valid, const uint64_t* __restrict__ keys,
                                                  const uint32_t* __restrict__ vals,
                                                  const uint32_t* __restrict__ pos, int bits, int32_t nodes,
                                                  int rule, uint64_t seed, int32_t wmax, int32_t* __restrict__ nindex,
                                                  int32_t* __restrict__ nlist, int32_t* __restrict__ eweight) {
  const uint64_t mask = (1ull << bits) - 1;
  const int32_t m = (int32_t)pos[valid];
  for (int64_t i = gtid(); i < valid; i += gstride()) {
    const uint64_t k = keys[i];
    const uint64_t prev_key = i == 0 ? ~0ull : keys[i - 1];
    const bool head = i == 0 || prev_key != k;
    const uint32_t a = (uint32_t)(k >> bits), b = (uint32_t)(k & mask);
    const int32_t at = (int32_t)pos[i] - (head ? 0 : 1);
    if (head) {
      nlist[at] = (int32_t)b;
      if (rule == ECL_WEIGHTS_HASH) eweight[at] = ecl_edge_weight(seed, a, b, wmax);
      if (rule == ECL_WEIGHTS_SYNTH) eweight[at] = ecl_synth_weight((int32_t)a, (int32_t)b, nodes);
      const int64_t prev_row = i == 0 ? -1 : (int64_t)(prev_key >> bits);
      for (int64_t r = prev_row + 1; r <= (int64_t)a; r++) nindex[r] = at;
    }
    if (rule == ECL_WEIGHTS_GIVEN) atomicMin(reinterpret_cast<unsigned*>(eweight) + at, vals[i]);
    if (i == valid - 1)
      for (int64_t r = (int64_t)a + 1; r <= nodes; r++) nindex[r] = m;
  }
}

// Erdos-Renyi samples, as ecl_gen_er draws them.
__global__ void __launch_bounds__(kPT) k_pairs_er(int64_t samples, uint32_t nodes, uint64_t seed,
                                                  int32_t* __restrict__ u, int32_t* __restrict__ v) {
  for (int64_t i = gtid(); i < samples; i += gstride()) {
    const uint64_t r = ecl_rng(seed, ECL_STREAM_ER, (uint64_t)i);
    u[i] = (int32_t)ecl_below((uint32_t)(r >> 32), nodes);
    v[i] = (int32_t)ecl_below((uint32_t)r, nodes);
  }
}

// RMAT samples, as ecl_gen_rmat draws them: 16 random bits per level.
__global__ void __launch_bounds__(kPT) k_pairs_rmat(int64_t samples, int scale, EclRmatCut cut, uint64_t seed,
                                                    int32_t* __restrict__ u, int32_t* __restrict__ v) {
  for (int64_t i = gtid(); i < samples; i += gstride()) {
    uint32_t a = 0, b = 0;
    uint64_t r = 0;
    for (int lvl = 0; lvl < scale; lvl++) {
      if ((lvl & 3) == 0) r = ecl_rng(seed, ECL_STREAM_RMAT, ((uint64_t)i << 3) | (uint64_t)(lvl >> 2));
      const uint32_t x = (uint32_t)(r >> (16 * (lvl & 3))) & 0xFFFFu;
      const uint32_t q = x < cut.ta ? 0u : x < cut.tab ? 1u : x < cut.tabc ? 2u : 3u;
      a = (a << 1) | (q >> 1);
      b = (b << 1) | (q & 1u);
    }
    u[i] = (int32_t)a;
    v[i] = (int32_t)b;
  }
}

// The 4-neighbour grid in closed form: row offsets from the degree prefix
// sums, neighbours in ascending order (up, left, right, down).
__global__ void __launch_bounds__(kPT) k_gen_grid(int32_t rows, int32_t cols, uint64_t seed, int32_t wmax,
                                                  int32_t* __restrict__ nindex, int32_t* __restrict__ nlist,
                                                  int32_t* __restrict__ eweight) {
  const int64_t n = (int64_t)rows * cols;
  for (int64_t id = gtid(); id < n; id += gstride()) {
    const int64_t r = id / cols, c = id % cols;
    const int64_t vert = (r > 0) + (r < rows - 1);
    // entries of rows 0..r-1, then of columns 0..c-1 of row r
    const int64_t before = (int64_t)cols * (max(r - 1, (int64_t)0) + min(r, (int64_t)rows - 1)) +
                           2 * (int64_t)(cols - 1) * r + c * vert + max(c - 1, (int64_t)0) +
                           min(c, (int64_t)cols - 1);
    nindex[id] = (int32_t)before;
    int64_t k = before;
    int64_t nb[4];
    int d = 0;
    if (r > 0) nb[d++] = id - cols;
    if (c > 0) nb[d++] = id - 1;
    if (c < cols - 1) nb[d++] = id + 1;
    if (r < rows - 1) nb[d++] = id + cols;
    for (int t = 0; t < d; t++, k++) {
      nlist[k] = (int32_t)nb[t];
      eweight[k] = ecl_edge_weight(seed, (uint32_t)id, (uint32_t)nb[t], wmax);
    }
    if (id == n - 1) nindex[n] = (int32_t)(before + d);
  }
}

// Random geometric graph, as ecl_gen_rgg2d builds it: points, then a sort by
// (cell, index) that numbers the vertices in cell order, then the pairs of
// each vertex with later vertices of the 3 x 3 cells around it.
__global__ void __launch_bounds__(kPT) k_rgg_keys(int32_t nodes, uint64_t seed, int64_t cells, uint64_t cell_w,
                                                  uint64_t* __restrict__ keys) {
  for (int64_t i = gtid(); i < nodes; i += gstride()) {
    const uint64_t r = ecl_rng(seed, ECL_STREAM_RGG, (uint64_t)i);
    const uint64_t cx = (r >> 33) / cell_w, cy = (r & 0x7FFFFFFFu) / cell_w;
    keys[i] = ((cy * (uint64_t)cells + cx) << 32) | (uint64_t)i;
  }
}

__global__ void __launch_bounds__(kPT) k_rgg_place(int32_t nodes, const uint64_t* __restrict__ keys,
                                                   uint64_t seed, int64_t ncell, uint32_t* __restrict__ sx,
                                                   uint32_t* __restrict__ sy, int32_t* __restrict__ cell_start) {
  for (int64_t k = gtid(); k < nodes; k += gstride()) {
    const uint64_t key = keys[k];
    const uint64_t r = ecl_rng(seed, ECL_STREAM_RGG, (uint64_t)(uint32_t)key);
    sx[k] = (uint32_t)(r >> 33);
    sy[k] = (uint32_t)(r & 0x7FFFFFFFu);
    const int64_t c = (int64_t)(key >> 32);
    const int64_t prev = k == 0 ? -1 : (int64_t)(keys[k - 1] >> 32);
    for (int64_t cc = prev + 1; cc <= c; cc++) cell_start[cc] = (int32_t)k;
    if (k == nodes - 1)
      for (int64_t cc = c + 1; cc <= ncell; cc++) cell_start[cc] = nodes;
  }
}

// kEmit = false: count[k] = pairs (k, q > k) within the radius.
// kEmit = true: write them at u/v[off[k]...].
template <bool kEmit>
__global__ void __launch_bounds__(kPT) k_rgg_pairs(int32_t nodes, const uint32_t* __restrict__ sx,
                                                   const uint32_t* __restrict__ sy,
                                                   const int32_t* __restrict__ cell_start, int64_t cells,
                                                   uint64_t cell_w, uint64_t r2, uint64_t* __restrict__ count_off,
                                                   int32_t* __restrict__ u, int32_t* __restrict__ v) {
  for (int64_t k = gtid(); k < nodes; k += gstride()) {
    const int64_t cx = sx[k] / cell_w, cy = sy[k] / cell_w;
    uint64_t at = kEmit ? count_off[k] : 0;
    for (int64_t dy = -1; dy <= 1; dy++) {
      const int64_t yy = cy + dy;
      if (yy < 0 || yy >= cells) continue;
      for (int64_t dx = -1; dx <= 1; dx++) {
        const int64_t xx = cx + dx;
        if (xx < 0 || xx >= cells) continue;
        const int64_t cid = yy * cells + xx;
        for (int64_t q = max((int64_t)cell_start[cid], k + 1); q < cell_start[cid + 1]; q++) {
          const int64_t ddx = (int64_t)sx[k] - (int64_t)sx[q];
          const int64_t ddy = (int64_t)sy[k] - (int64_t)sy[q];
          if ((uint64_t)(ddx * ddx) + (uint64_t)(ddy * ddy) < r2) {
            if (kEmit) {
              u[at] = (int32_t)k;
              v[at] = (int32_t)q;
            }
            at++;
          }
        }
      }
    }
    if (!kEmit) count_off[k] = at;
  }
}

// Where build_csr puts its result.
enum class Emit { kAlloc, kInto, kCount };

struct CsrDst {
  Emit mode = Emit::kAlloc;
  int32_t* nindex = nullptr;  // kInto: nodes + 1 entries
  int32_t* nlist = nullptr;   // kInto: cap entries
  int32_t* eweight = nullptr;
  int64_t cap = 0;
  int32_t edges = 0;  // out: CSR entries
};

int alloc_graph(int32_t nodes, int64_t edges, CsrDst& d) {
  PP_TRY(cudaMalloc(&d.nindex, ((size_t)nodes + 1) * 4));
  PP_TRY(cudaMalloc(&d.nlist, (size_t)std::max<int64_t>(edges, 1) * 4));
  PP_TRY(cudaMalloc(&d.eweight, (size_t)std::max<int64_t>(edges, 1) * 4));
  return ECL_OK;
}

void free_dst(CsrDst& d) {
  if (d.mode != Emit::kAlloc) return;
  cudaFree(d.nindex);
  cudaFree(d.nlist);
  cudaFree(d.eweight);
  d.nindex = d.nlist = d.eweight = nullptr;
}

int build_csr(int32_t nodes, int64_t pairs, const int32_t* u, const int32_t* v, const int32_t* w, int rule,
              uint64_t seed, int32_t wmax, cudaStream_t s, CsrDst& dst) {
  if (nodes < 1 || pairs < 0 || (pairs > 0 && (!u || !v))) return ECL_ERR_INVALID_ARG;
  if (rule < ECL_WEIGHTS_GIVEN || rule > ECL_WEIGHTS_SYNTH) return ECL_ERR_INVALID_ARG;
  if (rule == ECL_WEIGHTS_GIVEN && pairs > 0 && !w) return ECL_ERR_INVALID_ARG;
  if (2 * pairs > INT32_MAX) return ECL_ERR_TOO_LARGE;
  const int64_t total = 2 * pairs;
  const int bits = id_bits(nodes);
  const bool given = rule == ECL_WEIGHTS_GIVEN;
  Scratch sc(s);
  uint64_t *keys = nullptr, *keys_alt = nullptr;
  uint32_t *vals = nullptr, *vals_alt = nullptr, *pos = nullptr;
  unsigned long long* counters = nullptr;  // [0] dropped keys, [1] bad-id flag
  PP_CHECK(sc.get(&counters, 2));
  PP_CHECK(sc.get(&keys, total));
  PP_CHECK(sc.get(&keys_alt, total));
  if (given) {
    PP_CHECK(sc.get(&vals, total));
    PP_CHECK(sc.get(&vals_alt, total));
  }
  PP_TRY(cudaMemsetAsync(counters, 0, 2 * sizeof(unsigned long long), s));
  int64_t valid = 0;
  uint64_t* spare = keys_alt;  // the sort's other buffer, free after the sort
  if (total > 0) {
    k_pair_keys<<<blocks_for(pairs), kPT, 0, s>>>(pairs, u, v, w, (uint32_t)nodes, bits,
                                                   reinterpret_cast<ulonglong2*>(keys),
                                                   reinterpret_cast<uint2*>(vals), counters,
                                                   reinterpret_cast<unsigned*>(counters + 1));
    PP_TRY(cudaGetLastError());
    cub::DoubleBuffer<uint64_t> kb(keys, keys_alt);
    cub::DoubleBuffer<uint32_t> vb(vals, vals_alt);
    size_t tmp_bytes = 0;
    char* tmp = nullptr;
    if (given) {
      PP_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kb, vb, (int)total, 0, 2 * bits, s));
      PP_CHECK(sc.get(&tmp, tmp_bytes));
      PP_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kb, vb, (int)total, 0, 2 * bits, s));
      vals = vb.Current();
    } else {
      PP_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, kb, (int)total, 0, 2 * bits, s));
      PP_CHECK(sc.get(&tmp, tmp_bytes));
      PP_TRY(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, kb, (int)total, 0, 2 * bits, s));
    }
    keys = kb.Current();
    spare = kb.Alternate();
    unsigned long long host[2];
    PP_TRY(cudaMemcpyAsync(host, counters, sizeof(host), cudaMemcpyDeviceToHost, s));
    PP_TRY(cudaStreamSynchronize(s));
    if (host[1]) return ECL_ERR_FORMAT;
    valid = total - (int64_t)host[0];
  }
  int32_t m = 0;
  if (valid > 0) {
    // run-head flags in the spare sort buffer ((valid + 1) * 4 <= total * 8 bytes)
    uint32_t* flags = reinterpret_cast<uint32_t*>(spare);
    PP_CHECK(sc.get(&pos, (size_t)valid + 1));
    k_run_heads<<<blocks_for(valid + 1), kPT, 0, s>>>(valid, keys, flags);
    PP_TRY(cudaGetLastError());
    size_t tmp_bytes = 0;
    char* tmp = nullptr;
    PP_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flags, pos, (int)(valid + 1), s));
    PP_CHECK(sc.get(&tmp, tmp_bytes));
    PP_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flags, pos, (int)(valid + 1), s));
    uint32_t hm = 0;
    PP_TRY(cudaMemcpyAsync(&hm, pos + valid, sizeof(hm), cudaMemcpyDeviceToHost, s));
    PP_TRY(cudaStreamSynchronize(s));
    m = (int32_t)hm;
  }
  dst.edges = m;
  if (dst.mode == Emit::kCount) return ECL_OK;
  if (dst.mode == Emit::kAlloc) {
    const int st = alloc_graph(nodes, m, dst);
    if (st) {
      free_dst(dst);
      return st;
    }
  } else if (m > dst.cap || !dst.nindex || (m > 0 && (!dst.nlist || !dst.eweight))) {
    return ECL_ERR_OVERFLOW;
  }
  if (valid == 0) {
    PP_TRY(cudaMemsetAsync(dst.nindex, 0, ((size_t)nodes + 1) * 4, s));
  } else {
    if (given) PP_TRY(cudaMemsetAsync(dst.eweight, 0xFF, (size_t)m * 4, s));
    k_emit_csr<<<blocks_for(valid), kPT, 0, s>>>(valid, keys, vals, pos, bits, nodes, rule, seed, wmax,
                                                  dst.nindex, dst.nlist, dst.eweight);
    PP_TRY(cudaGetLastError());
  }
  PP_TRY(cudaStreamSynchronize(s));
  return ECL_OK;
}

// ------------------------------------------------------------ generators

int gen_grid(int32_t rows, int32_t cols, uint64_t seed, int32_t wmax, cudaStream_t s, CsrDst& dst) {
  if (rows < 1 || cols < 1 || wmax < 1) return ECL_ERR_INVALID_ARG;
  const int64_t n64 = (int64_t)rows * cols;
  const int64_t m64 = 2 * ((int64_t)rows * (cols - 1) + (int64_t)(rows - 1) * cols);
  if (n64 > INT32_MAX || m64 > INT32_MAX) return ECL_ERR_TOO_LARGE;
  dst.edges = (int32_t)m64;
  if (dst.mode == Emit::kCount) return ECL_OK;
  if (dst.mode == Emit::kAlloc) {
    const int st = alloc_graph((int32_t)n64, m64, dst);
    if (st) {
      free_dst(dst);
      return st;
    }
  } else if (m64 > dst.cap) {
    return ECL_ERR_OVERFLOW;
  }
  k_gen_grid<<<blocks_for(n64), kPT, 0, s>>>(rows, cols, seed, wmax, dst.nindex, dst.nlist, dst.eweight);
  PP_TRY(cudaGetLastError());
  PP_TRY(cudaStreamSynchronize(s));
  return ECL_OK;
}

int gen_er(int32_t nodes, double avg_degree, uint64_t seed, int32_t wmax, cudaStream_t s, CsrDst& dst) {
  if (nodes < 1 || avg_degree < 0 || wmax < 1) return ECL_ERR_INVALID_ARG;
  const int64_t samples = (int64_t)std::llround((double)nodes * avg_degree / 2.0);
  if (2 * samples > INT32_MAX) return ECL_ERR_TOO_LARGE;
  Scratch sc(s);
  int32_t *u = nullptr, *v = nullptr;
  PP_CHECK(sc.get(&u, samples));
  PP_CHECK(sc.get(&v, samples));
  if (samples > 0) {
    k_pairs_er<<<blocks_for(samples), kPT, 0, s>>>(samples, (uint32_t)nodes, seed, u, v);
    PP_TRY(cudaGetLastError());
  }
  return build_csr(nodes, samples, u, v, nullptr, ECL_WEIGHTS_HASH, seed, wmax, s, dst);
}

int gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed, int32_t wmax,
             cudaStream_t s, CsrDst& dst) {
  if (scale < 1 || scale > 30 || edge_factor < 0 || wmax < 1) return ECL_ERR_INVALID_ARG;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0 + 1e-12) return ECL_ERR_INVALID_ARG;
  const int64_t samples = (int64_t)edge_factor << scale;
  if (2 * samples > INT32_MAX) return ECL_ERR_TOO_LARGE;
  Scratch sc(s);
  int32_t *u = nullptr, *v = nullptr;
  PP_CHECK(sc.get(&u, samples));
  PP_CHECK(sc.get(&v, samples));
  if (samples > 0) {
    k_pairs_rmat<<<blocks_for(samples), kPT, 0, s>>>(samples, scale, ecl_rmat_cut(a, b, c), seed, u, v);
    PP_TRY(cudaGetLastError());
  }
  return build_csr(1 << scale, samples, u, v, nullptr, ECL_WEIGHTS_HASH, seed, wmax, s, dst);
}

int gen_rgg2d(int32_t nodes, double avg_degree, uint64_t seed, int32_t wmax, cudaStream_t s, CsrDst& dst) {
  if (nodes < 1 || avg_degree < 0 || wmax < 1) return ECL_ERR_INVALID_ARG;
  const EclRggGrid g = ecl_rgg_grid(nodes, avg_degree);
  const int64_t ncell = g.cells * g.cells;
  Scratch sc(s);
  uint64_t *keys = nullptr, *keys_alt = nullptr, *cnt = nullptr;
  uint32_t *sx = nullptr, *sy = nullptr;
  int32_t* cell_start = nullptr;
  PP_CHECK(sc.get(&keys, nodes));
  PP_CHECK(sc.get(&keys_alt, nodes));
  PP_CHECK(sc.get(&sx, nodes));
  PP_CHECK(sc.get(&sy, nodes));
  PP_CHECK(sc.get(&cell_start, (size_t)ncell + 1));
  PP_CHECK(sc.get(&cnt, (size_t)nodes + 1));
  k_rgg_keys<<<blocks_for(nodes), kPT, 0, s>>>(nodes, seed, g.cells, g.cell_w, keys);
  PP_TRY(cudaGetLastError());
  const int end_bit = 32 + id_bits(ncell);
  cub::DoubleBuffer<uint64_t> kb(keys, keys_alt);
  size_t tmp_bytes = 0;
  char* tmp = nullptr;
  PP_TRY(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, kb, nodes, 0, end_bit, s));
  PP_CHECK(sc.get(&tmp, tmp_bytes));
  PP_TRY(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, kb, nodes, 0, end_bit, s));
  k_rgg_place<<<blocks_for(nodes), kPT, 0, s>>>(nodes, kb.Current(), seed, ncell, sx, sy, cell_start);
  PP_TRY(cudaGetLastError());
  k_rgg_pairs<false><<<blocks_for(nodes), kPT, 0, s>>>(nodes, sx, sy, cell_start, g.cells, g.cell_w, g.r2, cnt,
                                                       nullptr, nullptr);
  PP_TRY(cudaGetLastError());
  PP_TRY(cudaMemsetAsync(cnt + nodes, 0, sizeof(uint64_t), s));
  uint64_t* off = nullptr;
  PP_CHECK(sc.get(&off, (size_t)nodes + 1));
  tmp_bytes = 0;
  PP_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, off, nodes + 1, s));
  PP_CHECK(sc.get(&tmp, tmp_bytes));
  PP_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, off, nodes + 1, s));
  uint64_t pairs = 0;
  PP_TRY(cudaMemcpyAsync(&pairs, off + nodes, sizeof(pairs), cudaMemcpyDeviceToHost, s));
  PP_TRY(cudaStreamSynchronize(s));
  if (2 * pairs > (uint64_t)INT32_MAX) return ECL_ERR_TOO_LARGE;
  int32_t *u = nullptr, *v = nullptr;
  PP_CHECK(sc.get(&u, pairs));
  PP_CHECK(sc.get(&v, pairs));
  k_rgg_pairs<true><<<blocks_for(nodes), kPT, 0, s>>>(nodes, sx, sy, cell_start, g.cells, g.cell_w, g.r2, off,
                                                      u, v);
  PP_TRY(cudaGetLastError());
  return build_csr(nodes, (int64_t)pairs, u, v, nullptr, ECL_WEIGHTS_HASH, seed, wmax, s, dst);
}

int gen_batch_one(const EclBatchPick& p, int32_t wmax, cudaStream_t s, CsrDst& dst) {
  switch (p.family) {
    case 0:
      return gen_grid(p.rows_or_scale, std::max<int32_t>(1, p.nodes / p.rows_or_scale), p.seed, wmax, s, dst);
    case 1:
      return gen_er(p.nodes, kBatchErDegree, p.seed, wmax, s, dst);
    case 2:
      return gen_rmat(p.rows_or_scale, kBatchRmatEdgeFactor, kBatchRmatA, kBatchRmatB, kBatchRmatC, p.seed, wmax, s,
                      dst);
    default:
      return gen_rgg2d(p.nodes, kBatchRggDegree, p.seed, wmax, s, dst);
  }
}

// Vertex count of a batch graph as its generator rounds it.
int32_t batch_nodes(const EclBatchPick& p) {
  if (p.family == 0) return p.rows_or_scale * std::max<int32_t>(1, p.nodes / p.rows_or_scale);
  if (p.family == 2) return 1 << p.rows_or_scale;
  return p.nodes;
}

int finish(int st, int32_t nodes, CsrDst& d, ecl_graph* out) {
  if (st) {
    free_dst(d);
    return st;
  }
  out->nodes = nodes;
  out->edges = d.edges;
  out->nindex = d.nindex;
  out->nlist = d.nlist;
  out->eweight = d.eweight;
  return ECL_OK;
}

int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

}  // namespace

extern "C" int ecl_csr_from_pairs_device(int32_t nodes, int64_t pairs, const int32_t* d_u, const int32_t* d_v,
                                         const int32_t* d_w, int32_t weight_rule, uint64_t seed, int32_t wmax,
                                         void* stream, ecl_graph* out) {
  if (!out) return ECL_ERR_INVALID_ARG;
  if (weight_rule == ECL_WEIGHTS_HASH && wmax < 1) return ECL_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TrimOnExit trim{s};
  CsrDst d;
  return finish(build_csr(nodes, pairs, d_u, d_v, d_w, weight_rule, seed, wmax, s, d), nodes, d, out);
}

extern "C" int ecl_gen_grid_device(int32_t rows, int32_t cols, uint64_t seed, int32_t wmax, void* stream,
                                   ecl_graph* out) {
  if (!out) return ECL_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TrimOnExit trim{s};
  CsrDst d;
  const int st = gen_grid(rows, cols, seed, wmax, s, d);
  return finish(st, st ? 0 : rows * cols, d, out);
}

extern "C" int ecl_gen_er_device(int32_t nodes, double avg_degree, uint64_t seed, int32_t wmax, void* stream,
                                 ecl_graph* out) {
  if (!out) return ECL_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TrimOnExit trim{s};
  CsrDst d;
  return finish(gen_er(nodes, avg_degree, seed, wmax, s, d), nodes, d, out);
}

extern "C" int ecl_gen_rmat_device(int32_t scale, int32_t edge_factor, double a, double b, double c,
                                   uint64_t seed, int32_t wmax, void* stream, ecl_graph* out) {
  if (!out) return ECL_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TrimOnExit trim{s};
  CsrDst d;
  const int st = gen_rmat(scale, edge_factor, a, b, c, seed, wmax, s, d);
  return finish(st, st ? 0 : 1 << scale, d, out);
}

extern "C" int ecl_gen_rgg2d_device(int32_t nodes, double avg_degree, uint64_t seed, int32_t wmax, void* stream,
                                    ecl_graph* out) {
  if (!out) return ECL_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TrimOnExit trim{s};
  CsrDst d;
  return finish(gen_rgg2d(nodes, avg_degree, seed, wmax, s, d), nodes, d, out);
}

extern "C" int ecl_gen_batch_graph_device(int32_t index, uint64_t seed0, int32_t nmin, int32_t nmax, int32_t wmax,
                                          void* stream, ecl_graph* out, int32_t* family) {
  if (!out || nmin < 1 || nmax < nmin || index < 0) return ECL_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TrimOnExit trim{s};
  const EclBatchPick p = ecl_batch_pick(index, seed0, nmin, nmax);
  if (family) *family = p.family;
  CsrDst d;
  const int st = gen_batch_one(p, wmax, s, d);
  return finish(st, st ? 0 : batch_nodes(p), d, out);
}

extern "C" void ecl_free_device_graph(ecl_graph* g) {
  if (!g) return;
  cudaFree(g->nindex);
  cudaFree(g->nlist);
  cudaFree(g->eweight);
  memset(g, 0, sizeof(*g));
}

extern "C" int ecl_graph_to_host(const ecl_graph* d_graph, ecl_graph* out) {
  if (!d_graph || !out || d_graph->nodes < 1 || d_graph->edges < 0 || !d_graph->nindex) return ECL_ERR_INVALID_ARG;
  if (d_graph->edges > 0 && !d_graph->nlist) return ECL_ERR_INVALID_ARG;
  const size_t nb = ((size_t)d_graph->nodes + 1) * 4, eb = (size_t)std::max(d_graph->edges, 1) * 4;
  ecl_graph h{};
  h.nodes = d_graph->nodes;
  h.edges = d_graph->edges;
  h.nindex = static_cast<int32_t*>(malloc(nb));
  h.nlist = static_cast<int32_t*>(malloc(eb));
  h.eweight = d_graph->eweight ? static_cast<int32_t*>(malloc(eb)) : nullptr;
  if (!h.nindex || !h.nlist || (d_graph->eweight && !h.eweight)) {
    ecl_free_graph(&h);
    return ECL_ERR_ALLOC;
  }
  const size_t mb = (size_t)d_graph->edges * 4;
  cudaError_t e = cudaMemcpy(h.nindex, d_graph->nindex, nb, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && mb) e = cudaMemcpy(h.nlist, d_graph->nlist, mb, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && mb && h.eweight) e = cudaMemcpy(h.eweight, d_graph->eweight, mb, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    ecl_free_graph(&h);
    return cuda_status(e);
  }
  *out = h;
  return ECL_OK;
}

extern "C" int ecl_gen_batch_device(int32_t count, uint64_t seed0, int32_t nmin, int32_t nmax, int32_t wmax,
                                    int32_t align, void* stream, ecl_batch* out, int32_t* family) {
  if (!out || count < 1 || nmin < 1 || nmax < nmin || wmax < 1 || align < 1) return ECL_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  TrimOnExit trim{s};
  memset(out, 0, sizeof(*out));
  ecl_batch b{};
  b.num_graphs = count;
  int32_t* nodes = static_cast<int32_t*>(malloc((size_t)count * 4));
  int32_t* edges = static_cast<int32_t*>(malloc((size_t)count * 4));
  int64_t* noff = static_cast<int64_t*>(malloc((size_t)count * 8));
  int64_t* eoff = static_cast<int64_t*>(malloc((size_t)count * 8));
  b.nodes = nodes;
  b.edges = edges;
  b.nindex_off = noff;
  b.edge_off = eoff;
  auto fail = [&](int st) {
    ecl_free_device_batch(&b);
    return st;
  };
  if (!nodes || !edges || !noff || !eoff) return fail(ECL_ERR_ALLOC);
  // Pass 1: every graph's size (the dedup decides the entry count), then the
  // packed layout; pass 2 draws each graph again straight into its segment,
  // so the peak is the batch plus one graph's scratch.
  std::vector<EclBatchPick> picks((size_t)count);
  int64_t no = 0, eo = 0;
  for (int32_t g = 0; g < count; g++) {
    picks[g] = ecl_batch_pick(g, seed0, nmin, nmax);
    if (family) family[g] = picks[g].family;
    CsrDst d;
    d.mode = Emit::kCount;
    const int st = gen_batch_one(picks[g], wmax, s, d);
    if (st) return fail(st);
    nodes[g] = batch_nodes(picks[g]);
    edges[g] = d.edges;
    noff[g] = no;
    eoff[g] = eo;
    no += round_up((int64_t)nodes[g] + 1, align);
    eo += round_up(std::max<int32_t>(edges[g], 1), align);
  }
  cudaError_t e = cudaMalloc(&b.nindex, (size_t)no * 4);
  if (e == cudaSuccess) e = cudaMalloc(&b.nlist, (size_t)eo * 4);
  if (e == cudaSuccess) e = cudaMalloc(&b.eweight, (size_t)eo * 4);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.nindex, 0, (size_t)no * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.nlist, 0, (size_t)eo * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.eweight, 0, (size_t)eo * 4, s);
  if (e != cudaSuccess) return fail(cuda_status(e));
  for (int32_t g = 0; g < count; g++) {
    CsrDst d;
    d.mode = Emit::kInto;
    d.nindex = b.nindex + noff[g];
    d.nlist = b.nlist + eoff[g];
    d.eweight = b.eweight + eoff[g];
    d.cap = edges[g];
    const int st = gen_batch_one(picks[g], wmax, s, d);
    if (st) return fail(st);
    if (d.edges != edges[g]) return fail(ECL_ERR_OVERFLOW);
  }
  *out = b;
  return ECL_OK;
}

extern "C" void ecl_free_device_batch(ecl_batch* b) {
  if (!b) return;
  free(const_cast<int32_t*>(b->nodes));
  free(const_cast<int32_t*>(b->edges));
  free(const_cast<int64_t*>(b->nindex_off));
  free(const_cast<int64_t*>(b->edge_off));
  cudaFree(b->nindex);
  cudaFree(b->nlist);
  cudaFree(b->eweight);
  memset(b, 0, sizeof(*b));
}
