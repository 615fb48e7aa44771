// B200 (sm_100a) engine of the ECL-MST minimum spanning forest: host side
// of the single-graph solve (context, launch sequence, C ABI). The kernels
// and their mapping to the reference's gpuMST (ECL-MST/ECL_MST.cu:265-362)
// are in mst_device.cuh.
#include <cuda_runtime.h>
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include "ecl_mst.h"
#include "internal.h"
#include "mst_device.cuh"
#include "batch_device.cuh"
#include <functional>
#include <vector>

// Learned threshold/split (learned.cu). ecl_learned_sample uploads changed
// weights and sorts the weight sample; ecl_learned_apply computes the
// features from it and from k_prep's degree statistics and runs the trained
// MLP, writing DevState::threshold, filtered, quantile and split.
int ecl_learned_sample(ecl_mst_ctx* c, const ecl_graph* d_graph, cudaStream_t s);
int ecl_learned_apply(ecl_mst_ctx* c, const ecl_graph* d_graph, cudaStream_t s, void* st);
int ecl_learned_upload(ecl_mst_ctx* c, cudaStream_t s);
unsigned ecl_learned_weights_version();

using namespace ecl;

namespace {
constexpr int kDefaultSplit = 8;
constexpr unsigned kDefaultSmallTail = 4096;
constexpr int kDefaultMinTiles = 1;  // round CTAs kept: one per tile of the round's worklist
constexpr int64_t kWlSlack = 1 << 19;  // worklist slots beyond `edges` (scan chunk tails)
constexpr int kLearnedMinEdges = 1 << 20;
}  // namespace

// =================================================================== host
struct ecl_mst_ctx {
  int device = 0;
  int sm_count = 0;
  int64_t max_nodes = 0, max_edges = 0;
  cudaStream_t stream = nullptr;
  // the learned schedule's sample sort and MLP run on `side`, beside k_prep
  // and the fill scan; the scan variants its split does not select run on
  // `side` and `side2`, beside the selected one
  cudaStream_t side = nullptr, side2 = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr, prep_done = nullptr;
  cudaEvent_t scan_fork = nullptr, scan_join[2] = {nullptr, nullptr};
  // the last solve's key, and the captured solve (CUDA graph) with its key
  std::vector<long long> last_key, exec_key;
  cudaGraphExec_t exec = nullptr;
  // [minv0 | minv1 | parent] in one allocation, laid out per solve for the
  // graph's vertex count (minv0 = slots, minv1 = minv0 + n, parent after
  // minv1), so one L2 access-policy window covers exactly the 20n bytes used
  void* slots = nullptr;
  // L2 persistence (ECL_FLAG_L2_PERSIST): the device's persisting set-aside
  // and window limits, and the set-aside this context raised (restored at
  // destroy)
  size_t l2_persist_max = 0, l2_window_max = 0;
  size_t l2_limit_prev = 0;
  bool l2_limit_set = false;
  int4* wl[2] = {nullptr, nullptr};
  unsigned wl_cap = 0;
  // false: each list holds max_edges / 2 entries plus slack (every symmetric
  // input); true: max_edges plus slack (any input). A solve whose scan
  // overflows the half-size lists is repeated after they are grown.
  bool wl_full = false;
  // the last device solve, kept so ecl_mst_ctx_sync can repeat it after a
  // worklist overflow
  bool pending = false;
  ecl_graph pend_graph = {};
  unsigned char* pend_out = nullptr;
  mst_opts pend_opts = {};
  cudaStream_t pend_stream = nullptr;
  bool resolved = false;  // the last ecl_mst_ctx_sync repeated the solve
  // pipelined host-buffer solves (ecl_mst_ctx_run_host_async): two device
  // buffer sets used in turn (set 0 is the one run_host uses), a copy-in and a
  // copy-out stream, the events that order them, a sticky device error word
  // and the calls since the last ecl_mst_ctx_wait (repeated after a
  // worklist overflow)
  struct HostSet {
    int* nindex = nullptr;
    int* nlist = nullptr;
    int* eweight = nullptr;
    unsigned char* inMST = nullptr;
    cudaEvent_t in_done = nullptr, solved = nullptr, out_done = nullptr;
    bool used = false;
  };
  HostSet hs[2];
  cudaStream_t cin = nullptr, cout = nullptr;
  unsigned async_seq = 0;
  unsigned* sticky = nullptr;
  struct AsyncCall {
    ecl_graph g;
    uint8_t* out;
    mst_opts opts;
  };
  std::vector<AsyncCall> async_calls;
  int* slist = nullptr;    // ECL_FLAG_NO_TUPLES: vertex of every CSR entry (allocated on first use)
  int vertex_grid = 0;     // ECL_FLAG_NO_EDGE_BASED: cooperative grid of the vertex-centric rounds
  int* first_v = nullptr;  // tile -> vertex table of the edge-balanced scans
  int first_v_cap = 0;
  DevState* st = nullptr;
  DevState* st_host = nullptr;  // pinned
  int round_grid = 0;
  // device CSR + output for host-buffer runs (allocated on first use)
  int* d_nindex = nullptr;
  int* d_nlist = nullptr;
  int* d_eweight = nullptr;
  unsigned char* d_inMST = nullptr;
  // timed solves: start, light scan end, light rounds end, heavy scan end, end,
  // prep end, flatten end
  cudaEvent_t ev[7] = {};
  // learned schedule: MLP parameters (and the load they came from), the 16
  // features, degree accumulators, the sorted 4096-entry weight sample
  float* ml_params = nullptr;
  unsigned ml_version = ~0u;
  float* ml_feat = nullptr;  // the features of the last learned solve
  bool ml_features_set = false;
  void* ml_acc = nullptr;
  int* ml_sample = nullptr;
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

// The solve's slot arrays inside ctx->slots, packed for n vertices.
struct Slots {
  u64* minv0;
  u64* minv1;
  int* parent;
  size_t bytes;  // 20n
};
Slots slots_for(void* base, int n) {
  Slots sl;
  sl.minv0 = (u64*)base;
  sl.minv1 = sl.minv0 + n;
  sl.parent = (int*)(sl.minv1 + n);
  sl.bytes = (size_t)n * (2 * sizeof(u64) + sizeof(int));
  return sl;
}

// Launch `kernel` with optional launch attributes: cooperative (grid-wide
// barriers) and an L2 access-policy window. Without either it is a plain
// launch.
template <typename... KArgs, typename... Args>
int launch_ex(void (*kernel)(KArgs...), int grid, int threads, size_t smem, cudaStream_t s, bool coop,
              const cudaAccessPolicyWindow* win, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  unsigned na = 0;
  if (coop) {
    at[na].id = cudaLaunchAttributeCooperative;
    at[na].val.cooperative = 1;
    na++;
  }
  if (win) {
    at[na].id = cudaLaunchAttributeAccessPolicyWindow;
    at[na].val.accessPolicyWindow = *win;
    na++;
  }
  cfg.attrs = na ? at : nullptr;
  cfg.numAttrs = na;
  return cuda_status(cudaLaunchKernelEx(&cfg, kernel, args...));
}

int prepare_scan_kernels();

// Entries of the tile->vertex table buffer for up to `edges` CSR entries: the
// table (tiles + 1) and the fill scan's chunk maxima.
int64_t first_v_entries(int64_t edges) {
  const int64_t tiles = edges / kGran + 1;
  return tiles + 1 + tiles / kFillChunk + 1;
}

// k_prep, then the fill scan that completes the tile->vertex table
// (first_v: pa.tiles + 1 entries, then room for the chunk maxima).
// k_prep, then the max scan of the tile->vertex table. `after_prep`, when
// given, is enqueued between the two (the learned schedule forks its MLP off
// there, once k_prep's degree statistics are complete).
int enqueue_prep(const PrepArgs& pa, int sm_count, cudaStream_t s, const cudaAccessPolicyWindow* win = nullptr,
                 const std::function<int()>& after_prep = nullptr) {
  ECL_CUDA_TRY(cudaMemsetAsync(pa.first_v, 0, sizeof(int) * (size_t)pa.tiles, s));
  const int prep_grid = (int)std::min<int64_t>((pa.nodes + kThreads - 1) / kThreads, (int64_t)sm_count * 16);
  if (win) {
    int st = launch_ex(k_prep, std::max(prep_grid, 1), kThreads, 0, s, false, win, pa);
    if (st) return st;
  } else {
    k_prep<<<std::max(prep_grid, 1), kThreads, 0, s>>>(pa);
  }
  ECL_CUDA_TRY(cudaGetLastError());
  if (after_prep) {
    const int st = after_prep();
    if (st) return st;
  }
  const int chunks = (pa.tiles + kFillChunk - 1) / kFillChunk;
  int* chunk_max = pa.first_v + pa.tiles + 1;
  k_fill_chunks<<<chunks, 1024, 0, s>>>(pa.first_v, pa.tiles, chunk_max);
  k_fill_carry<<<chunks, 1024, 0, s>>>(pa.first_v, pa.tiles, chunk_max, pa.nodes);
  return cuda_status(cudaGetLastError());
}

// Round-kernel ablation bits from the option flags.
unsigned round_ablation(int flags) {
  return ((flags & ECL_FLAG_NO_GUARDS) ? kAblNoGuards : 0u) | ((flags & ECL_FLAG_NO_WARP_COOP) ? kAblNoCoop : 0u) |
         ((flags & ECL_FLAG_DEDUP) ? kDedup : 0u) | ((flags & ECL_FLAG_NO_FIND_CACHE) ? kAblNoFindCache : 0u) |
         ((flags & ECL_FLAG_NO_IMPLICIT_COMPRESSION) ? kAblNoIPC : 0u) |
         ((flags & ECL_FLAG_NO_TUPLES) ? kAblNoTuples : 0u) | ((flags & ECL_FLAG_NO_DATA_DRIVEN) ? kAblNoDD : 0u);
}

// The reference's later ablation steps, which only the single-graph engine runs.
constexpr int kDeoptFlags = ECL_FLAG_NO_IMPLICIT_COMPRESSION | ECL_FLAG_NO_TUPLES | ECL_FLAG_NO_DATA_DRIVEN |
                            ECL_FLAG_NO_EDGE_BASED;

}  // namespace

namespace {

// A phase's worklist holds one entry per one-direction CSR entry
// (nlist[j] > v) at most. That is edges / 2 for a symmetric input (the size
// the reference gives it, ECL_MST.cu:279) and up to `edges` otherwise; the
// lists start at the symmetric size and grow to the full one when a solve
// overflows them. Both carry slack for the unused tails of the scan warps'
// slot chunks.
int alloc_worklists(ecl_mst_ctx* c, bool full) {
  cudaFree(c->wl[0]);
  cudaFree(c->wl[1]);
  c->wl[0] = c->wl[1] = nullptr;
  const int64_t keep = full ? c->max_edges : c->max_edges / 2;
  c->wl_cap = (unsigned)std::max<int64_t>(keep + std::min<int64_t>(c->max_edges, kWlSlack), 1);
  c->wl_full = full;
  for (int i = 0; i < 2; i++)
    ECL_CUDA_TRY(cudaMalloc(&c->wl[i], (size_t)c->wl_cap * sizeof(int4)));
  return ECL_OK;
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
  if ((st = cuda_status(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking)))) return fail(st);
  if ((st = cuda_status(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming)))) return fail(st);
  if ((st = cuda_status(cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming)))) return fail(st);
  if ((st = cuda_status(cudaEventCreateWithFlags(&c->prep_done, cudaEventDisableTiming)))) return fail(st);
  if ((st = cuda_status(cudaStreamCreateWithFlags(&c->side2, cudaStreamNonBlocking)))) return fail(st);
  if ((st = cuda_status(cudaEventCreateWithFlags(&c->scan_fork, cudaEventDisableTiming)))) return fail(st);
  for (auto& e : c->scan_join)
    if ((st = cuda_status(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)))) return fail(st);
  const size_t slot_bytes = (size_t)max_nodes * (2 * sizeof(u64) + sizeof(int));
  if ((st = cuda_status(cudaMalloc(&c->slots, slot_bytes)))) return fail(st);
  c->l2_persist_max = prop.persistingL2CacheMaxSize > 0 ? (size_t)prop.persistingL2CacheMaxSize : 0;
  c->l2_window_max = prop.accessPolicyMaxWindowSize > 0 ? (size_t)prop.accessPolicyMaxWindowSize : 0;
  if ((st = alloc_worklists(c, false))) return fail(st);
  c->first_v_cap = (int)first_v_entries(max_edges);
  if ((st = cuda_status(cudaMalloc(&c->first_v, (size_t)c->first_v_cap * sizeof(int))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->st, sizeof(DevState))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->ml_params, ECL_MLP_PARAMS * sizeof(float))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->ml_feat, ECL_MLP_INPUTS * sizeof(float))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->ml_acc, sizeof(FeatAcc))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->ml_sample, 4096 * sizeof(int))))) return fail(st);
  if ((st = cuda_status(cudaHostAlloc(&c->st_host, sizeof(DevState), cudaHostAllocDefault))))
    return fail(st);
  for (auto& e : c->ev)
    if ((st = cuda_status(cudaEventCreate(&e)))) return fail(st);
  // every CTA of a round pass writes one segment of the round's output list
  c->round_grid = std::min(coop_grid((const void*)k_rounds, kRoundThreads, c->sm_count), kMaxRoundCtas);
  c->vertex_grid = coop_grid((const void*)k_rounds_vertex, kRoundThreads, c->sm_count);
  if ((st = prepare_scan_kernels())) return fail(st);
  if (c->round_grid <= 0 || c->vertex_grid <= 0) return fail(ECL_ERR_CUDA);
  *out = c;
  return ECL_OK;
}

extern "C" void ecl_mst_ctx_destroy(ecl_mst_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->l2_limit_set) {  // hand the persisting set-aside back as it was
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, c->l2_limit_prev);
  }
  cudaFree(c->slots);
  cudaFree(c->wl[0]);
  cudaFree(c->wl[1]);
  cudaFree(c->first_v);
  cudaFree(c->slist);
  cudaFree(c->ml_params);
  cudaFree(c->ml_feat);
  cudaFree(c->ml_acc);
  cudaFree(c->ml_sample);
  cudaFree(c->st);
  cudaFreeHost(c->st_host);
  cudaFree(c->d_nindex);
  cudaFree(c->d_nlist);
  cudaFree(c->d_eweight);
  cudaFree(c->d_inMST);
  if (c->cin) cudaStreamSynchronize(c->cin);
  if (c->cout) cudaStreamSynchronize(c->cout);
  cudaFree(c->hs[1].nindex);
  cudaFree(c->hs[1].nlist);
  cudaFree(c->hs[1].eweight);
  cudaFree(c->hs[1].inMST);
  cudaFree(c->sticky);
  for (auto& h : c->hs)
    for (cudaEvent_t e : {h.in_done, h.solved, h.out_done})
      if (e) cudaEventDestroy(e);
  if (c->cin) cudaStreamDestroy(c->cin);
  if (c->cout) cudaStreamDestroy(c->cout);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->side) cudaStreamSynchronize(c->side);
  if (c->side2) cudaStreamSynchronize(c->side2);
  if (c->exec) cudaGraphExecDestroy(c->exec);
  if (c->fork) cudaEventDestroy(c->fork);
  if (c->join) cudaEventDestroy(c->join);
  if (c->prep_done) cudaEventDestroy(c->prep_done);
  if (c->scan_fork) cudaEventDestroy(c->scan_fork);
  for (cudaEvent_t e : c->scan_join)
    if (e) cudaEventDestroy(e);
  if (c->side2) cudaStreamDestroy(c->side2);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" void* ecl_mst_ctx_stream(ecl_mst_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" int ecl_mst_ctx_learned_features(ecl_mst_ctx* c, float* out16) {
  if (!c || !out16) return ECL_ERR_INVALID_ARG;
  if (!c->ml_features_set) return ECL_ERR_UNSUPPORTED;
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  ECL_CUDA_TRY(cudaStreamSynchronize(c->side));
  ECL_CUDA_TRY(cudaMemcpy(out16, c->ml_feat, ECL_MLP_INPUTS * sizeof(float), cudaMemcpyDeviceToHost));
  return ECL_OK;
}

extern "C" int ecl_mst_ctx_l2_reset(ecl_mst_ctx* c) {
  if (!c) return ECL_ERR_INVALID_ARG;
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  ECL_CUDA_TRY(cudaCtxResetPersistingL2Cache());
  return ECL_OK;
}

namespace {
int run_device_once(ecl_mst_ctx* c, const ecl_graph* g, uint8_t* d_inMST, const mst_opts* opts, void* stream,
                    ecl_mst_stats* stats);
int grow_worklists(ecl_mst_ctx* c);
}  // namespace

extern "C" int ecl_mst_ctx_sync(ecl_mst_ctx* c) {
  if (!c) return ECL_ERR_INVALID_ARG;
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  c->resolved = false;
  cudaStream_t s = c->pending ? c->pend_stream : c->stream;
  ECL_CUDA_TRY(cudaStreamSynchronize(s));
  if (s != c->stream) ECL_CUDA_TRY(cudaStreamSynchronize(c->stream));
  unsigned err = 0;
  ECL_CUDA_TRY(cudaMemcpy(&err, &c->st->error, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if ((err & kErrOverflow) && c->pending && !c->wl_full) {
    // the input had more one-direction entries than half its CSR entries:
    // solve it again with worklists that hold every entry
    c->pending = false;
    int st = grow_worklists(c);
    if (st) return st;
    if ((st = run_device_once(c, &c->pend_graph, c->pend_out, &c->pend_opts, c->pend_stream, nullptr))) return st;
    c->resolved = true;
    ECL_CUDA_TRY(cudaStreamSynchronize(c->pend_stream));
    ECL_CUDA_TRY(cudaMemcpy(&err, &c->st->error, sizeof(unsigned), cudaMemcpyDeviceToHost));
  }
  c->pending = false;
  return device_error_status(err);
}

namespace {

int launch_coop(const void* fn, int grid, int threads, void* arg, cudaStream_t s) {
  void* args[] = {arg};
  return cuda_status(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(threads), args, 0, s));
}

// Opt the scan variants into their dynamic shared memory (once per device).
int prepare_scan_kernels() {
  ECL_CUDA_TRY(cudaFuncSetAttribute(k_scan<kLight, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scan_smem_bytes<4>()));
  ECL_CUDA_TRY(cudaFuncSetAttribute(k_scan<kLight, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scan_smem_bytes<8>()));
  ECL_CUDA_TRY(cudaFuncSetAttribute(k_scan<kLight, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scan_smem_bytes<16>()));
  ECL_CUDA_TRY(cudaFuncSetAttribute(k_scan<kHeavy, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scan_smem_bytes<4>()));
  ECL_CUDA_TRY(cudaFuncSetAttribute(k_scan<kHeavy, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scan_smem_bytes<8>()));
  ECL_CUDA_TRY(cudaFuncSetAttribute(k_scan<kHeavy, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scan_smem_bytes<16>()));
  return ECL_OK;
}

// Persistent scan: exactly as many CTAs as can be resident at once (a CTA
// started late would finish its share late), each looping over tiles. The
// warps' slot chunk is sized so that the unused chunk tails (at most
// chunk - 1 per warp) fit in the worklist's slack.
template <int KIND, int EPT>
int launch_scan_ept(const ScanArgs& sa, cudaStream_t s, const cudaAccessPolicyWindow* win) {
  const int64_t m = sa.edges;
  const int64_t tile = ScanCfg<EPT>::kTile;
  const int tiles = (int)((m + tile - 1) / tile);
  int per_sm = 0;
  ECL_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scan<KIND, EPT>, kScanThreads,
                                                             scan_smem_bytes<EPT>()));
  int blocks = std::max(1, std::min(tiles, std::max(1, per_sm) * sa.sm_count));
  ScanArgs a = sa;
  const int64_t warps = (int64_t)blocks * kScanWarps;
  a.chunk = (unsigned)std::max<int64_t>(1, std::min<int64_t>(kScanMaxChunk, (int64_t)sa.wl_slack / warps));
  if (win) return launch_ex(k_scan<KIND, EPT>, blocks, kScanThreads, scan_smem_bytes<EPT>(), s, false, win, a);
  k_scan<KIND, EPT><<<blocks, kScanThreads, scan_smem_bytes<EPT>(), s>>>(a);
  return cuda_status(cudaGetLastError());
}

template <int KIND>
int launch_scan(int ept, const ScanArgs& sa, cudaStream_t s, const cudaAccessPolicyWindow* win = nullptr) {
  if (ept == 4) return launch_scan_ept<KIND, 4>(sa, s, win);
  if (ept == 8) return launch_scan_ept<KIND, 8>(sa, s, win);
  return launch_scan_ept<KIND, 16>(sa, s, win);
}

// Scan variants to launch: the one the split selects, or all three (each
// exits unless st->split selects it) when the split is chosen on the device.
// Those three go on forked streams, so the two that exit at once do so beside
// the selected one instead of after it.
template <int KIND>
int launch_scans(ecl_mst_ctx* c, bool device_split, int split, const ScanArgs& sa, cudaStream_t s,
                 const cudaAccessPolicyWindow* win) {
  if (KIND == kHeavy && ECL_HEAVY_EPT) return launch_scan<KIND>(ECL_HEAVY_EPT, sa, s, win);
  if (!device_split) return launch_scan<KIND>(scan_ept(split), sa, s, win);
  const cudaStream_t br[2] = {c->side, c->side2};
  ECL_CUDA_TRY(cudaEventRecord(c->scan_fork, s));
  for (cudaStream_t b : br) ECL_CUDA_TRY(cudaStreamWaitEvent(b, c->scan_fork, 0));
  int st;
  if ((st = launch_scan<KIND>(8, sa, s, win))) return st;  // the split the network picks most often
  if ((st = launch_scan<KIND>(4, sa, br[0], win))) return st;
  if ((st = launch_scan<KIND>(16, sa, br[1], win))) return st;
  for (int i = 0; i < 2; i++) {
    ECL_CUDA_TRY(cudaEventRecord(c->scan_join[i], br[i]));
    ECL_CUDA_TRY(cudaStreamWaitEvent(s, c->scan_join[i], 0));
  }
  return ECL_OK;
}

// The L2 access-policy window of a solve (ECL_FLAG_L2_PERSIST): the packed
// min-slot and parent arrays (20n bytes; the min slots alone when the window
// limit is smaller), with the share of lines the persisting set-aside can
// hold marked persisting and the rest left normal.
bool l2_window(const ecl_mst_ctx* c, const Slots& sl, bool parent_only, cudaAccessPolicyWindow* w) {
  if (!c->l2_limit_set || c->l2_window_max == 0) return false;
  memset(w, 0, sizeof(*w));
  w->base_ptr = parent_only ? (void*)sl.parent : (void*)sl.minv0;
  size_t bytes = parent_only ? (sl.bytes / 5) : sl.bytes;  // parent is 4n of the 20n
  bytes = std::min(bytes, c->l2_window_max);
  if (bytes == 0) return false;
  w->num_bytes = bytes;
  size_t persist = 0;
  cudaDeviceGetLimit(&persist, cudaLimitPersistingL2CacheSize);
  w->hitRatio = (float)std::min(1.0, (double)persist / (double)bytes);
  w->hitProp = cudaAccessPropertyPersisting;
  w->missProp = cudaAccessPropertyStreaming;
  return true;
}

// The learned schedule's steps around k_prep. The weight sample is sorted on
// `side` from the start of the solve (ecl_learned_sample); k_prep gathers the
// degree statistics into `acc` on the solve's stream; the MLP then runs on
// `side` beside the fill scan, and the light scan waits for it.
struct LearnedPlan {
  cudaStream_t side;
  cudaEvent_t prep_done, join;
  FeatAcc* acc;
};

// Start of a learned solve on stream q: zero the degree accumulator (before
// k_prep adds to it), then fork the side stream and sort the weight sample
// there. Fills lp->acc.
int learned_fork(ecl_mst_ctx* c, const ecl_graph* g, cudaStream_t q, LearnedPlan* lp) {
  lp->acc = static_cast<FeatAcc*>(c->ml_acc);
  c->ml_features_set = true;
  ECL_CUDA_TRY(cudaMemsetAsync(lp->acc, 0, sizeof(FeatAcc), q));
  ECL_CUDA_TRY(cudaEventRecord(c->fork, q));
  ECL_CUDA_TRY(cudaStreamWaitEvent(lp->side, c->fork, 0));
  return ecl_learned_sample(c, g, lp->side);
}

int enqueue_solve(ecl_mst_ctx* c, const ecl_graph* g, unsigned char* d_inMST, const mst_opts* o,
                  cudaStream_t s, bool timed, const LearnedPlan* lp = nullptr) {
  const int n = g->nodes, m = g->edges;
  const int split = o->degree_split > 0 ? o->degree_split : kDefaultSplit;
  const bool device_split = o->threshold_mode == ECL_THRESH_LEARNED;
  const int tiles = (int)(((int64_t)m + kGran - 1) / kGran);
  const Slots sl = slots_for(c->slots, n);
  // L2 persistence: k_prep writes the slots and parent, the rounds hammer
  // them, the flatten pass and the heavy scan gather parent[]
  cudaAccessPolicyWindow w_all, w_par;
  const bool l2 = (o->flags & ECL_FLAG_L2_PERSIST) != 0;
  const cudaAccessPolicyWindow* win_all = l2 && l2_window(c, sl, false, &w_all) ? &w_all : nullptr;
  const cudaAccessPolicyWindow* win_par = l2 && l2_window(c, sl, true, &w_par) ? &w_par : nullptr;
  PrepArgs pa{};
  pa.nodes = n;
  pa.edges = m;
  pa.nindex = g->nindex;
  pa.eweight = g->eweight;
  pa.parent = sl.parent;
  pa.minv0 = sl.minv0;
  pa.minv1 = sl.minv1;
  pa.first_v = c->first_v;
  pa.tiles = tiles;
  pa.mode = o->threshold_mode;
  pa.explicit_thr = o->threshold;
  pa.split = split;
  pa.quantile = o->quantile;
  pa.st = c->st;
  pa.feat = lp ? lp->acc : nullptr;
  int st;
  std::function<int()> fork_mlp;
  if (lp)
    fork_mlp = [&]() -> int {
      ECL_CUDA_TRY(cudaEventRecord(lp->prep_done, s));
      ECL_CUDA_TRY(cudaStreamWaitEvent(lp->side, lp->prep_done, 0));
      const int r = ecl_learned_apply(c, g, lp->side, c->st);
      if (r) return r;
      ECL_CUDA_TRY(cudaEventRecord(lp->join, lp->side));
      return ECL_OK;
    };
  if ((st = enqueue_prep(pa, c->sm_count, s, win_all, fork_mlp))) return st;
  if (lp) ECL_CUDA_TRY(cudaStreamWaitEvent(s, lp->join, 0));
  const bool no_tuples = (o->flags & (ECL_FLAG_NO_TUPLES | ECL_FLAG_NO_EDGE_BASED)) == ECL_FLAG_NO_TUPLES;
  if (no_tuples) {  // the vertex of every entry, for the gathers of the rounds
    const int sgrid = (int)std::min<int64_t>(((int64_t)m + kThreads - 1) / kThreads, (int64_t)c->sm_count * 16);
    k_slist<<<std::max(sgrid, 1), kThreads, 0, s>>>(g->nindex, c->first_v, c->slist, m, c->st);
    ECL_CUDA_TRY(cudaGetLastError());
  }
  ScanArgs sa{};
  sa.nodes = n;
  sa.edges = m;
  sa.nindex = g->nindex;
  sa.nlist = g->nlist;
  sa.eweight = g->eweight;
  sa.first_v = c->first_v;
  sa.tiles = tiles;
  sa.parent = sl.parent;
  sa.wl = c->wl[0];
  sa.wl_cap = c->wl_cap;
  // a scan keeps at most m entries, m / 2 for the symmetric input the
  // half-size lists assume (more overflows, and the solve is repeated)
  sa.wl_slack = c->wl_cap - (unsigned)(c->wl_full ? m : m / 2);
  sa.inMST = d_inMST;
  sa.vec_ok = ((((uintptr_t)g->nlist) | ((uintptr_t)g->eweight)) & 15) == 0;
  sa.zero_vec = (((uintptr_t)d_inMST) & 15) == 0;
  sa.st = c->st;
  sa.sm_count = c->sm_count;
  sa.ids = no_tuples ? 1 : 0;
  RoundArgs ra{};
  ra.nodes = n;
  ra.wl0 = c->wl[0];
  ra.wl1 = c->wl[1];
  ra.wl_cap = c->wl_cap;
  ra.parent = sl.parent;
  ra.minv0 = sl.minv0;
  ra.minv1 = sl.minv1;
  ra.inMST = d_inMST;
  ra.st = c->st;
  ra.small_tail = o->small_tail < 0 ? 0u : (o->small_tail == 0 ? kDefaultSmallTail : (unsigned)o->small_tail);
  if (o->flags & ECL_FLAG_NO_SMALL_TAIL) ra.small_tail = 0;
  ra.count_atomics = (o->flags & ECL_FLAG_STATS) ? 1 : 0;
  ra.abl = round_ablation(o->flags);
  ra.nlist = g->nlist;
  ra.eweight = g->eweight;
  ra.slist = c->slist;
  // entries that keep their endpoints clear the whole previous min array
  // each round, which one CTA of a small tail would do alone
  if (ra.abl & kAblKeepEnds) ra.small_tail = 0;
  ra.min_tiles = o->round_min_tiles < 0 ? 0 : (o->round_min_tiles == 0 ? kDefaultMinTiles : o->round_min_tiles);
  int rmax = c->round_grid;
  if (o->ctas_per_sm > 0) rmax = std::min(rmax, o->ctas_per_sm * c->sm_count);
  const int rgrid = std::max(1, std::min(rmax, (m / 2 + kRoundThreads - 1) / kRoundThreads + 1));
  if (o->flags & ECL_FLAG_NO_EDGE_BASED) {
    // vertex-centric rounds straight over the CSR: no scans, no worklists
    if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[5], s));
    ECL_CUDA_TRY(cudaMemsetAsync(d_inMST, 0, (size_t)m, s));
    if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[1], s));
    ra.phase = 0;
    if ((st = launch_ex(k_rounds_vertex, c->vertex_grid, kRoundThreads, 0, s, true, nullptr, ra, g->nindex)))
      return st;
    if (timed) {
      ECL_CUDA_TRY(cudaEventRecord(c->ev[2], s));
      ECL_CUDA_TRY(cudaEventRecord(c->ev[6], s));
      ECL_CUDA_TRY(cudaEventRecord(c->ev[3], s));
    }
    ra.phase = 1;
    if ((st = launch_ex(k_rounds_vertex, c->vertex_grid, kRoundThreads, 0, s, true, nullptr, ra, g->nindex)))
      return st;
    if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[4], s));
    return ECL_OK;
  }
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[5], s));
  if ((st = launch_scans<kLight>(c, device_split, split, sa, s, nullptr))) return st;
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  ra.phase = 0;
  if (win_all) st = launch_ex(k_rounds, rgrid, kRoundThreads, 0, s, true, win_all, ra);
  else st = launch_coop((const void*)k_rounds, rgrid, kRoundThreads, &ra, s);
  if (st) return st;
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[2], s));
  const int fgrid = (int)std::min<int64_t>(((int64_t)n + kThreads - 1) / kThreads, (int64_t)c->sm_count * 16);
  if (win_par) {
    if ((st = launch_ex(k_flatten, std::max(fgrid, 1), kThreads, 0, s, false, win_par, sl.parent, n,
                        (const DevState*)c->st)))
      return st;
  } else {
    k_flatten<<<std::max(fgrid, 1), kThreads, 0, s>>>(sl.parent, n, c->st);
    ECL_CUDA_TRY(cudaGetLastError());
  }
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[6], s));
  if ((st = launch_scans<kHeavy>(c, device_split, split, sa, s, win_par))) return st;
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[3], s));
  ra.phase = 1;
  if (win_all) st = launch_ex(k_rounds, rgrid, kRoundThreads, 0, s, true, win_all, ra);
  else st = launch_coop((const void*)k_rounds, rgrid, kRoundThreads, &ra, s);
  if (st) return st;
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[4], s));
  return ECL_OK;
}

int fill_stats(ecl_mst_ctx* c, ecl_mst_stats* stats, bool timed, bool breakdown = true) {
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
    stats->scan_kept[p] = h.scan_kept[p];
    for (int r = 0; r < ECL_MAX_ROUNDS; r++) {
      stats->wl_in[p][r] = h.wl_count[p][r];
      stats->wl_real[p][r] = r == 0 ? h.scan_kept[p] : h.wl_kept[p][r];
    }
  }
  stats->atomics = (int64_t)h.atomics;
  for (int p = 0; p < 2; p++) {
    u64 prev = h.t_round_start[p];
    for (int r = 0; r < h.rounds[p] && r < ECL_MAX_ROUNDS; r++) {
      const u64 a = h.t_round[p][2 * r], b = h.t_round[p][2 * r + 1];
      if (a && prev) stats->us_round[p][r][0] = (a - prev) * 1e-3f;
      if (b && a) stats->us_round[p][r][1] = (b - a) * 1e-3f;
      prev = b ? b : a;
    }
  }
  if (timed && !breakdown) {  // a replayed graph: only the whole solve is timed
    cudaEventElapsedTime(&stats->ms_total, c->ev[0], c->ev[4]);
  } else if (timed) {
    float t01, t12, t23, t34, t04;
    cudaEventElapsedTime(&t01, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&t12, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&t23, c->ev[2], c->ev[3]);
    cudaEventElapsedTime(&t34, c->ev[3], c->ev[4]);
    cudaEventElapsedTime(&t04, c->ev[0], c->ev[4]);
    stats->ms_scan = t01 + t23;
    stats->ms_rounds = t12 + t34;
    stats->ms_total = t04;
    float t05, t26;
    cudaEventElapsedTime(&t05, c->ev[0], c->ev[5]);
    cudaEventElapsedTime(&t26, c->ev[2], c->ev[6]);
    stats->us_scan[0][0] = t01 * 1e3f;
    stats->us_scan[0][1] = t05 * 1e3f;
    stats->us_scan[0][2] = (t01 - t05) * 1e3f;
    stats->us_scan[1][0] = t23 * 1e3f;
    stats->us_scan[1][1] = t26 * 1e3f;
    stats->us_scan[1][2] = (t23 - t26) * 1e3f;
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
  if (o->ctas_per_sm < 0) return ECL_ERR_INVALID_ARG;
  if (o->batch_large_streams < 0 || o->batch_large_streams > 8) return ECL_ERR_INVALID_ARG;
  if (o->threshold_mode == ECL_THRESH_QUANTILE && !(o->quantile >= 0.0f)) return ECL_ERR_INVALID_ARG;
  return ECL_OK;
}

}  // namespace

int ecl_ctx_learned_buffers(ecl_mst_ctx* c, float** params, float** feat, void** acc, int** sample,
                            unsigned** version, int* sm_count) {
  *sample = c->ml_sample;
  *version = &c->ml_version;
  *params = c->ml_params;
  *feat = c->ml_feat;
  *acc = c->ml_acc;
  *sm_count = c->sm_count;
  return ECL_OK;
}

namespace {

int run_device_once(ecl_mst_ctx* c, const ecl_graph* g, uint8_t* d_inMST, const mst_opts* opts, void* stream,
                    ecl_mst_stats* stats) {
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
  // Graphs below kLearnedMinEdges CSR entries keep the reference heuristic:
  // there the feature pass costs about as much as any schedule can save.
  // Without loaded weights the heuristic is the fallback.
  if (o.threshold_mode == ECL_THRESH_LEARNED && (g->edges < kLearnedMinEdges || !ecl_learned_has_weights()))
    o.threshold_mode = ECL_THRESH_HEURISTIC;
  const bool timed = stats != nullptr;
  if ((o.flags & ECL_FLAG_NO_TUPLES) && !c->slist)  // the ablation's per-entry vertex list, once
    ECL_CUDA_TRY(cudaMalloc(&c->slist, (size_t)std::max<int64_t>(c->max_edges, 1) * sizeof(int)));
  if (o.flags & ECL_FLAG_L2_PERSIST) {
    // Persisting set-aside for this process's context, sized for the solve's
    // slot arrays (20n bytes) up to the device maximum; set before any
    // capture, restored when the context is destroyed.
    const size_t want = std::min(c->l2_persist_max, (size_t)g->nodes * (2 * sizeof(u64) + sizeof(int)));
    size_t cur = 0;
    ECL_CUDA_TRY(cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize));
    if (!c->l2_limit_set) c->l2_limit_prev = cur;
    if (want > cur) ECL_CUDA_TRY(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want));
    c->l2_limit_set = want > 0 || c->l2_limit_set;
  }
  // inner_events: the per-phase timing events (not inside a captured graph)
  auto enqueue_all = [&](cudaStream_t q, bool inner_events) -> int {
    ECL_CUDA_TRY(cudaMemsetAsync(c->st, 0, sizeof(DevState), q));
    // the timed window starts before the learned schedule's feature pass
    if (inner_events) ECL_CUDA_TRY(cudaEventRecord(c->ev[0], q));
    if (o.threshold_mode != ECL_THRESH_LEARNED) return enqueue_solve(c, g, d_inMST, &o, q, inner_events);
    LearnedPlan lp{c->side, c->prep_done, c->join, nullptr};
    const int r = learned_fork(c, g, q, &lp);
    return r ? r : enqueue_solve(c, g, d_inMST, &o, q, inner_events, &lp);
  };
  // A solve repeated with the same graph, buffers and options (benchmarks,
  // iterative callers) is captured once as a CUDA graph and then replayed
  // with a single launch: the first repeat captures, later ones replay. A
  // replay is timed as a whole (events around the launch), so its stats have
  // ms_total but no per-phase breakdown; ECL_FLAG_NO_GRAPH keeps the direct
  // launches and the breakdown.
  int32_t qbits;  // the quantile's bit pattern
  memcpy(&qbits, &o.quantile, sizeof(qbits));
  const std::vector<long long> key = {
      g->nodes, g->edges, (long long)(uintptr_t)g->nindex, (long long)(uintptr_t)g->nlist,
      (long long)(uintptr_t)g->eweight, (long long)(uintptr_t)d_inMST, o.threshold_mode, o.threshold,
      (long long)qbits, o.degree_split, o.small_tail, o.flags, o.round_min_tiles, o.ctas_per_sm,
      (long long)(uintptr_t)c->wl[0], (long long)ecl_learned_weights_version()};
  const bool graph_ok = !(o.flags & ECL_FLAG_NO_GRAPH);
  bool replayed = false;
  auto replay = [&]() -> int {
    if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[0], s));
    ECL_CUDA_TRY(cudaGraphLaunch(c->exec, s));
    if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[4], s));
    replayed = true;
    return ECL_OK;
  };
  if (graph_ok && c->exec && c->exec_key == key) {
    if ((st = replay())) return st;
  } else if (graph_ok && key == c->last_key) {
    if (c->exec) {
      cudaGraphExecDestroy(c->exec);
      c->exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    bool captured = false;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      const int r = enqueue_all(s, false);
      const cudaError_t e = cudaStreamEndCapture(s, &graph);
      if (r == ECL_OK && e == cudaSuccess && graph && cudaGraphInstantiate(&c->exec, graph, 0) == cudaSuccess) {
        captured = true;
        c->exec_key = key;
      }
      if (graph) cudaGraphDestroy(graph);
    }
    cudaGetLastError();  // clear a failed capture's error state
    if (captured) {
      if ((st = replay())) return st;
    } else {
      c->exec = nullptr;
      if ((st = enqueue_all(s, timed))) return st;
    }
  } else {
    if ((st = enqueue_all(s, timed))) return st;
  }
  c->last_key = key;
  if (stats) {
    if (s != c->stream) {
      ECL_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return fill_stats(c, stats, true, !replayed);
  }
  return ECL_OK;
}

// Worklists grown to hold every CSR entry; the captured solve refers to the
// old lists and is dropped.
int grow_worklists(ecl_mst_ctx* c) {
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  ECL_CUDA_TRY(cudaDeviceSynchronize());
  if (c->exec) {
    cudaGraphExecDestroy(c->exec);
    c->exec = nullptr;
  }
  c->exec_key.clear();
  c->last_key.clear();
  return alloc_worklists(c, true);
}

}  // namespace

extern "C" int ecl_mst_run_device(ecl_mst_ctx* c, const ecl_graph* g, uint8_t* d_inMST,
                                  const mst_opts* opts, void* stream, ecl_mst_stats* stats) {
  int st = run_device_once(c, g, d_inMST, opts, stream, stats);
  if (!c) return st;
  if (stats) {
    // The solve has finished: an input with more one-direction entries than
    // the half-size worklists hold is solved again with full-size ones.
    c->pending = false;
    if (st == ECL_ERR_OVERFLOW && !c->wl_full && (c->st_host->error & kErrOverflow)) {
      if ((st = grow_worklists(c))) return st;
      st = run_device_once(c, g, d_inMST, opts, stream, stats);
    }
    return st;
  }
  if (st == ECL_OK) {  // enqueued: ecl_mst_ctx_sync checks it and repeats it on overflow
    c->pending = true;
    c->pend_graph = *g;
    c->pend_out = d_inMST;
    if (opts) c->pend_opts = *opts;
    else ecl_default_opts(&c->pend_opts);
    c->pend_stream = stream ? (cudaStream_t)stream : c->stream;
  }
  return st;
}

namespace {

// Device CSR and inMST buffers for host-buffer solves, allocated on first use.
int host_buffers(ecl_mst_ctx* c, int** ni, int** nl, int** ew, unsigned char** out) {
  if (*ni) return ECL_OK;
  const size_t nb = ((size_t)c->max_nodes + 1) * 4, eb = (size_t)std::max<int64_t>(c->max_edges, 1) * 4;
  ECL_CUDA_TRY(cudaMalloc(ni, nb));
  ECL_CUDA_TRY(cudaMalloc(nl, eb));
  ECL_CUDA_TRY(cudaMalloc(ew, eb));
  ECL_CUDA_TRY(cudaMalloc(out, eb / 4));
  return ECL_OK;
}

}  // namespace

extern "C" int ecl_mst_ctx_run_host(ecl_mst_ctx* c, const ecl_graph* g, uint8_t* inMST,
                                    const mst_opts* opts, ecl_mst_stats* stats) {
  int st = check_graph_args(c, g, inMST);
  if (st) return st;
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  if ((st = host_buffers(c, &c->d_nindex, &c->d_nlist, &c->d_eweight, &c->d_inMST))) return st;
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
  if (c->resolved && m > 0) {  // the solve was repeated after a worklist overflow
    ECL_CUDA_TRY(cudaMemcpyAsync(inMST, c->d_inMST, (size_t)m, cudaMemcpyDeviceToHost, c->stream));
    ECL_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
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

namespace {

__global__ void k_sticky_or(const DevState* st, unsigned* sticky) {
  const unsigned e = ld_volatile(&st->error);
  if (e) atomicOr(sticky, e);
}

// Streams, events, the second buffer set and the sticky error word of the
// pipelined solves, created on first use.
int async_setup(ecl_mst_ctx* c) {
  if (c->cin) return ECL_OK;
  int st;
  if ((st = host_buffers(c, &c->d_nindex, &c->d_nlist, &c->d_eweight, &c->d_inMST))) return st;
  c->hs[0].nindex = c->d_nindex;
  c->hs[0].nlist = c->d_nlist;
  c->hs[0].eweight = c->d_eweight;
  c->hs[0].inMST = c->d_inMST;
  if ((st = host_buffers(c, &c->hs[1].nindex, &c->hs[1].nlist, &c->hs[1].eweight, &c->hs[1].inMST))) return st;
  for (auto& h : c->hs)
    for (cudaEvent_t* e : {&h.in_done, &h.solved, &h.out_done})
      ECL_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  ECL_CUDA_TRY(cudaMalloc(&c->sticky, sizeof(unsigned)));
  ECL_CUDA_TRY(cudaMemset(c->sticky, 0, sizeof(unsigned)));
  ECL_CUDA_TRY(cudaStreamCreateWithFlags(&c->cout, cudaStreamNonBlocking));
  ECL_CUDA_TRY(cudaStreamCreateWithFlags(&c->cin, cudaStreamNonBlocking));
  return ECL_OK;
}

}  // namespace

extern "C" int ecl_mst_ctx_run_host_async(ecl_mst_ctx* c, const ecl_graph* g, uint8_t* inMST,
                                          const mst_opts* opts) {
  int st = check_graph_args(c, g, inMST);
  if (st) return st;
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  if ((st = async_setup(c))) return st;
  auto& h = c->hs[c->async_seq++ & 1];
  const int n = g->nodes, m = g->edges;
  // copy in, once the solve that last read this set's CSR has finished
  if (h.used) ECL_CUDA_TRY(cudaStreamWaitEvent(c->cin, h.solved, 0));
  ECL_CUDA_TRY(cudaMemcpyAsync(h.nindex, g->nindex, ((size_t)n + 1) * 4, cudaMemcpyHostToDevice, c->cin));
  if (m > 0) {
    ECL_CUDA_TRY(cudaMemcpyAsync(h.nlist, g->nlist, (size_t)m * 4, cudaMemcpyHostToDevice, c->cin));
    ECL_CUDA_TRY(cudaMemcpyAsync(h.eweight, g->eweight, (size_t)m * 4, cudaMemcpyHostToDevice, c->cin));
  }
  ECL_CUDA_TRY(cudaEventRecord(h.in_done, c->cin));
  // solve on the context's stream once the inputs are in and the set's
  // previous inMST has been copied out; its device errors accumulate
  ECL_CUDA_TRY(cudaStreamWaitEvent(c->stream, h.in_done, 0));
  if (h.used) ECL_CUDA_TRY(cudaStreamWaitEvent(c->stream, h.out_done, 0));
  ecl_graph dg = {n, m, h.nindex, h.nlist, h.eweight};
  if ((st = run_device_once(c, &dg, h.inMST, opts, c->stream, nullptr))) return st;
  k_sticky_or<<<1, 1, 0, c->stream>>>(c->st, c->sticky);
  ECL_CUDA_TRY(cudaGetLastError());
  ECL_CUDA_TRY(cudaEventRecord(h.solved, c->stream));
  // copy out beside the next graph's copy in and solve
  ECL_CUDA_TRY(cudaStreamWaitEvent(c->cout, h.solved, 0));
  if (m > 0) ECL_CUDA_TRY(cudaMemcpyAsync(inMST, h.inMST, (size_t)m, cudaMemcpyDeviceToHost, c->cout));
  ECL_CUDA_TRY(cudaEventRecord(h.out_done, c->cout));
  h.used = true;
  ecl_mst_ctx::AsyncCall call;
  call.g = *g;
  call.out = inMST;
  if (opts) call.opts = *opts;
  else ecl_default_opts(&call.opts);
  c->async_calls.push_back(call);
  c->pending = false;
  return ECL_OK;
}

extern "C" int ecl_mst_ctx_wait(ecl_mst_ctx* c) {
  if (!c) return ECL_ERR_INVALID_ARG;
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  if (!c->cin) return ECL_OK;
  ECL_CUDA_TRY(cudaStreamSynchronize(c->cin));
  ECL_CUDA_TRY(cudaStreamSynchronize(c->stream));
  ECL_CUDA_TRY(cudaStreamSynchronize(c->cout));
  unsigned err = 0;
  ECL_CUDA_TRY(cudaMemcpy(&err, c->sticky, sizeof(unsigned), cudaMemcpyDeviceToHost));
  ECL_CUDA_TRY(cudaMemset(c->sticky, 0, sizeof(unsigned)));
  std::vector<ecl_mst_ctx::AsyncCall> calls;
  calls.swap(c->async_calls);
  if ((err & kErrOverflow) && !c->wl_full) {
    // an input had more one-direction entries than half its CSR entries:
    // grow the worklists and solve the calls since the last wait again
    int st = grow_worklists(c);
    if (st) return st;
    for (auto& call : calls)
      if ((st = ecl_mst_ctx_run_host(c, &call.g, call.out, &call.opts, nullptr))) return st;
    return ECL_OK;
  }
  return device_error_status(err);
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

// ===================================================== allocation-free solve
// Some callers cannot allocate device memory: code that runs inside a host
// allocator hook or a memory-pool callback, an embedding that owns every
// allocation of the process, or a service whose device memory budget is
// fixed at start-up. ecl_mst_run_device_noalloc serves them: its scratch
// (min slots, parent array, worklists, control block) is one file-scope
// device array, created when the module loads and kept until the process
// exits, on every GPU that loads this library. The caller passes only the
// device CSR and the device inMST output.
#include <mutex>

namespace {

constexpr int64_t kNaMaxNodes = 1 << 18;              // 262,144 vertices
constexpr int64_t kNaMaxEdges = 1 << 20;              // 1,048,576 directed CSR entries
constexpr int64_t kNaWlCap = kNaMaxEdges / 2;         // one-direction entries per worklist
// tile -> vertex table entries, with the fill scan's chunk maxima
constexpr int64_t kNaTiles = kNaMaxEdges / kGran + 2 + (kNaMaxEdges / kGran + 1) / kFillChunk + 1;

constexpr size_t na_align(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kNaOffState = 0;
constexpr size_t kNaOffMinv0 = na_align(kNaOffState + sizeof(DevState));
constexpr size_t kNaOffMinv1 = na_align(kNaOffMinv0 + sizeof(u64) * kNaMaxNodes);
constexpr size_t kNaOffParent = na_align(kNaOffMinv1 + sizeof(u64) * kNaMaxNodes);
constexpr size_t kNaOffFirstV = na_align(kNaOffParent + sizeof(int) * kNaMaxNodes);
constexpr size_t kNaOffWl0 = na_align(kNaOffFirstV + sizeof(int) * kNaTiles);
constexpr size_t kNaOffWl1 = na_align(kNaOffWl0 + sizeof(int4) * kNaWlCap);
constexpr size_t kNaBytes = na_align(kNaOffWl1 + sizeof(int4) * kNaWlCap);  // about 21 MB

// The scratch itself. In host code this name is only a stand-in for the
// symbol, never a device address: the address comes from
// cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_na_scratch[kNaBytes];

struct NaDevice {
  bool ready = false;
  unsigned char* base = nullptr;  // device address of g_na_scratch on this device
  int sm_count = 0;
  int round_grid = 0;
};
constexpr int kNaMaxDevices = 64;
NaDevice g_na_dev[kNaMaxDevices];
std::mutex g_na_mu;

// Once per device, with that device current: resolve the scratch address and
// the cooperative grid size. No allocation happens here.
int na_setup(int dev, NaDevice** out) {
  if (dev < 0 || dev >= kNaMaxDevices) return ECL_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_na_mu);
  NaDevice& d = g_na_dev[dev];
  // The scratch array's address is looked up on every call: a device reset
  // reloads the module, and the array then lives elsewhere.
  void* p = nullptr;
  ECL_CUDA_TRY(cudaGetSymbolAddress(&p, g_na_scratch));
  d.base = (unsigned char*)p;
  if (!d.ready) {
    int coop = 0;
    ECL_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return ECL_ERR_UNSUPPORTED;
    ECL_CUDA_TRY(cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev));
    d.round_grid = std::min(coop_grid((const void*)k_rounds, kRoundThreads, d.sm_count), kMaxRoundCtas);
    int ps = prepare_scan_kernels();
    if (ps) return ps;
    if (d.round_grid <= 0) return ECL_ERR_CUDA;
    d.ready = true;
  }
  *out = &d;
  return ECL_OK;
}

}  // namespace

extern "C" int ecl_mst_run_device_noalloc(const ecl_graph* g, uint8_t* d_inMST,
                                          const mst_opts* opts, void* stream) {
  if (!g || !d_inMST || g->nodes < 1 || g->edges < 0) return ECL_ERR_INVALID_ARG;
  if (g->nodes > kNaMaxNodes || g->edges > kNaMaxEdges) return ECL_ERR_TOO_LARGE;
  if (!g->nindex || (g->edges > 0 && (!g->nlist || !g->eweight))) return ECL_ERR_INVALID_ARG;
  mst_opts o;
  if (opts) o = *opts;
  else ecl_default_opts(&o);
  int st = check_opts(&o);
  if (st) return st;
  // The learned schedule's feature pass needs scratch this entry point does
  // not hold; it takes the reference heuristic, as ecl_mst_run_device does
  // below its learned-schedule cut-off.
  if (o.threshold_mode == ECL_THRESH_LEARNED) o.threshold_mode = ECL_THRESH_HEURISTIC;
  if (o.flags & kDeoptFlags) return ECL_ERR_UNSUPPORTED;  // single-graph contexts only
  if (g->edges == 0) return ECL_OK;
  int dev = 0;
  ECL_CUDA_TRY(cudaGetDevice(&dev));
  NaDevice* d = nullptr;
  if ((st = na_setup(dev, &d))) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const int n = g->nodes, m = g->edges;
  DevState* dst = (DevState*)(d->base + kNaOffState);
  int* parent = (int*)(d->base + kNaOffParent);
  u64* minv0 = (u64*)(d->base + kNaOffMinv0);
  u64* minv1 = (u64*)(d->base + kNaOffMinv1);
  int* first_v = (int*)(d->base + kNaOffFirstV);
  int4* wl0 = (int4*)(d->base + kNaOffWl0);
  int4* wl1 = (int4*)(d->base + kNaOffWl1);
  // The array keeps the previous call's contents: the control block (error
  // word, worklist counters, barrier) must start at zero; k_prep initialises
  // parent[] and both min arrays.
  ECL_CUDA_TRY(cudaMemsetAsync(dst, 0, sizeof(DevState), s));
  const int split = o.degree_split > 0 ? o.degree_split : kDefaultSplit;
  const int tiles = (int)(((int64_t)m + kGran - 1) / kGran);
  PrepArgs pa{};
  pa.nodes = n;
  pa.edges = m;
  pa.nindex = g->nindex;
  pa.eweight = g->eweight;
  pa.parent = parent;
  pa.minv0 = minv0;
  pa.minv1 = minv1;
  pa.first_v = first_v;
  pa.tiles = tiles;
  pa.mode = o.threshold_mode;
  pa.explicit_thr = o.threshold;
  pa.split = split;
  pa.quantile = o.quantile;
  pa.st = dst;
  st = enqueue_prep(pa, d->sm_count, s);
  if (st) return st;
  ScanArgs sa{};
  sa.nodes = n;
  sa.edges = m;
  sa.nindex = g->nindex;
  sa.nlist = g->nlist;
  sa.eweight = g->eweight;
  sa.first_v = first_v;
  sa.tiles = tiles;
  sa.parent = parent;
  sa.wl = wl0;
  sa.wl_cap = (unsigned)kNaWlCap;
  // within the stated limit a scan keeps at most m / 2 entries
  sa.wl_slack = (unsigned)std::max<int64_t>(0, kNaWlCap - m / 2);
  sa.inMST = d_inMST;
  sa.vec_ok = ((((uintptr_t)g->nlist) | ((uintptr_t)g->eweight)) & 15) == 0;
  sa.zero_vec = (((uintptr_t)d_inMST) & 15) == 0;
  sa.st = dst;
  sa.sm_count = d->sm_count;
  RoundArgs ra{};
  ra.nodes = n;
  ra.wl0 = wl0;
  ra.wl1 = wl1;
  ra.wl_cap = (unsigned)kNaWlCap;
  ra.parent = parent;
  ra.minv0 = minv0;
  ra.minv1 = minv1;
  ra.inMST = d_inMST;
  ra.st = dst;
  ra.small_tail = o.small_tail < 0 ? 0u : (o.small_tail == 0 ? kDefaultSmallTail : (unsigned)o.small_tail);
  if (o.flags & ECL_FLAG_NO_SMALL_TAIL) ra.small_tail = 0;
  ra.count_atomics = (o.flags & ECL_FLAG_STATS) ? 1 : 0;
  ra.abl = round_ablation(o.flags);
  const int rgrid = std::max(1, std::min(d->round_grid, (m / 2 + kRoundThreads - 1) / kRoundThreads + 1));
  if ((st = launch_scan<kLight>(scan_ept(split), sa, s))) return st;
  ra.phase = 0;
  if ((st = launch_coop((const void*)k_rounds, rgrid, kRoundThreads, &ra, s))) return st;
  const int fgrid = (int)std::min<int64_t>(((int64_t)n + kThreads - 1) / kThreads, (int64_t)d->sm_count * 16);
  k_flatten<<<std::max(fgrid, 1), kThreads, 0, s>>>(parent, n, dst);
  ECL_CUDA_TRY(cudaGetLastError());
  if ((st = launch_scan<kHeavy>(heavy_ept(split), sa, s))) return st;
  ra.phase = 1;
  if ((st = launch_coop((const void*)k_rounds, rgrid, kRoundThreads, &ra, s))) return st;
  // Report device-side errors (malformed CSR, worklist overflow) to the caller.
  unsigned err = 0;
  ECL_CUDA_TRY(cudaMemcpyAsync(&err, &dst->error, sizeof(err), cudaMemcpyDeviceToHost, s));
  ECL_CUDA_TRY(cudaStreamSynchronize(s));
  return device_error_status(err);
}

// ============================================================== batched mode
namespace {

__global__ void k_or_error(const DevState* src, DevState* dst) {
  const unsigned e = ld_volatile(&src->error);
  if (e) atomicOr(&dst->error, e);
}

constexpr int kBatchDefaultCap = 1 << 19;
constexpr int kMaxLargeStreams = 8;      // concurrent streams for a batch's large graphs
constexpr int kDefaultLargeStreams = 4;  // measured: 957 large graphs of the mixed batch 1.5x faster than on one

}  // namespace

struct ecl_batch_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 0;
  int max_graphs = 0;
  int64_t max_nodes = 0, max_edges = 0;
  int cap = 0;        // per-CTA scratch: vertices and CSR entries
  int small_grid = 0; // CTAs of the persistent kernel
  int* parent_pool = nullptr;
  u64* minv_pool = nullptr;
  int4* wl_pool = nullptr;
  long long* d_node_off = nullptr;
  long long* d_edge_off = nullptr;
  int* d_small = nullptr;
  unsigned* d_queue = nullptr;
  DevState* st = nullptr;
  // grid-wide engines for the graphs beyond the cutoff, one per concurrent
  // stream: [0] is made with the context, the others when a solve asks for
  // more streams (opts batch_large_streams)
  ecl_mst_ctx* big[kMaxLargeStreams] = {};
  cudaEvent_t large_fork = nullptr, large_join[kMaxLargeStreams] = {};
  cudaEvent_t ev[3] = {};
  // the large-graph launch sequence captured as a CUDA graph, keyed by the batch
  cudaGraphExec_t exec = nullptr;
  std::vector<long long> exec_key;
};

// Grid-wide engine k of a batch context, sized for its largest graph. The
// batch's solves are captured and replayed without a host check in between,
// so its lists hold every entry of any input.
static int batch_big_ctx(ecl_batch_ctx* c, int k) {
  if (c->big[k]) return ECL_OK;
  int st = ecl_mst_ctx_create(c->device, c->max_nodes, std::max<int64_t>(c->max_edges, 1), &c->big[k]);
  if (!st) st = alloc_worklists(c->big[k], true);
  if (st) {
    ecl_mst_ctx_destroy(c->big[k]);
    c->big[k] = nullptr;
  }
  return st;
}

extern "C" void ecl_batch_ctx_destroy(ecl_batch_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->exec) cudaGraphExecDestroy(c->exec);
  cudaFree(c->parent_pool);
  cudaFree(c->minv_pool);
  cudaFree(c->wl_pool);
  cudaFree(c->d_node_off);
  cudaFree(c->d_edge_off);
  cudaFree(c->d_small);
  cudaFree(c->d_queue);
  cudaFree(c->st);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->large_fork) cudaEventDestroy(c->large_fork);
  for (auto& e : c->large_join)
    if (e) cudaEventDestroy(e);
  for (ecl_mst_ctx* b : c->big) ecl_mst_ctx_destroy(b);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" int ecl_batch_ctx_create(int device, int32_t max_graphs, int64_t max_graph_nodes,
                                    int64_t max_graph_edges, int32_t small_cap, ecl_batch_ctx** out) {
  if (!out || max_graphs < 1 || max_graph_nodes < 1 || max_graph_edges < 0 || small_cap < 0)
    return ECL_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return ECL_ERR_NO_DEVICE;
  if (device < 0 || device >= ndev) return ECL_ERR_INVALID_ARG;
  ECL_CUDA_TRY(cudaSetDevice(device));
  ecl_batch_ctx* c = new (std::nothrow) ecl_batch_ctx();
  if (!c) return ECL_ERR_ALLOC;
  c->device = device;
  c->max_graphs = max_graphs;
  c->max_nodes = max_graph_nodes;
  c->max_edges = max_graph_edges;
  c->cap = small_cap > 0 ? small_cap : kBatchDefaultCap;
  int st;
  auto fail = [&](int s) {
    ecl_batch_ctx_destroy(c);
    return s;
  };
  if ((st = cuda_status(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device))))
    return fail(st);
  if ((st = cuda_status(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)))) return fail(st);
  int per_sm = 0;
  if ((st = cuda_status(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_batch_small,
                                                                      kThreads, 0))))
    return fail(st);
  c->small_grid = std::max(1, per_sm) * c->sm_count;
  const size_t ctas = (size_t)c->small_grid, cap = (size_t)c->cap;
  if ((st = cuda_status(cudaMalloc(&c->parent_pool, ctas * cap * sizeof(int))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->minv_pool, ctas * 2 * cap * sizeof(u64))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->wl_pool, ctas * 2 * cap * sizeof(int4))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->d_node_off, 2 * (size_t)max_graphs * sizeof(long long))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->d_edge_off, 2 * (size_t)max_graphs * sizeof(long long))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->d_small, (size_t)max_graphs * sizeof(int))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->d_queue, sizeof(unsigned))))) return fail(st);
  if ((st = cuda_status(cudaMalloc(&c->st, sizeof(DevState))))) return fail(st);
  for (auto& e : c->ev)
    if ((st = cuda_status(cudaEventCreate(&e)))) return fail(st);
  if ((st = cuda_status(cudaEventCreateWithFlags(&c->large_fork, cudaEventDisableTiming)))) return fail(st);
  for (auto& e : c->large_join)
    if ((st = cuda_status(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)))) return fail(st);
  if (max_graph_edges > c->cap || max_graph_nodes > c->cap)
    if ((st = batch_big_ctx(c, 0))) return fail(st);
  *out = c;
  return ECL_OK;
}

namespace {

// Per-graph descriptors for the persistent kernel use the "nodes / edges"
// form: node_off[g] = nindex_off[g] - g keeps nindex at node_off[g] + g, and
// edge_off[g + 1] - edge_off[g] must give edges[g], so the kernel gets its own
// compact offset arrays built here (one entry per small graph, in queue order).
int batch_enqueue(ecl_batch_ctx* c, const ecl_batch* b, uint8_t* d_inMST, const mst_opts* o,
                  cudaStream_t s, bool timed, ecl_batch_stats* stats) {
  const int G = b->num_graphs;
  const int cutoff = std::min(o->batch_small_edges > 0 ? o->batch_small_edges : c->cap, c->cap);
  std::vector<int> small, large;
  int64_t edges_total = 0;
  for (int g = 0; g < G; g++) {
    const int n = b->nodes[g], m = b->edges[g];
    if (n < 1 || m < 0) return ECL_ERR_INVALID_ARG;
    if (n > c->max_nodes || m > c->max_edges) return ECL_ERR_TOO_LARGE;
    edges_total += m;
    if (m <= cutoff && n <= c->cap) small.push_back(g);
    else large.push_back(g);
  }
  if (!large.empty() && !c->big[0]) return ECL_ERR_TOO_LARGE;
  // largest first: the persistent kernel's tail then consists of small graphs
  std::sort(small.begin(), small.end(), [&](int x, int y) { return b->edges[x] > b->edges[y]; });
  // compact descriptors: small graph i -> (node_off, edge_off) pairs at i, i + 1
  const int S = (int)small.size();
  std::vector<long long> noff(2 * (size_t)S), eoff(2 * (size_t)S);
  std::vector<int> ids(S);
  for (int i = 0; i < S; i++) {
    const int g = small[i];
    noff[2 * i] = b->nindex_off[g] - 2 * (long long)i;     // + id (= 2i) gives nindex_off
    noff[2 * i + 1] = noff[2 * i] + b->nodes[g];
    eoff[2 * i] = b->edge_off[g];
    eoff[2 * i + 1] = b->edge_off[g] + b->edges[g];
    ids[i] = 2 * i;
  }
  ECL_CUDA_TRY(cudaMemsetAsync(c->st, 0, sizeof(DevState), s));
  ECL_CUDA_TRY(cudaMemsetAsync(c->d_queue, 0, sizeof(unsigned), s));
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  if (S > 0) {
    ECL_CUDA_TRY(cudaMemcpyAsync(c->d_node_off, noff.data(), noff.size() * sizeof(long long),
                                 cudaMemcpyHostToDevice, s));
    ECL_CUDA_TRY(cudaMemcpyAsync(c->d_edge_off, eoff.data(), eoff.size() * sizeof(long long),
                                 cudaMemcpyHostToDevice, s));
    ECL_CUDA_TRY(cudaMemcpyAsync(c->d_small, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    BatchArgs ba;
    ba.num_small = S;
    ba.small_list = c->d_small;
    ba.node_off = c->d_node_off;
    ba.edge_off = c->d_edge_off;
    ba.nindex = b->nindex;
    ba.nlist = b->nlist;
    ba.eweight = b->eweight;
    ba.inMST = d_inMST;
    ba.parent_pool = c->parent_pool;
    ba.minv_pool = c->minv_pool;
    ba.wl_pool = c->wl_pool;
    ba.cap_n = c->cap;
    ba.cap_m = c->cap;
    ba.queue = c->d_queue;
    ba.st = c->st;
    ba.mode = o->threshold_mode == ECL_THRESH_LEARNED ? ECL_THRESH_HEURISTIC : o->threshold_mode;
    ba.explicit_thr = o->threshold;
    ba.quantile = o->quantile;
    ba.count_atomics = (o->flags & ECL_FLAG_STATS) ? 1 : 0;
    ba.abl = round_ablation(o->flags);
    const int grid = std::min(c->small_grid, S);
    k_batch_small<<<grid, kThreads, 0, s>>>(ba);
    ECL_CUDA_TRY(cudaGetLastError());
  }
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  bool replayed = false;
  if (!large.empty()) {
    // The large graphs' launch sequence (per graph: control-block reset and
    // six kernels, no host round trip) is captured once per batch layout as a
    // CUDA graph and replayed; if capture is unavailable it is enqueued.
    std::vector<long long> key;
    key.push_back((long long)(uintptr_t)b->nindex);
    key.push_back((long long)(uintptr_t)b->nlist);
    key.push_back((long long)(uintptr_t)b->eweight);
    key.push_back((long long)(uintptr_t)d_inMST);
    key.push_back(o->threshold_mode);
    key.push_back(o->threshold);
    key.push_back((long long)(o->quantile * 1e6f));
    key.push_back(o->degree_split);
    key.push_back(o->small_tail);
    key.push_back(o->flags);
    key.push_back(o->round_min_tiles);
    key.push_back(o->ctas_per_sm);
    key.push_back(o->batch_large_streams);
    key.push_back((long long)ecl_learned_weights_version());
    for (int g : large) {
      key.push_back(g);
      key.push_back(b->nindex_off[g]);
      key.push_back(b->edge_off[g]);
      key.push_back(b->nodes[g]);
      key.push_back(b->edges[g]);
    }
    // The learned schedule runs for the large graphs it serves (as the
    // single-graph solve: at least kLearnedMinEdges entries, weights loaded),
    // its feature pass on the engine's side stream beside k_prep; the others
    // take the reference heuristic.
    mst_opts lo = *o;
    const bool learned = lo.threshold_mode == ECL_THRESH_LEARNED && ecl_learned_has_weights();
    if (lo.threshold_mode == ECL_THRESH_LEARNED && !learned) lo.threshold_mode = ECL_THRESH_HEURISTIC;
    // K concurrent streams, each with its own engine; the graphs go largest
    // first, each to the stream with the fewest entries so far. With several
    // streams the round kernels take one CTA per SM unless ctas_per_sm says
    // otherwise, so the streams' rounds run side by side.
    int K = std::max(1, std::min((int)large.size(), o->batch_large_streams > 0
                                                       ? std::min(o->batch_large_streams, kMaxLargeStreams)
                                                       : kDefaultLargeStreams));
    for (int k = 0; k < K; k++) {
      int r = batch_big_ctx(c, k);
      if (r == ECL_ERR_ALLOC && k > 0) {  // no room for another engine: fewer streams
        cudaGetLastError();
        K = k;
        break;
      }
      if (!r && learned) r = ecl_learned_upload(c->big[k], s);  // before any capture
      if (r) return r;
    }
    if (K > 1 && lo.ctas_per_sm == 0) lo.ctas_per_sm = 1;
    key.push_back(K);  // the streams in use (fewer than asked when memory ran short)
    std::vector<int> order(large);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->edges[x] > b->edges[y]; });
    std::vector<int> lane_of(order.size());
    {
      std::vector<int64_t> load(K, 0);
      for (size_t i = 0; i < order.size(); i++) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        lane_of[i] = k;
        load[k] += b->edges[order[i]];
      }
    }
    auto enqueue_large = [&](cudaStream_t q) -> int {
      if (K > 1) {
        ECL_CUDA_TRY(cudaEventRecord(c->large_fork, q));
        for (int k = 0; k < K; k++) ECL_CUDA_TRY(cudaStreamWaitEvent(c->big[k]->stream, c->large_fork, 0));
      }
      for (size_t i = 0; i < order.size(); i++) {
        const int g = order[i];
        ecl_mst_ctx* e = c->big[lane_of[i]];
        const cudaStream_t sq = K > 1 ? e->stream : q;
        ecl_graph dg = {b->nodes[g], b->edges[g], b->nindex + b->nindex_off[g], b->nlist + b->edge_off[g],
                        b->eweight + b->edge_off[g]};
        ECL_CUDA_TRY(cudaMemsetAsync(e->st, 0, sizeof(DevState), sq));
        mst_opts go = lo;
        LearnedPlan lp{e->side, e->prep_done, e->join, nullptr};
        const LearnedPlan* plan = nullptr;
        if (learned && dg.edges >= kLearnedMinEdges) {
          const int r = learned_fork(e, &dg, sq, &lp);
          if (r) return r;
          plan = &lp;
        } else if (go.threshold_mode == ECL_THRESH_LEARNED) {
          go.threshold_mode = ECL_THRESH_HEURISTIC;
        }
        int r = enqueue_solve(e, &dg, d_inMST + b->edge_off[g], &go, sq, false, plan);
        if (r) return r;
        k_or_error<<<1, 1, 0, sq>>>(e->st, c->st);
        ECL_CUDA_TRY(cudaGetLastError());
      }
      if (K > 1)
        for (int k = 0; k < K; k++) {
          ECL_CUDA_TRY(cudaEventRecord(c->large_join[k], c->big[k]->stream));
          ECL_CUDA_TRY(cudaStreamWaitEvent(q, c->large_join[k], 0));
        }
      return ECL_OK;
    };
    if (c->exec && c->exec_key == key) {
      ECL_CUDA_TRY(cudaGraphLaunch(c->exec, s));
      replayed = true;
    } else {
      if (c->exec) {
        cudaGraphExecDestroy(c->exec);
        c->exec = nullptr;
      }
      cudaGraph_t graph = nullptr;
      bool captured = false;
      if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int r = enqueue_large(s);
        const cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (r == ECL_OK && e == cudaSuccess && graph &&
            cudaGraphInstantiate(&c->exec, graph, 0) == cudaSuccess) {
          captured = true;
          c->exec_key = key;
        }
        if (graph) cudaGraphDestroy(graph);
      }
      cudaGetLastError();  // clear a failed capture's error state
      if (captured) {
        ECL_CUDA_TRY(cudaGraphLaunch(c->exec, s));
        replayed = true;
      } else {
        c->exec = nullptr;
        int r = enqueue_large(s);
        if (r) return r;
      }
    }
  }
  if (timed) ECL_CUDA_TRY(cudaEventRecord(c->ev[2], s));
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->graphs_small = S;
    stats->graphs_large = (int)large.size();
    stats->graph_replay = replayed ? 1 : 0;
    stats->edges_total = edges_total;
  }
  return ECL_OK;
}

int batch_finish(ecl_batch_ctx* c, cudaStream_t s, ecl_batch_stats* stats) {
  ECL_CUDA_TRY(cudaStreamSynchronize(s));
  unsigned err = 0;
  ECL_CUDA_TRY(cudaMemcpy(&err, &c->st->error, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (stats) {
    stats->status = (int32_t)err;
    cudaEventElapsedTime(&stats->ms_small, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&stats->ms_large, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&stats->ms_total, c->ev[0], c->ev[2]);
  }
  return device_error_status(err);
}

}  // namespace

extern "C" int ecl_mst_run_batch_device(ecl_batch_ctx* c, const ecl_batch* b, uint8_t* d_inMST,
                                        const mst_opts* opts, void* stream, ecl_batch_stats* stats) {
  if (!c || !b || !d_inMST || b->num_graphs < 0 || !b->nodes || !b->edges || !b->nindex_off ||
      !b->edge_off || !b->nindex)
    return ECL_ERR_INVALID_ARG;
  if (b->num_graphs > c->max_graphs) return ECL_ERR_TOO_LARGE;
  mst_opts o;
  if (opts) o = *opts;
  else ecl_default_opts(&o);
  int st = check_opts(&o);
  if (st) return st;
  if (o.flags & kDeoptFlags) return ECL_ERR_UNSUPPORTED;  // single-graph contexts only
  ECL_CUDA_TRY(cudaSetDevice(c->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  if ((st = batch_enqueue(c, b, d_inMST, &o, s, stats != nullptr, stats))) return st;
  if (stats) return batch_finish(c, s, stats);
  return ECL_OK;
}

extern "C" int ecl_batch_autotune(ecl_batch_ctx* c, const ecl_batch* b, uint8_t* d_inMST,
                                  const mst_opts* base, mst_opts* best, float* best_ms) {
  if (!c || !b || !best) return ECL_ERR_INVALID_ARG;
  mst_opts o0;
  if (base) o0 = *base;
  else ecl_default_opts(&o0);
  float best_t = 1e30f;
  mst_opts best_o = o0;
  // one candidate: a warm-up run (which also captures), then a timed one
  auto trial = [&](const mst_opts& o) -> int {
    float t = 0.f;
    for (int rep = 0; rep < 2; rep++) {
      ecl_batch_stats bs;
      const int st = ecl_mst_run_batch_device(c, b, d_inMST, &o, nullptr, &bs);
      if (st) return st;
      if (rep > 0) t += bs.ms_total;
    }
    if (t < best_t) {
      best_t = t;
      best_o = o;
    }
    return ECL_OK;
  };
  int st;
  const int cutoffs[] = {c->cap / 8, c->cap / 4, c->cap / 2, c->cap};
  // 1. per-CTA cutoff, scan entries per lane and schedule. The learned
  //    schedule (large graphs only) is kept only where it beats the
  //    reference heuristic on this batch.
  const int modes[] = {o0.threshold_mode, ECL_THRESH_HEURISTIC};
  const int nmodes = o0.threshold_mode == ECL_THRESH_LEARNED ? 2 : 1;
  for (int mi = 0; mi < nmodes; mi++)
    for (int cut : cutoffs) {
      if (cut < 1) continue;
      for (int sp : {8, 16}) {
        mst_opts o = o0;
        o.threshold_mode = modes[mi];
        o.batch_small_edges = cut;
        o.degree_split = sp;
        if ((st = trial(o))) return st;
      }
    }
  // 2. the large graphs' streams and round CTAs per SM, unless *base sets them
  if (best_o.batch_large_streams == 0 && best_o.ctas_per_sm == 0) {
    const mst_opts o1 = best_o;
    for (int k : {1, 2, 4, 8})
      for (int cps : {1, 2}) {
        mst_opts o = o1;
        o.batch_large_streams = k;
        o.ctas_per_sm = cps;
        if ((st = trial(o))) return st;
      }
    // 3. the cutoff again, now that the large graphs run concurrently
    const mst_opts o2 = best_o;
    for (int cut : cutoffs) {
      if (cut < 1 || cut == o2.batch_small_edges) continue;
      mst_opts o = o2;
      o.batch_small_edges = cut;
      if ((st = trial(o))) return st;
    }
  }
  *best = best_o;
  if (best_ms) *best_ms = best_t;
  return ECL_OK;
}
