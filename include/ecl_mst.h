/*
 * ecl_mst.h -- C ABI of the B200 (sm_100a) ECL-MST minimum spanning forest.
 *
 * The ABI replaces one in-file interface of the reference artifact
 * (alexfallin/MST-Artifact-SC23):
 *
 *   ECL-MST/ECLgraph.h:29-35     struct ECLgraph {int nodes, edges; int *nindex, *nlist, *eweight;}
 *   ECL-MST/ECLgraph.h:37-64     ECLgraph readECLgraph(const char*)
 *   ECL-MST/ECLgraph.h:66-80     void writeECLgraph(const ECLgraph, const char*)
 *   ECL-MST/ECLgraph.h:82-90     void freeECLgraph(ECLgraph&)
 *   ECL-MST/ECL_MST.cu:265-362   template<bool filter> bool* gpuMST(const ECLgraph&, int threshold)
 *   ECL-MST/ECL_MST.cu:389-395,
 *                      :432-444  threshold heuristic (20 hashed samples, "300% of nodes")
 *   ECL-MST/ECL_MST.cu:410-419   weight synthesis for weightless inputs
 *   ECL-MST/ECL_MST.cu:365-386   verify()
 *
 * Differences in behaviour, all deliberate:
 *   - nothing here calls exit(); every entry point returns an ecl_status code;
 *   - the caller owns every buffer (inMST is caller-allocated, m bytes);
 *   - malformed CSR content (nindex not monotone, neighbour ids out of range) is
 *     reported as ECL_ERR_FORMAT instead of reading out of bounds.
 *
 * Output contract (identical to the reference GPU path): inMST[j] == 1 iff the
 * CSR entry j = (v -> nlist[j]) with nlist[j] > v is an edge of the minimum
 * spanning forest under the strict order (uint32(eweight[j]), j); all other
 * entries, including the reverse direction of every forest edge, are 0.
 */
#ifndef ECL_MST_B200_H
#define ECL_MST_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum ecl_status {
  ECL_OK = 0,
  ECL_ERR_INVALID_ARG = -1, /* NULL pointer, nodes < 1, edges < 0, bad option   */
  ECL_ERR_IO = -2,          /* file could not be opened / read / written        */
  ECL_ERR_FORMAT = -3,      /* truncated file or inconsistent CSR content        */
  ECL_ERR_ALLOC = -4,       /* host or device allocation failed                 */
  ECL_ERR_CUDA = -5,        /* a CUDA runtime call failed                        */
  ECL_ERR_NO_DEVICE = -6,   /* no CUDA device is visible                         */
  ECL_ERR_OVERFLOW = -7,    /* a worklist or batch exceeded its capacity        */
  ECL_ERR_TIMEOUT = -8,     /* a device-side wait hit its limit (no hang)        */
  ECL_ERR_TOO_LARGE = -9,   /* input beyond a stated maximum                     */
  ECL_ERR_UNSUPPORTED = -10 /* option not supported by the library or device    */
} ecl_status;

/* Human-readable name of a status code (static string). */
const char* ecl_status_string(int status);

/* ------------------------------------------------------------------ graph */
/* Byte-for-byte the reference ECLgraph (ECLgraph.h:29-35). The arrays are
 * host pointers for the host entry points and device pointers for the
 * *_device entry points. eweight may be NULL (weightless file). */
typedef struct ecl_graph {
  int32_t nodes;
  int32_t edges;
  int32_t* nindex; /* nodes + 1 */
  int32_t* nlist;  /* edges     */
  int32_t* eweight;/* edges, or NULL */
} ecl_graph;

/* Read a binary ECLgraph file (replaces readECLgraph, ECLgraph.h:37-64).
 * Layout: int32 nodes, int32 edges, int32 nindex[nodes+1], int32 nlist[edges],
 * optionally int32 eweight[edges]. A file that ends right after nlist yields
 * eweight == NULL, as in the reference. Arrays are malloc'd; free them with
 * ecl_free_graph. */
int ecl_read_graph(const char* path, ecl_graph* out);

/* Write a binary ECLgraph file (replaces writeECLgraph, ECLgraph.h:66-80). */
int ecl_write_graph(const ecl_graph* g, const char* path);

/* Free arrays allocated by ecl_read_graph / ecl_gen_* (replaces freeECLgraph,
 * ECLgraph.h:82-90). Sets the pointers to NULL. */
void ecl_free_graph(ecl_graph* g);

/* Weights for a weightless graph, bit-exact with ECL_MST.cu:410-419:
 * eweight[j] = |1 + (int32 wrap(v * nlist[j]) % nodes)| for j in row v.
 * g->eweight must point to a caller-allocated array of g->edges ints. */
int ecl_synthesize_weights(ecl_graph* g);

/* Check CSR consistency on the host: nindex[0] == 0, nindex monotone,
 * nindex[nodes] == edges, 0 <= nlist[j] < nodes. Returns ECL_OK or
 * ECL_ERR_FORMAT. */
int ecl_validate_graph(const ecl_graph* g);

/* ---------------------------------------------------------- synthetic inputs */
/* Seeded, deterministic generators. Every graph is deduplicated, free of
 * self-loops, symmetric, with rows sorted by neighbour id, and each undirected
 * edge {u,v} carries one weight drawn uniformly from [1, wmax] from a hash of
 * (seed, min(u,v), max(u,v)) and mirrored to both directions. Arrays are
 * malloc'd (free with ecl_free_graph). threads <= 0 means all host cores. */
int ecl_gen_grid(int32_t rows, int32_t cols, uint64_t seed, int32_t wmax,
                 int threads, ecl_graph* out);
int ecl_gen_er(int32_t nodes, double avg_degree, uint64_t seed, int32_t wmax,
               int threads, ecl_graph* out);
int ecl_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b,
                 double c, uint64_t seed, int32_t wmax, int threads,
                 ecl_graph* out);
int ecl_gen_rgg2d(int32_t nodes, double avg_degree, uint64_t seed,
                  int32_t wmax, int threads, ecl_graph* out);

/* Graph `index` of the mixed-family batch: seed seed0 + index, family uniform
 * over {2D grid, Erdos-Renyi avg degree 8, RMAT (.57,.19,.19) edge factor 8,
 * random geometric 2D avg degree 3}, vertex count log-uniform in
 * [nmin, nmax]; *family receives 0..3 in that order. Single-threaded. */
int ecl_gen_batch_graph(int32_t index, uint64_t seed0, int32_t nmin, int32_t nmax,
                        int32_t wmax, ecl_graph* out, int32_t* family);

/* ------------------------------------------------ GPU-side preprocessing */
/* The reference builds and converts its inputs on the host
 * (Inputs/download_inputs.sh, PBBS_CPU/inputs/ecl2pbbs_genweights.cpp:14-41,
 * cuGraph_GPU/inputs/ecl2mtx_genweights_cugraph.cpp:16-50). These build them
 * on the device. Every call is synchronous; on success the ecl_graph holds
 * DEVICE arrays from cudaMalloc, freed with ecl_free_device_graph. */

/* Weight of each CSR entry built by ecl_csr_from_pairs_device. */
typedef enum ecl_weight_rule {
  ECL_WEIGHTS_GIVEN = 0, /* d_w[i] of the pair; duplicates of an undirected
                            pair keep the smallest as uint32 (the MST order) */
  ECL_WEIGHTS_HASH = 1,  /* the generators' rule: uniform in [1, wmax] from a
                            hash of (seed, min(u,v), max(u,v))               */
  ECL_WEIGHTS_SYNTH = 2  /* the reference's weight for weightless inputs,
                            1 + ((u*v) % nodes) made non-negative
                            (ECL_MST.cu:410-419)                            */
} ecl_weight_rule;

/* Symmetric, deduplicated, self-loop-free CSR with rows sorted by neighbour
 * id, from `pairs` undirected pairs (d_u[i], d_v[i]) in DEVICE memory (either
 * orientation; duplicates and self-loops allowed). An id outside
 * [0, nodes) gives ECL_ERR_FORMAT; 2 * pairs > INT32_MAX gives
 * ECL_ERR_TOO_LARGE. stream NULL = the default stream. */
int ecl_csr_from_pairs_device(int32_t nodes, int64_t pairs, const int32_t* d_u,
                              const int32_t* d_v, const int32_t* d_w,
                              int32_t weight_rule, uint64_t seed, int32_t wmax,
                              void* stream, ecl_graph* out);

/* The synthetic families drawn on the device: for equal arguments the result
 * equals the host generator's (ecl_gen_grid, ...) entry for entry. */
int ecl_gen_grid_device(int32_t rows, int32_t cols, uint64_t seed, int32_t wmax,
                        void* stream, ecl_graph* out);
int ecl_gen_er_device(int32_t nodes, double avg_degree, uint64_t seed,
                      int32_t wmax, void* stream, ecl_graph* out);
int ecl_gen_rmat_device(int32_t scale, int32_t edge_factor, double a, double b,
                        double c, uint64_t seed, int32_t wmax, void* stream,
                        ecl_graph* out);
int ecl_gen_rgg2d_device(int32_t nodes, double avg_degree, uint64_t seed,
                         int32_t wmax, void* stream, ecl_graph* out);
int ecl_gen_batch_graph_device(int32_t index, uint64_t seed0, int32_t nmin,
                               int32_t nmax, int32_t wmax, void* stream,
                               ecl_graph* out, int32_t* family);
void ecl_free_device_graph(ecl_graph* g);

/* Copy a device graph into malloc'd host arrays (free with ecl_free_graph). */
int ecl_graph_to_host(const ecl_graph* d_graph, ecl_graph* out);

/* ------------------------------------------------------------- exporters */
/* Text formats of the reference's converters, byte for byte. Weightless
 * graphs (eweight NULL) get the ECL_WEIGHTS_SYNTH weights, as there.
 *   PBBS WeightedEdgeArray: every CSR entry as "src dst weight" with the
 *     weight printed as float with %f (ecl2pbbs_genweights.cpp:34-41);
 *   MatrixMarket coordinate real symmetric: the entries with src > dst,
 *     1-based, weight with %.1f (ecl2mtx_genweights_cugraph.cpp:37-50). */
int ecl_write_pbbs(const ecl_graph* g, const char* path);
int ecl_write_mtx(const ecl_graph* g, const char* path);

/* ------------------------------------------------------------- threshold */
typedef enum ecl_threshold_mode {
  ECL_THRESH_HEURISTIC = 0, /* the reference rule (ECL_MST.cu:408,432-444)      */
  ECL_THRESH_NONE = 1,      /* single unfiltered phase (gpuMST<false>, INT_MAX) */
  ECL_THRESH_EXPLICIT = 2,  /* opts.threshold                                   */
  ECL_THRESH_QUANTILE = 3,  /* opts.quantile of a 4096-entry weight sample      */
  ECL_THRESH_LEARNED = 4    /* quantile + split predicted by the trained MLP     */
} ecl_threshold_mode;

/* The reference threshold heuristic on host arrays. *filtered = 1 iff
 * edges/nodes >= 4 (integer division); the threshold is then the
 * min(19, int(3.0*nodes*20/edges))-th smallest of 20 weights sampled at
 * hash(i) % edges. *filtered = 0 gives threshold INT32_MAX. */
int ecl_heuristic_threshold(const ecl_graph* g, int32_t* threshold,
                            int32_t* filtered);

/* --------------------------------------------------------------- options */
enum {
  ECL_FLAG_L2_PERSIST = 1 << 0, /* L2 access-policy window on parent/min slots
                                   (opt-in: measured 6 % slower on RMAT-22, the
                                   set-aside takes L2 from the heavy scan)      */
  ECL_FLAG_STATS = 1 << 1,      /* count guarded atomics (slower; off in timing) */
  ECL_FLAG_NO_SMALL_TAIL = 1 << 2, /* keep every round grid-wide (ablation)     */
  /* Ablation switches: each turns one technique of the round kernel off, to
   * measure what it buys (the answer is unchanged). NO_GUARDS is the
   * reference's NoAtomicGuards variant (Deoptimizations/
   * ECL_MST_NoAtomicGuards.cu:222-223); NO_WARP_COOP stands for its NoWarp
   * variant, applied to this engine's warp/CTA cooperation on shared reps. */
  ECL_FLAG_NO_GUARDS = 1 << 3,     /* atomicMin without reading the slot first  */
  ECL_FLAG_NO_WARP_COOP = 1 << 4,  /* no warp reduction / CTA table for shared reps */
  ECL_FLAG_DEDUP = 1 << 5,         /* per-tile parallel-edge elimination in the
                                      rounds (off by default: on RMAT it costs
                                      more than the smaller worklists save)     */
  ECL_FLAG_NO_FIND_CACHE = 1 << 6, /* no per-CTA root cache in the finds        */
  /* A solve repeated with identical arguments is captured as a CUDA graph on
   * the first repeat and replayed as one launch after that; a replayed
   * solve's stats carry ms_total only. NO_GRAPH keeps direct launches (and
   * the per-phase timings). */
  ECL_FLAG_NO_GRAPH = 1 << 7,
  /* The reference's later deoptimization steps (Deoptimizations/, the
   * ablation of generate_deoptimize_tables.py:6-14), restated so that the
   * forest is unchanged: one direction is kept (the reference's
   * NoOneDirection step marks the reverse entry instead and is not
   * reproduced). Single-graph contexts only; the batched and the
   * allocation-free entry points return ECL_ERR_UNSUPPORTED for them. */
  ECL_FLAG_NO_IMPLICIT_COMPRESSION = 1 << 8, /* compacted entries keep their
                                      endpoints; finds split paths from the
                                      first step; the mark pass finds again
                                      (..._NoImplicitPathCompression.cu:121-133,
                                      193-216)                                */
  ECL_FLAG_NO_TUPLES = 1 << 9,     /* worklists hold CSR indices; endpoints and
                                      weights are gathered every round through
                                      a per-entry vertex list (..._NoTuples.cu;
                                      implies NO_IMPLICIT_COMPRESSION; the
                                      context allocates the list on first use) */
  ECL_FLAG_NO_DATA_DRIVEN = 1 << 10, /* topology-driven: every round reads the
                                      phase's whole list, nothing is compacted
                                      (..._NoDataDriven.cu:166-180, 263-270;
                                      implies NO_IMPLICIT_COMPRESSION)         */
  ECL_FLAG_NO_EDGE_BASED = 1 << 11 /* vertex-centric rounds over the CSR, one
                                      thread per vertex, no worklists
                                      (..._NoEdgeBased.cu:152-195)             */
};

typedef struct mst_opts {
  int32_t threshold_mode; /* ecl_threshold_mode                              */
  int32_t threshold;      /* ECL_THRESH_EXPLICIT: edges with w <= threshold    */
                          /* form the first (light) phase                      */
  float quantile;         /* ECL_THRESH_QUANTILE, in [0,1]; >= 1 disables      */
  int32_t degree_split;   /* thread/cooperative split of the light CSR scan:   */
                          /* each thread takes E consecutive entries, E = 4    */
                          /* for split <= 4, 8 for split <= 8, else 16; rows   */
                          /* shorter than E stay in one thread, longer rows    */
                          /* are spread over threads/warps; 0 = default (8).   */
                          /* The heavy scan always takes E = 4                 */
  int32_t round_min_tiles; /* the round kernel keeps one CTA per this many   */
                          /* 512-entry tiles of a round's worklist: CTAs       */
                          /* beyond it leave the launch as the rounds shrink,  */
                          /* and its grid barriers wait for the rest only;     */
                          /* 0 = default (1), < 0 = keep every CTA             */
  int32_t ctas_per_sm;    /* round-kernel CTAs per SM, 0 = as many as fit      */
  int32_t small_tail;     /* worklist size at which one CTA finishes the      */
                          /* rounds alone; 0 = default, < 0 = never            */
  int32_t flags;          /* ECL_FLAG_*                                        */
  int32_t batch_small_edges; /* batched mode: graphs with at most this many   */
                          /* CSR entries (and fitting the per-CTA scratch) are */
                          /* solved one per CTA by the persistent kernel;      */
                          /* 0 = the context's per-CTA capacity                */
  int32_t batch_large_streams; /* batched mode: the other graphs are solved on */
                          /* this many concurrent streams (1..8), each with    */
                          /* its own workspace, largest graph first to the     */
                          /* least-loaded stream; with more than one, their    */
                          /* round kernels take one CTA per SM unless          */
                          /* ctas_per_sm is set; 0 = default (4); fewer when   */
                          /* the device has no room for another workspace      */
  int32_t reserved[6];
} mst_opts;

/* Fill *opts with the defaults (heuristic threshold, reference semantics). */
void ecl_default_opts(mst_opts* opts);

/* Per-run counters, filled when a stats pointer is passed. */
#define ECL_MAX_ROUNDS 64
typedef struct ecl_mst_stats {
  int32_t threshold;       /* threshold used (INT32_MAX when unfiltered)        */
  int32_t filtered;        /* 1 if two phases ran                               */
  int32_t degree_split;    /* split used by the light scan                      */
  int32_t rounds[2];       /* Boruvka rounds of the light / heavy phase         */
  int32_t status;          /* device error word (0 = clean)                     */
  int64_t scan_kept[2];    /* worklist entries appended by each scan            */
  int64_t wl_in[2][ECL_MAX_ROUNDS];  /* worklist slots entering each round (the
                                        first also holds null padding)       */
  int64_t atomics;         /* guarded atomicMin issued (ECL_FLAG_STATS only)    */
  int64_t forest_edges;    /* number of inMST entries set                       */
  uint64_t forest_weight;  /* sum of eweight over inMST (as verify(), :377)     */
  float ms_total;          /* device time of the whole solve (CUDA events),
                              the learned schedule's feature pass included      */
  float ms_rounds;         /* device time of the round kernels                  */
  float ms_scan;           /* device time of everything else (scans, prep,
                              features, flatten)                                */
  /* breakdown (microseconds); us_scan from CUDA events, us_round from the
   * device clock at the round kernel's barriers:                            */
  float us_scan[2][3];     /* [0]: {features + prep + light scan, features +
                              prep, light scan kernel}; [1]: {flatten + heavy
                              scan, flatten, heavy scan kernel}                */
  float us_round[2][ECL_MAX_ROUNDS][2]; /* per round: find/min pass, mark pass  */
  int64_t wl_real[2][ECL_MAX_ROUNDS];   /* entries entering each round without
                                           the scans' null padding            */
} ecl_mst_stats;

/* ------------------------------------------------------------- the solve */
/* One-shot drop-in for gpuMST (ECL_MST.cu:265-362) plus the heuristic choice
 * of main (:432-444): host CSR in, caller-allocated host inMST (edges bytes)
 * out. Allocates and frees its own device workspace on the current device.
 * opts == NULL means ecl_default_opts. stats may be NULL. */
int ecl_mst_run(const ecl_graph* g, uint8_t* inMST, const mst_opts* opts,
                ecl_mst_stats* stats);

/* Reusable device workspace, sized for graphs up to (max_nodes, max_edges).
 * Creating it allocates; runs through it allocate nothing. */
typedef struct ecl_mst_ctx ecl_mst_ctx;
int ecl_mst_ctx_create(int device, int64_t max_nodes, int64_t max_edges,
                       ecl_mst_ctx** out);
void ecl_mst_ctx_destroy(ecl_mst_ctx* ctx);

/* Host CSR in, host inMST out, through the context's device buffers and the
 * context's stream: H2D copies, the solve and the D2H copy of inMST. */
int ecl_mst_ctx_run_host(ecl_mst_ctx* ctx, const ecl_graph* g, uint8_t* inMST,
                         const mst_opts* opts, ecl_mst_stats* stats);

/* Pipelined host-buffer solves, for a stream of graphs: each call enqueues
 * the copy in of g's arrays, the solve and the copy back of inMST, and
 * returns; ecl_mst_ctx_wait waits for every call since the last wait and
 * reports their device errors. Consecutive calls overlap: a graph's copy in
 * runs beside the previous graph's solve and copy back (two device buffer
 * sets used in turn, a copy-in and a copy-out stream beside the context's).
 * g's arrays and inMST must stay valid until the wait, and pinned host
 * memory (ecl_host_alloc_pinned) keeps the copies asynchronous. Call
 * ecl_mst_ctx_wait before any other solve on the context. An input with
 * more one-direction entries than edges/2 is solved again inside the wait,
 * with grown worklists. No counterpart in the reference, which solves one
 * graph per process run. */
int ecl_mst_ctx_run_host_async(ecl_mst_ctx* ctx, const ecl_graph* g,
                               uint8_t* inMST, const mst_opts* opts);
int ecl_mst_ctx_wait(ecl_mst_ctx* ctx);

/* Device-resident solve: d_graph holds DEVICE pointers, d_inMST is a device
 * buffer of edges bytes. Enqueued on `stream` (cudaStream_t, NULL = the
 * context's stream); returns after enqueueing unless stats != NULL, in which
 * case it synchronises and fills stats. Errors found on the device are
 * returned by ecl_mst_ctx_sync.
 * A context's worklists start at the size a symmetric input needs (edges/2
 * one-direction entries nlist[j] > v, as the reference sizes them,
 * ECL_MST.cu:279, plus slack). An input with more one-direction entries
 * overflows them; the library then grows them to hold every CSR entry and
 * solves again, inside this call when stats != NULL, else inside
 * ecl_mst_ctx_sync, which must therefore be called before inMST is read
 * when the input may not be symmetric. */
int ecl_mst_run_device(ecl_mst_ctx* ctx, const ecl_graph* d_graph,
                       uint8_t* d_inMST, const mst_opts* opts, void* stream,
                       ecl_mst_stats* stats);

/* Allocation-free device solve. This entry point has no counterpart in the
 * reference; it exists for callers that must not allocate device memory
 * (code running inside an allocator or memory-pool callback, embeddings that
 * own every allocation of the process, services with a device-memory budget
 * fixed at start-up). It calls no cudaMalloc, cudaFree or allocating library
 * routine: its scratch is one file-scope device array of about 21 MB that
 * every GPU loading this library holds until the process exits.
 *   - d_graph holds DEVICE pointers, d_inMST a device buffer of edges bytes;
 *   - limits: nodes <= 262,144 and edges <= 1,048,576, else ECL_ERR_TOO_LARGE;
 *     the worklists hold 524,288 entries, enough for every symmetric input
 *     (at most edges/2 one-direction entries nlist[j] > v); an input with
 *     more one-direction entries than that returns ECL_ERR_OVERFLOW;
 *   - ECL_THRESH_LEARNED takes the reference heuristic here, as
 *     ecl_mst_run_device does for graphs below its learned-schedule cut-off
 *     (the feature pass needs scratch this entry point does not hold);
 *   - every call looks up the scratch array's address on the current device
 *     (a device reset reloads the module that owns it); the first call on a
 *     device also reads its attributes, so make it before any stream
 *     capture; the call enqueues on `stream`
 *     (cudaStream_t, NULL = legacy default stream) and returns after the solve
 *     finished, with device-side errors as its status;
 *   - all calls share the one scratch array: calls that overlap on the GPU
 *     (other threads, other streams) race and give wrong results. */
int ecl_mst_run_device_noalloc(const ecl_graph* d_graph, uint8_t* d_inMST,
                               const mst_opts* opts, void* stream);

/* ------------------------------------------------------------- batched mode */
/* Many independent graphs in one call. Graph g has nodes[g] vertices and
 * edges[g] CSR entries; its nindex (nodes[g] + 1 local offsets) starts at
 * nindex[nindex_off[g]], its local neighbour ids and weights at
 * nlist[edge_off[g]] / eweight[edge_off[g]], and its inMST flags are written
 * at inMST[edge_off[g]]. nodes/edges/nindex_off/edge_off are HOST arrays,
 * nindex/nlist/eweight DEVICE arrays. Segments may be padded (offsets that
 * are multiples of 4 entries keep 128-bit loads aligned). Each graph gets the
 * reference treatment (its own threshold per opts, its own rounds), with
 * results identical to solving it alone. */
typedef struct ecl_batch {
  int32_t num_graphs;
  const int32_t* nodes;
  const int32_t* edges;
  const int64_t* nindex_off;
  const int64_t* edge_off;
  int32_t* nindex;
  int32_t* nlist;
  int32_t* eweight;
} ecl_batch;

typedef struct ecl_batch_stats {
  int32_t graphs_small;  /* solved one per CTA in the persistent launch */
  int32_t graphs_large;  /* solved by the grid-wide engine                */
  int32_t status;        /* device error word                             */
  int32_t graph_replay;  /* 1 if the large graphs ran from a CUDA graph     */
  int64_t edges_total;
  float ms_total, ms_small, ms_large;
} ecl_batch_stats;

typedef struct ecl_batch_ctx ecl_batch_ctx;

/* Workspace for batches of up to max_graphs graphs, none larger than
 * (max_graph_nodes, max_graph_edges). small_cap sizes the per-CTA scratch of
 * the persistent kernel (vertices and entries of the largest graph it may
 * take; 0 = 2^19). */
int ecl_batch_ctx_create(int device, int32_t max_graphs, int64_t max_graph_nodes,
                         int64_t max_graph_edges, int32_t small_cap,
                         ecl_batch_ctx** out);
void ecl_batch_ctx_destroy(ecl_batch_ctx* ctx);

/* Solve every graph of the batch (device-resident, on `stream` or the
 * context's stream). Returns after completion when stats != NULL. */
int ecl_mst_run_batch_device(ecl_batch_ctx* ctx, const ecl_batch* batch,
                             uint8_t* d_inMST, const mst_opts* opts, void* stream,
                             ecl_batch_stats* stats);

/* Autotuner: times candidate schedules (per-CTA cutoff, scan entries per
 * thread and, when *base asks for the learned schedule, learned against the
 * reference heuristic for the large graphs; then, unless *base sets them,
 * the large graphs' streams and round-kernel CTAs per SM, and the cutoff
 * again with those) on the batch and
 * writes the fastest into *best (a copy of *base with those fields set).
 * The answer is the same for every candidate; only the time differs. */
int ecl_batch_autotune(ecl_batch_ctx* ctx, const ecl_batch* batch, uint8_t* d_inMST,
                       const mst_opts* base, mst_opts* best, float* best_ms);

/* The first `count` graphs of the mixed batch (ecl_gen_batch_graph's
 * sequence), drawn on the device and packed into one ecl_batch whose segments
 * start at multiples of `align` entries (nindex: nodes + 1 entries per graph,
 * nlist/eweight: max(edges, 1)). Graph g's inMST segment of a solve is
 * [edge_off[g], edge_off[g] + edges[g]); the packed length is
 * edge_off[count-1] + round_up(max(edges[count-1], 1), align). The host arrays
 * are malloc'd, the device arrays cudaMalloc'd; free both with
 * ecl_free_device_batch. family (count entries) may be NULL. Synchronous. */
int ecl_gen_batch_device(int32_t count, uint64_t seed0, int32_t nmin, int32_t nmax,
                         int32_t wmax, int32_t align, void* stream, ecl_batch* out,
                         int32_t* family);
void ecl_free_device_batch(ecl_batch* b);

/* ---------------------------------------------------- learned schedule */
/* A 16 -> 64 -> 64 -> 2 ReLU MLP (fp32) maps 16 graph features to the light-
 * phase filter quantile (output 0: log2 q minus the log2 of the reference
 * heuristic's quantile, (idx+1)/21 or 1 when it does not filter; a total
 * >= 0 means no filter) and the scans' degree split (output 1, log2 split). It changes the schedule only.
 * Parameter blob (ECL_MLP_PARAMS floats): W1[16][64], b1[64], W2[64][64],
 * b2[64], W3[64][2], b3[2], feature mean[16], feature std[16]. */
#define ECL_MLP_INPUTS 16
#define ECL_MLP_HIDDEN 64
#define ECL_MLP_OUTPUTS 2
#define ECL_MLP_PARAMS 5410

/* Load the weights used by ECL_THRESH_LEARNED (process-wide). Without
 * weights, ECL_THRESH_LEARNED falls back to the reference heuristic. */
int ecl_learned_set_weights(const float* params, int count);
int ecl_learned_has_weights(void);

/* The 16 features of a device-resident graph (computed on the device):
 * log2 n, log2 m, log2(avg degree + 1), log2(max degree + 1), degree CV,
 * fractions of vertices with degree 0, < 4, >= 32, 3n/m, and the 1, 2, 5,
 * 10, 20, 30, 50 % quantiles of a 4096-entry weight sample over its max. */
int ecl_graph_features(const ecl_graph* d_graph, float* out16);

/* MLP kernels on the current device, host buffers in and out:
 * forward (B samples of raw features -> B x 2 outputs), full-batch
 * mean-squared-error gradient of W1..b3 (5378 floats; inputs already
 * standardised), and a whole Adam training run in one launch (minibatches of
 * 64 standardised samples, in the given order; params updated in place;
 * loss_hist gets one mean loss per epoch). */
int ecl_mlp_forward(const float* params, const float* x, int B, float* y);
int ecl_mlp_grad(const float* params, const float* x, const float* t, int B,
                 float* grad, float* loss);
int ecl_mlp_train(float* params, const float* x, const float* t, int B,
                  int epochs, float lr, float* loss_hist);

/* Wait for the context's stream and report a device-side error if any. */
int ecl_mst_ctx_sync(ecl_mst_ctx* ctx);

/* The stream the context enqueues on (a cudaStream_t). */
void* ecl_mst_ctx_stream(ecl_mst_ctx* ctx);

/* Returns every L2 line a solve with ECL_FLAG_L2_PERSIST marked persisting to
 * normal status (cudaCtxResetPersistingL2Cache on the context's device), so
 * later traffic can evict them. No counterpart in the reference, which sets
 * no L2 policy. */
int ecl_mst_ctx_l2_reset(ecl_mst_ctx* ctx);

/* The 16 features the last learned-schedule solve on this context fed its
 * network (the degree statistics k_prep gathered and the sorted weight
 * sample), copied to host out16 after the context's streams finish; they
 * equal ecl_graph_features() of the same graph. ECL_ERR_UNSUPPORTED before
 * any learned solve on the context. No counterpart in the reference. */
int ecl_mst_ctx_learned_features(ecl_mst_ctx* ctx, float* out16);

/* Pinned host memory for fast H2D/D2H (cudaHostAlloc / cudaFreeHost). */
int ecl_host_alloc_pinned(size_t bytes, void** out);
void ecl_host_free_pinned(void* p);

/* ---------------------------------------------------------------- verify */
/* Restates verify() (ECL_MST.cu:365-386): per-entry comparison of two inMST
 * arrays and their uint64 forest weights. Returns 1 if they agree (no entry in
 * only one of them and equal weights), 0 otherwise; counts may be NULL
 * (4 int64: both, neither, only_a, only_b). */
int ecl_verify(const ecl_graph* g, const uint8_t* a, const uint8_t* b,
               int64_t counts[4], uint64_t* weight_a, uint64_t* weight_b);

/* uint64 sum of eweight over set inMST entries (as verify(), :377-378). */
uint64_t ecl_forest_weight(const ecl_graph* g, const uint8_t* inMST);

/* Library version string. */
const char* ecl_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ECL_MST_B200_H */
