/*
 * ORACLE -- test infrastructure only. Nothing in the product library links,
 * loads or calls this file.
 *
 * Draws the benchmark's seeded synthetic inputs on the host: the 2D grid, the
 * Erdos-Renyi and the RMAT graphs, as symmetric, deduplicated, self-loop-free
 * CSRs with rows sorted by neighbour id and one weight per undirected edge.
 * The random stream (splitmix64 finalizer over a counter), the RMAT quadrant
 * cut-offs in 16-bit fixed point and the per-pair weight rule are restated
 * from the product's generator description (mst-artifact-sc23_b200/csrc/
 * generators.cpp, internal.h) so that both draw the same graph for a seed.
 *
 * Purpose: the benchmark's reference arm (bench.py --impl reference) times
 * the reference's cpuMST (ECL-MST/ECL_MST.cu:82-124) on exactly the graph the
 * GPU arm solves, and builds that graph here so that the reference process
 * loads none of the product's libraries. tests/test_oracle.py checks these
 * generators entry for entry against the product's.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define GG_STREAM_WEIGHT 1
#define GG_STREAM_RMAT 2
#define GG_STREAM_ER 3

static uint64_t gg_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

static uint64_t gg_rng(uint64_t seed, uint64_t stream, uint64_t idx) {
  return gg_mix(gg_mix(seed * 0x9E3779B97F4A7C15ULL + stream) ^ (idx * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL));
}

static int32_t gg_weight(uint64_t seed, uint32_t u, uint32_t v, int32_t wmax) {
  const uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
  const uint64_t r = gg_rng(seed, GG_STREAM_WEIGHT, ((uint64_t)lo << 32) | hi);
  return 1 + (int32_t)(r % (uint64_t)(wmax < 1 ? 1 : wmax));
}

static uint32_t gg_below(uint32_t bits, uint32_t n) { return (uint32_t)(((uint64_t)bits * n) >> 32); }

/* ---- a small work-sharing pool: body(lo, hi, arg) over [0, n) in chunks */
typedef void (*gg_body)(int64_t lo, int64_t hi, void* arg);
typedef struct {
  gg_body body;
  void* arg;
  int64_t n, chunk;
  int64_t next; /* shared, taken with atomic fetch-add */
} gg_job;

static void* gg_worker(void* p) {
  gg_job* j = (gg_job*)p;
  for (;;) {
    const int64_t lo = __atomic_fetch_add(&j->next, j->chunk, __ATOMIC_RELAXED);
    if (lo >= j->n) break;
    const int64_t hi = lo + j->chunk < j->n ? lo + j->chunk : j->n;
    j->body(lo, hi, j->arg);
  }
  return NULL;
}

static int gg_threads(void) {
  const long c = sysconf(_SC_NPROCESSORS_ONLN);
  return c < 1 ? 1 : (c > 64 ? 64 : (int)c);
}

static void gg_parallel(int64_t n, int64_t chunk, gg_body body, void* arg) {
  if (n <= 0) return;
  gg_job j = {body, arg, n, chunk < 1 ? 1 : chunk, 0};
  int t = gg_threads();
  if (t > n / j.chunk + 1) t = (int)(n / j.chunk + 1);
  pthread_t th[64];
  int started = 0;
  for (int i = 1; i < t; i++)
    if (pthread_create(&th[started], NULL, gg_worker, &j) == 0) started++;
  gg_worker(&j);
  for (int i = 0; i < started; i++) pthread_join(th[i], NULL);
}

/* ---- CSR from an undirected pair list (u << 32 | v) */
typedef struct {
  const uint64_t* pairs;
  int64_t* deg; /* atomic counters, then cursors */
  uint32_t* adj;
  const int64_t* off;
  int64_t* uniq;
  int32_t *nindex, *nlist, *eweight;
  uint64_t seed;
  int32_t wmax;
} gg_csr;

static void gg_count(int64_t lo, int64_t hi, void* a) {
  gg_csr* c = (gg_csr*)a;
  for (int64_t i = lo; i < hi; i++) {
    const uint32_t u = (uint32_t)(c->pairs[i] >> 32), v = (uint32_t)c->pairs[i];
    if (u == v) continue;
    __atomic_fetch_add(&c->deg[u], 1, __ATOMIC_RELAXED);
    __atomic_fetch_add(&c->deg[v], 1, __ATOMIC_RELAXED);
  }
}

static void gg_fill(int64_t lo, int64_t hi, void* a) {
  gg_csr* c = (gg_csr*)a;
  for (int64_t i = lo; i < hi; i++) {
    const uint32_t u = (uint32_t)(c->pairs[i] >> 32), v = (uint32_t)c->pairs[i];
    if (u == v) continue;
    c->adj[__atomic_fetch_add(&c->deg[u], 1, __ATOMIC_RELAXED)] = v;
    c->adj[__atomic_fetch_add(&c->deg[v], 1, __ATOMIC_RELAXED)] = u;
  }
}

static int gg_cmp_u32(const void* x, const void* y) {
  const uint32_t a = *(const uint32_t*)x, b = *(const uint32_t*)y;
  return (a > b) - (a < b);
}

static void gg_sort_rows(int64_t lo, int64_t hi, void* a) {
  gg_csr* c = (gg_csr*)a;
  for (int64_t v = lo; v < hi; v++) {
    uint32_t* r = c->adj + c->off[v];
    const int64_t d = c->off[v + 1] - c->off[v];
    if (d < 24) {
      for (int64_t i = 1; i < d; i++) {
        const uint32_t x = r[i];
        int64_t k = i - 1;
        while (k >= 0 && r[k] > x) {
          r[k + 1] = r[k];
          k--;
        }
        r[k + 1] = x;
      }
    } else {
      qsort(r, (size_t)d, sizeof(uint32_t), gg_cmp_u32);
    }
    int64_t u = 0;
    for (int64_t i = 0; i < d; i++)
      if (u == 0 || r[i] != r[u - 1]) r[u++] = r[i];
    c->uniq[v] = u;
  }
}

static void gg_emit(int64_t lo, int64_t hi, void* a) {
  gg_csr* c = (gg_csr*)a;
  for (int64_t v = lo; v < hi; v++) {
    const int32_t base = c->nindex[v];
    for (int64_t k = 0; k < c->uniq[v]; k++) {
      const uint32_t w = c->adj[c->off[v] + k];
      c->nlist[base + k] = (int32_t)w;
      c->eweight[base + k] = gg_weight(c->seed, (uint32_t)v, w, c->wmax);
    }
  }
}

/* Allocated with malloc; the caller frees with gg_free. Returns 0, -1 bad
 * input, -4 allocation failure, -9 too large. */
typedef struct {
  int32_t nodes, edges;
  int32_t *nindex, *nlist, *eweight;
} gg_graph;

void gg_free(gg_graph* g) {
  if (!g) return;
  free(g->nindex);
  free(g->nlist);
  free(g->eweight);
  memset(g, 0, sizeof(*g));
}

static int gg_build(int32_t n, const uint64_t* pairs, int64_t P, uint64_t seed, int32_t wmax, gg_graph* out) {
  gg_csr c;
  memset(&c, 0, sizeof(c));
  int rc = -4;
  c.pairs = pairs;
  c.seed = seed;
  c.wmax = wmax;
  c.deg = (int64_t*)calloc((size_t)n, sizeof(int64_t));
  int64_t* off = (int64_t*)malloc(((size_t)n + 1) * sizeof(int64_t));
  c.uniq = (int64_t*)malloc((size_t)n * sizeof(int64_t));
  if (!c.deg || !off || !c.uniq) goto done;
  gg_parallel(P, 1 << 16, gg_count, &c);
  off[0] = 0;
  for (int32_t v = 0; v < n; v++) off[v + 1] = off[v] + c.deg[v];
  c.adj = (uint32_t*)malloc((size_t)(off[n] > 0 ? off[n] : 1) * sizeof(uint32_t));
  if (!c.adj) goto done;
  for (int32_t v = 0; v < n; v++) c.deg[v] = off[v];
  gg_parallel(P, 1 << 16, gg_fill, &c);
  c.off = off;
  gg_parallel(n, 1 << 10, gg_sort_rows, &c);
  int64_t m = 0;
  for (int32_t v = 0; v < n; v++) m += c.uniq[v];
  if (m > INT32_MAX) {
    rc = -9;
    goto done;
  }
  out->nodes = n;
  out->edges = (int32_t)m;
  out->nindex = (int32_t*)malloc(((size_t)n + 1) * 4);
  out->nlist = (int32_t*)malloc((size_t)(m > 0 ? m : 1) * 4);
  out->eweight = (int32_t*)malloc((size_t)(m > 0 ? m : 1) * 4);
  if (!out->nindex || !out->nlist || !out->eweight) {
    gg_free(out);
    goto done;
  }
  out->nindex[0] = 0;
  for (int32_t v = 0; v < n; v++) out->nindex[v + 1] = out->nindex[v] + (int32_t)c.uniq[v];
  c.nindex = out->nindex;
  c.nlist = out->nlist;
  c.eweight = out->eweight;
  gg_parallel(n, 1 << 12, gg_emit, &c);
  rc = 0;
done:
  free(c.deg);
  free(off);
  free(c.uniq);
  free(c.adj);
  return rc;
}

/* ---- RMAT: each recursion level consumes 16 random bits, four per draw */
typedef struct {
  uint64_t* pairs;
  uint64_t seed;
  int scale;
  uint32_t ta, tab, tabc;
} gg_rmat_arg;

static void gg_rmat_body(int64_t lo, int64_t hi, void* a) {
  gg_rmat_arg* r = (gg_rmat_arg*)a;
  for (int64_t i = lo; i < hi; i++) {
    uint32_t u = 0, v = 0;
    uint64_t x64 = 0;
    for (int lvl = 0; lvl < r->scale; lvl++) {
      if ((lvl & 3) == 0) x64 = gg_rng(r->seed, GG_STREAM_RMAT, ((uint64_t)i << 3) | (uint64_t)(lvl >> 2));
      const uint32_t x = (uint32_t)(x64 >> (16 * (lvl & 3))) & 0xFFFFu;
      const uint32_t q = x < r->ta ? 0u : x < r->tab ? 1u : x < r->tabc ? 2u : 3u;
      u = (u << 1) | (q >> 1);
      v = (v << 1) | (q & 1u);
    }
    r->pairs[i] = ((uint64_t)u << 32) | v;
  }
}

int gg_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed, int32_t wmax,
            gg_graph* out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 0 || wmax < 1) return -1;
  memset(out, 0, sizeof(*out));
  const int32_t n = 1 << scale;
  const int64_t samples = (int64_t)edge_factor << scale;
  if (2 * samples > INT32_MAX) return -9;
  uint64_t* pairs = (uint64_t*)malloc((size_t)(samples > 0 ? samples : 1) * sizeof(uint64_t));
  if (!pairs) return -4;
  gg_rmat_arg r = {pairs, seed, scale, (uint32_t)lround(a * 65536.0), (uint32_t)lround((a + b) * 65536.0),
                   (uint32_t)lround((a + b + c) * 65536.0)};
  gg_parallel(samples, 1 << 16, gg_rmat_body, &r);
  const int rc = gg_build(n, pairs, samples, seed, wmax, out);
  free(pairs);
  return rc;
}

/* ---- Erdos-Renyi: round(n * avg_degree / 2) uniform pairs */
typedef struct {
  uint64_t* pairs;
  uint64_t seed;
  uint32_t n;
} gg_er_arg;

static void gg_er_body(int64_t lo, int64_t hi, void* a) {
  gg_er_arg* r = (gg_er_arg*)a;
  for (int64_t i = lo; i < hi; i++) {
    const uint64_t x = gg_rng(r->seed, GG_STREAM_ER, (uint64_t)i);
    r->pairs[i] = ((uint64_t)gg_below((uint32_t)(x >> 32), r->n) << 32) | gg_below((uint32_t)x, r->n);
  }
}

int gg_er(int32_t nodes, double avg_degree, uint64_t seed, int32_t wmax, gg_graph* out) {
  if (!out || nodes < 1 || avg_degree < 0 || wmax < 1) return -1;
  memset(out, 0, sizeof(*out));
  const int64_t samples = (int64_t)llround((double)nodes * avg_degree / 2.0);
  if (2 * samples > INT32_MAX) return -9;
  uint64_t* pairs = (uint64_t*)malloc((size_t)(samples > 0 ? samples : 1) * sizeof(uint64_t));
  if (!pairs) return -4;
  gg_er_arg r = {pairs, seed, (uint32_t)nodes};
  gg_parallel(samples, 1 << 16, gg_er_body, &r);
  const int rc = gg_build(nodes, pairs, samples, seed, wmax, out);
  free(pairs);
  return rc;
}

/* ---- 2D 4-neighbour grid, rows x cols, neighbours in increasing id order */
int gg_grid(int32_t rows, int32_t cols, uint64_t seed, int32_t wmax, gg_graph* out) {
  if (!out || rows < 1 || cols < 1 || wmax < 1) return -1;
  memset(out, 0, sizeof(*out));
  const int64_t n = (int64_t)rows * cols;
  const int64_t m = 2 * ((int64_t)rows * (cols - 1) + (int64_t)(rows - 1) * cols);
  if (n > INT32_MAX || m > INT32_MAX) return -9;
  out->nodes = (int32_t)n;
  out->edges = (int32_t)m;
  out->nindex = (int32_t*)malloc(((size_t)n + 1) * 4);
  out->nlist = (int32_t*)malloc((size_t)(m > 0 ? m : 1) * 4);
  out->eweight = (int32_t*)malloc((size_t)(m > 0 ? m : 1) * 4);
  if (!out->nindex || !out->nlist || !out->eweight) {
    gg_free(out);
    return -4;
  }
  int32_t k = 0;
  out->nindex[0] = 0;
  for (int64_t id = 0; id < n; id++) {
    const int32_t r = (int32_t)(id / cols), c = (int32_t)(id % cols);
    int32_t nb[4];
    int d = 0;
    if (r > 0) nb[d++] = (int32_t)(id - cols);
    if (c > 0) nb[d++] = (int32_t)(id - 1);
    if (c < cols - 1) nb[d++] = (int32_t)(id + 1);
    if (r < rows - 1) nb[d++] = (int32_t)(id + cols);
    for (int t = 0; t < d; t++, k++) {
      out->nlist[k] = nb[t];
      out->eweight[k] = gg_weight(seed, (uint32_t)id, (uint32_t)nb[t], wmax);
    }
    out->nindex[id + 1] = k;
  }
  return 0;
}
