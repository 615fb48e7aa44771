// Seeded synthetic ECLgraph inputs: 2D grid, Erdos-Renyi, RMAT and random
// geometric 2D graphs. These stand in for the reference's downloaded .egr
// benchmark inputs (Inputs/download_inputs.sh), which are not available
// offline. Every generator is deterministic for a given seed and thread count
// independent: sampling uses a counter-based hash and the CSR builder sorts
// and deduplicates each row, so the result does not depend on scheduling.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

#include "ecl_mst.h"
#include "internal.h"

namespace {

int resolve_threads(int threads) {
  if (threads > 0) return threads;
  unsigned hc = std::thread::hardware_concurrency();
  return hc ? (int)hc : 1;
}

// Run body(begin, end, tid) over [0, n) split into `threads` contiguous parts.
void parallel_for(int64_t n, int threads, const std::function<void(int64_t, int64_t, int)>& body) {
  if (n <= 0) return;
  threads = (int)std::max<int64_t>(1, std::min<int64_t>(threads, n / 4096 + 1));
  if (threads == 1) {
    body(0, n, 0);
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; t++) {
    const int64_t b = n * t / threads, e = n * (t + 1) / threads;
    pool.emplace_back(body, b, e, t);
  }
  for (auto& th : pool) th.join();
}

// Build a symmetric, deduplicated, self-loop-free CSR from an undirected pair
// list. Rows are sorted by neighbour id; weights come from ecl_edge_weight.
int build_csr(int32_t n, const std::vector<uint64_t>& pairs, uint64_t seed, int32_t wmax,
              int threads, ecl_graph* out) {
  std::vector<std::atomic<int64_t>> deg(n);
  for (auto& d : deg) d.store(0, std::memory_order_relaxed);
  const int64_t P = (int64_t)pairs.size();
  parallel_for(P, threads, [&](int64_t b, int64_t e, int) {
    for (int64_t i = b; i < e; i++) {
      const uint32_t u = (uint32_t)(pairs[i] >> 32), v = (uint32_t)pairs[i];
      if (u == v) continue;
      deg[u].fetch_add(1, std::memory_order_relaxed);
      deg[v].fetch_add(1, std::memory_order_relaxed);
    }
  });
  std::vector<int64_t> off((size_t)n + 1, 0);
  for (int32_t v = 0; v < n; v++) off[v + 1] = off[v] + deg[v].load(std::memory_order_relaxed);
  const int64_t raw = off[n];
  std::vector<uint32_t> adj((size_t)std::max<int64_t>(raw, 1));
  std::vector<std::atomic<int64_t>> cur(n);
  for (int32_t v = 0; v < n; v++) cur[v].store(off[v], std::memory_order_relaxed);
  parallel_for(P, threads, [&](int64_t b, int64_t e, int) {
    for (int64_t i = b; i < e; i++) {
      const uint32_t u = (uint32_t)(pairs[i] >> 32), v = (uint32_t)pairs[i];
      if (u == v) continue;
      adj[cur[u].fetch_add(1, std::memory_order_relaxed)] = v;
      adj[cur[v].fetch_add(1, std::memory_order_relaxed)] = u;
    }
  });
  std::vector<int64_t> uniq((size_t)n, 0);
  parallel_for(n, threads, [&](int64_t b, int64_t e, int) {
    for (int64_t v = b; v < e; v++) {
      uint32_t* first = adj.data() + off[v];
      uint32_t* last = adj.data() + off[v + 1];
      std::sort(first, last);
      uniq[v] = std::unique(first, last) - first;
    }
  });
  int64_t m = 0;
  for (int32_t v = 0; v < n; v++) m += uniq[v];
  if (m > INT32_MAX) return ECL_ERR_TOO_LARGE;
  ecl_graph g{};
  g.nodes = n;
  g.edges = (int32_t)m;
  g.nindex = (int32_t*)malloc(((size_t)n + 1) * 4);
  g.nlist = (int32_t*)malloc((size_t)std::max<int64_t>(m, 1) * 4);
  g.eweight = (int32_t*)malloc((size_t)std::max<int64_t>(m, 1) * 4);
  if (!g.nindex || !g.nlist || !g.eweight) {
    ecl_free_graph(&g);
    return ECL_ERR_ALLOC;
  }
  g.nindex[0] = 0;
  for (int32_t v = 0; v < n; v++) g.nindex[v + 1] = g.nindex[v] + (int32_t)uniq[v];
  parallel_for(n, threads, [&](int64_t b, int64_t e, int) {
    for (int64_t v = b; v < e; v++) {
      const int32_t base = g.nindex[v];
      for (int64_t k = 0; k < uniq[v]; k++) {
        const uint32_t w = adj[off[v] + k];
        g.nlist[base + k] = (int32_t)w;
        g.eweight[base + k] = ecl_edge_weight(seed, (uint32_t)v, w, wmax);
      }
    }
  });
  *out = g;
  return ECL_OK;
}

}  // namespace

EclRmatCut ecl_rmat_cut(double a, double b, double c) {
  EclRmatCut cut;
  cut.ta = (uint32_t)std::lround(a * 65536.0);
  cut.tab = (uint32_t)std::lround((a + b) * 65536.0);
  cut.tabc = (uint32_t)std::lround((a + b + c) * 65536.0);
  return cut;
}

EclRggGrid ecl_rgg_grid(int32_t nodes, double avg_degree) {
  // Unit square in 31-bit fixed point; radius from E[deg] = n * pi * r^2.
  const double kOne = 2147483648.0;
  const double rad = std::sqrt(avg_degree / (M_PI * (double)nodes));
  const uint64_t r_fix = (uint64_t)std::min(kOne, std::floor(rad * kOne));
  EclRggGrid g;
  g.r2 = r_fix * r_fix;
  // Cells at least one radius wide, and no more than about 4n of them.
  const int64_t cap = 2 * (int64_t)std::sqrt((double)nodes) + 1;
  g.cells = std::max<int64_t>(1, std::min<int64_t>(cap, (int64_t)(kOne / std::max<uint64_t>(r_fix, 1))));
  g.cell_w = (uint64_t)std::ceil(kOne / (double)g.cells);
  return g;
}

// Graph `index` of the mixed batch: seed = seed0 + index; the family is
// uniform over {grid, Erdos-Renyi (avg degree 8), RMAT (0.57, 0.19, 0.19,
// edge factor 8), random geometric 2D (avg degree 3)} and the vertex count
// log-uniform in [nmin, nmax] (RMAT rounds it to a power of two, the grid to
// rows x cols with rows = floor(sqrt(n))).
EclBatchPick ecl_batch_pick(int32_t index, uint64_t seed0, int32_t nmin, int32_t nmax) {
  EclBatchPick p;
  p.seed = seed0 + (uint64_t)index;
  const uint64_t r0 = ecl_rng(p.seed, 5, 0), r1 = ecl_rng(p.seed, 5, 1);
  p.family = (int)(r0 % 4);
  const double u = (double)(r1 >> 11) * (1.0 / 9007199254740992.0);
  const double ln = std::log((double)nmin) + u * (std::log((double)nmax) - std::log((double)nmin));
  p.nodes = (int32_t)std::max<double>(nmin, std::min<double>(nmax, std::llround(std::exp(ln))));
  p.rows_or_scale = 0;
  if (p.family == 0) p.rows_or_scale = std::max<int32_t>(1, (int32_t)std::sqrt((double)p.nodes));
  if (p.family == 2) p.rows_or_scale = std::max<int32_t>(1, (int32_t)std::lround(std::log2((double)p.nodes)));
  return p;
}

extern "C" int ecl_gen_grid(int32_t rows, int32_t cols, uint64_t seed, int32_t wmax, int threads,
                            ecl_graph* out) {
  if (!out || rows < 1 || cols < 1 || wmax < 1) return ECL_ERR_INVALID_ARG;
  const int64_t n64 = (int64_t)rows * cols;
  const int64_t m64 = 2 * ((int64_t)rows * (cols - 1) + (int64_t)(rows - 1) * cols);
  if (n64 > INT32_MAX || m64 > INT32_MAX) return ECL_ERR_TOO_LARGE;
  threads = resolve_threads(threads);
  ecl_graph g{};
  g.nodes = (int32_t)n64;
  g.edges = (int32_t)m64;
  g.nindex = (int32_t*)malloc(((size_t)n64 + 1) * 4);
  g.nlist = (int32_t*)malloc((size_t)std::max<int64_t>(m64, 1) * 4);
  g.eweight = (int32_t*)malloc((size_t)std::max<int64_t>(m64, 1) * 4);
  if (!g.nindex || !g.nlist || !g.eweight) {
    ecl_free_graph(&g);
    return ECL_ERR_ALLOC;
  }
  // Row offsets in closed form: degree = 4 minus the missing borders.
  g.nindex[0] = 0;
  for (int64_t id = 0; id < n64; id++) {
    const int32_t r = (int32_t)(id / cols), c = (int32_t)(id % cols);
    const int d = (r > 0) + (c > 0) + (c < cols - 1) + (r < rows - 1);
    g.nindex[id + 1] = g.nindex[id] + d;
  }
  parallel_for(n64, threads, [&](int64_t b, int64_t e, int) {
    for (int64_t id = b; id < e; id++) {
      const int32_t r = (int32_t)(id / cols), c = (int32_t)(id % cols);
      int32_t k = g.nindex[id];
      int32_t nb[4];
      int d = 0;
      if (r > 0) nb[d++] = (int32_t)(id - cols);
      if (c > 0) nb[d++] = (int32_t)(id - 1);
      if (c < cols - 1) nb[d++] = (int32_t)(id + 1);
      if (r < rows - 1) nb[d++] = (int32_t)(id + cols);
      for (int t = 0; t < d; t++, k++) {
        g.nlist[k] = nb[t];
        g.eweight[k] = ecl_edge_weight(seed, (uint32_t)id, (uint32_t)nb[t], wmax);
      }
    }
  });
  *out = g;
  return ECL_OK;
}

extern "C" int ecl_gen_er(int32_t nodes, double avg_degree, uint64_t seed, int32_t wmax,
                          int threads, ecl_graph* out) {
  if (!out || nodes < 1 || avg_degree < 0 || wmax < 1) return ECL_ERR_INVALID_ARG;
  threads = resolve_threads(threads);
  const int64_t samples = (int64_t)std::llround((double)nodes * avg_degree / 2.0);
  if (2 * samples > INT32_MAX) return ECL_ERR_TOO_LARGE;
  std::vector<uint64_t> pairs((size_t)samples);
  parallel_for(samples, threads, [&](int64_t b, int64_t e, int) {
    for (int64_t i = b; i < e; i++) {
      const uint64_t r = ecl_rng(seed, ECL_STREAM_ER, (uint64_t)i);
      const uint32_t u = ecl_below((uint32_t)(r >> 32), (uint32_t)nodes);
      const uint32_t v = ecl_below((uint32_t)r, (uint32_t)nodes);
      pairs[i] = ((uint64_t)u << 32) | v;
    }
  });
  return build_csr(nodes, pairs, seed, wmax, threads, out);
}

extern "C" int ecl_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                            uint64_t seed, int32_t wmax, int threads, ecl_graph* out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 0 || wmax < 1) return ECL_ERR_INVALID_ARG;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0 + 1e-12) return ECL_ERR_INVALID_ARG;
  threads = resolve_threads(threads);
  const int32_t n = 1 << scale;
  const int64_t samples = (int64_t)edge_factor << scale;
  if (2 * samples > INT32_MAX) return ECL_ERR_TOO_LARGE;
  // Each recursion level consumes 16 random bits, four levels per 64-bit draw.
  const EclRmatCut cut = ecl_rmat_cut(a, b, c);
  const uint32_t ta = cut.ta, tab = cut.tab, tabc = cut.tabc;
  std::vector<uint64_t> pairs((size_t)samples);
  parallel_for(samples, threads, [&](int64_t bb, int64_t e, int) {
    for (int64_t i = bb; i < e; i++) {
      uint32_t u = 0, v = 0;
      uint64_t r = 0;
      for (int lvl = 0; lvl < scale; lvl++) {
        if ((lvl & 3) == 0) r = ecl_rng(seed, ECL_STREAM_RMAT, ((uint64_t)i << 3) | (uint64_t)(lvl >> 2));
        const uint32_t x = (uint32_t)(r >> (16 * (lvl & 3))) & 0xFFFFu;
        const uint32_t q = x < ta ? 0u : x < tab ? 1u : x < tabc ? 2u : 3u;
        u = (u << 1) | (q >> 1);
        v = (v << 1) | (q & 1u);
      }
      pairs[i] = ((uint64_t)u << 32) | v;
    }
  });
  return build_csr(n, pairs, seed, wmax, threads, out);
}

extern "C" int ecl_gen_rgg2d(int32_t nodes, double avg_degree, uint64_t seed, int32_t wmax,
                             int threads, ecl_graph* out) {
  if (!out || nodes < 1 || avg_degree < 0 || wmax < 1) return ECL_ERR_INVALID_ARG;
  threads = resolve_threads(threads);
  const EclRggGrid grid = ecl_rgg_grid(nodes, avg_degree);
  const uint64_t r2 = grid.r2, cell_w = grid.cell_w;
  const int64_t cells = grid.cells;
  std::vector<uint32_t> px(nodes), py(nodes);
  std::vector<uint64_t> order(nodes);
  parallel_for(nodes, threads, [&](int64_t b, int64_t e, int) {
    for (int64_t i = b; i < e; i++) {
      const uint64_t r = ecl_rng(seed, ECL_STREAM_RGG, (uint64_t)i);
      px[i] = (uint32_t)(r >> 33);
      py[i] = (uint32_t)(r & 0x7FFFFFFFu);
    }
  });
  // Number vertices in cell order (row-major over cells) so ids follow space,
  // like road networks. Key: cell id (high) | original index (low).
  for (int64_t i = 0; i < nodes; i++) {
    const uint64_t cx = px[i] / cell_w, cy = py[i] / cell_w;
    order[i] = ((cy * (uint64_t)cells + cx) << 32) | (uint64_t)i;
  }
  std::sort(order.begin(), order.end());
  std::vector<uint32_t> sx(nodes), sy(nodes);
  std::vector<int64_t> cell_start((size_t)(cells * cells) + 1, 0);
  for (int64_t k = 0; k < nodes; k++) {
    const uint32_t i = (uint32_t)order[k];
    sx[k] = px[i];
    sy[k] = py[i];
    cell_start[(order[k] >> 32) + 1]++;
  }
  for (int64_t cidx = 0; cidx < cells * cells; cidx++) cell_start[cidx + 1] += cell_start[cidx];
  std::vector<std::vector<uint64_t>> part(threads);
  parallel_for(nodes, threads, [&](int64_t b, int64_t e, int tid) {
    auto& mine = part[tid];
    for (int64_t k = b; k < e; k++) {
      const int64_t cx = sx[k] / cell_w, cy = sy[k] / cell_w;
      for (int64_t dy = -1; dy <= 1; dy++) {
        const int64_t yy = cy + dy;
        if (yy < 0 || yy >= cells) continue;
        for (int64_t dx = -1; dx <= 1; dx++) {
          const int64_t xx = cx + dx;
          if (xx < 0 || xx >= cells) continue;
          const int64_t cid = yy * cells + xx;
          for (int64_t q = cell_start[cid]; q < cell_start[cid + 1]; q++) {
            if (q <= k) continue;  // each unordered pair once
            const int64_t ddx = (int64_t)sx[k] - (int64_t)sx[q];
            const int64_t ddy = (int64_t)sy[k] - (int64_t)sy[q];
            if ((uint64_t)(ddx * ddx) + (uint64_t)(ddy * ddy) < r2)
              mine.push_back(((uint64_t)k << 32) | (uint64_t)q);
          }
        }
      }
    }
  });
  std::vector<uint64_t> pairs;
  size_t total = 0;
  for (auto& p : part) total += p.size();
  if (2 * total > (size_t)INT32_MAX) return ECL_ERR_TOO_LARGE;
  pairs.reserve(total);
  for (auto& p : part) pairs.insert(pairs.end(), p.begin(), p.end());
  return build_csr(nodes, pairs, seed, wmax, threads, out);
}

// Graph `index` of the mixed batch (family, size and seed from
// ecl_batch_pick). Single-threaded, so many graphs can be generated in
// parallel.
extern "C" int ecl_gen_batch_graph(int32_t index, uint64_t seed0, int32_t nmin, int32_t nmax,
                                   int32_t wmax, ecl_graph* out, int32_t* family) {
  if (!out || nmin < 1 || nmax < nmin || index < 0) return ECL_ERR_INVALID_ARG;
  const EclBatchPick p = ecl_batch_pick(index, seed0, nmin, nmax);
  if (family) *family = p.family;
  switch (p.family) {
    case 0:
      return ecl_gen_grid(p.rows_or_scale, std::max<int32_t>(1, p.nodes / p.rows_or_scale), p.seed, wmax, 1,
                          out);
    case 1:
      return ecl_gen_er(p.nodes, kBatchErDegree, p.seed, wmax, 1, out);
    case 2:
      return ecl_gen_rmat(p.rows_or_scale, kBatchRmatEdgeFactor, kBatchRmatA, kBatchRmatB, kBatchRmatC, p.seed,
                          wmax, 1, out);
    default:
      return ecl_gen_rgg2d(p.nodes, kBatchRggDegree, p.seed, wmax, 1, out);
  }
}
