// Host side of the ECLgraph boundary: binary CSR I/O, weight synthesis,
// validation, the reference threshold heuristic and verify().
//
// Format and rules follow the reference artifact:
//   ECL-MST/ECLgraph.h:37-64  file layout and the "no weights" case (fread
//                             count 0 -> eweight NULL)
//   ECL-MST/ECLgraph.h:66-80  writer (weights written only when present)
//   ECL-MST/ECL_MST.cu:410-419 weight synthesis 1 + ((i*k) % nodes), abs
//   ECL-MST/ECL_MST.cu:389-395 integer hash used to pick samples
//   ECL-MST/ECL_MST.cu:408,432-440 threshold heuristic
//   ECL-MST/ECL_MST.cu:365-386 verify
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ecl_mst.h"
#include "internal.h"

extern "C" const char* ecl_status_string(int s) {
  switch (s) {
    case ECL_OK: return "ok";
    case ECL_ERR_INVALID_ARG: return "invalid argument";
    case ECL_ERR_IO: return "i/o error";
    case ECL_ERR_FORMAT: return "malformed graph";
    case ECL_ERR_ALLOC: return "allocation failed";
    case ECL_ERR_CUDA: return "CUDA error";
    case ECL_ERR_NO_DEVICE: return "no CUDA device";
    case ECL_ERR_OVERFLOW: return "capacity exceeded";
    case ECL_ERR_TIMEOUT: return "device wait limit reached";
    case ECL_ERR_TOO_LARGE: return "input exceeds the supported maximum";
    case ECL_ERR_UNSUPPORTED: return "unsupported option";
    default: return "unknown status";
  }
}

extern "C" const char* ecl_version(void) { return "ecl-mst-b200 0.1 (sm_100a)"; }

extern "C" void ecl_free_graph(ecl_graph* g) {
  if (!g) return;
  free(g->nindex);
  free(g->nlist);
  free(g->eweight);
  g->nindex = g->nlist = g->eweight = nullptr;
}

extern "C" int ecl_read_graph(const char* path, ecl_graph* out) {
  if (!path || !out) return ECL_ERR_INVALID_ARG;
  memset(out, 0, sizeof(*out));
  FILE* f = fopen(path, "rb");
  if (!f) return ECL_ERR_IO;
  ecl_graph g{};
  int status = ECL_OK;
  size_t cnt;
  if (fread(&g.nodes, 4, 1, f) != 1 || fread(&g.edges, 4, 1, f) != 1) {
    status = ECL_ERR_FORMAT;
    goto done;
  }
  if (g.nodes < 1 || g.edges < 0) { status = ECL_ERR_FORMAT; goto done; }
  g.nindex = (int32_t*)malloc(((size_t)g.nodes + 1) * 4);
  g.nlist = (int32_t*)malloc((size_t)std::max(g.edges, 1) * 4);
  g.eweight = (int32_t*)malloc((size_t)std::max(g.edges, 1) * 4);
  if (!g.nindex || !g.nlist || !g.eweight) { status = ECL_ERR_ALLOC; goto done; }
  if (fread(g.nindex, 4, (size_t)g.nodes + 1, f) != (size_t)g.nodes + 1) {
    status = ECL_ERR_FORMAT;
    goto done;
  }
  if (fread(g.nlist, 4, (size_t)g.edges, f) != (size_t)g.edges) {
    status = ECL_ERR_FORMAT;
    goto done;
  }
  cnt = fread(g.eweight, 4, (size_t)g.edges, f);
  if (cnt == 0) {  // weightless file (ECLgraph.h:54-58); an empty graph also lands here
    free(g.eweight);
    g.eweight = nullptr;
  } else if (cnt != (size_t)g.edges) {
    status = ECL_ERR_FORMAT;
  }
done:
  fclose(f);
  if (status != ECL_OK) {
    ecl_free_graph(&g);
    return status;
  }
  *out = g;
  return ECL_OK;
}

extern "C" int ecl_write_graph(const ecl_graph* g, const char* path) {
  if (!g || !path) return ECL_ERR_INVALID_ARG;
  if (g->nodes < 1 || g->edges < 0 || !g->nindex || (g->edges > 0 && !g->nlist))
    return ECL_ERR_INVALID_ARG;
  FILE* f = fopen(path, "wb");
  if (!f) return ECL_ERR_IO;
  bool ok = fwrite(&g->nodes, 4, 1, f) == 1 && fwrite(&g->edges, 4, 1, f) == 1 &&
            fwrite(g->nindex, 4, (size_t)g->nodes + 1, f) == (size_t)g->nodes + 1 &&
            fwrite(g->nlist, 4, (size_t)g->edges, f) == (size_t)g->edges;
  if (ok && g->eweight)
    ok = fwrite(g->eweight, 4, (size_t)g->edges, f) == (size_t)g->edges;
  if (fclose(f) != 0) ok = false;
  return ok ? ECL_OK : ECL_ERR_IO;
}

extern "C" int ecl_validate_graph(const ecl_graph* g) {
  if (!g || g->nodes < 1 || g->edges < 0 || !g->nindex) return ECL_ERR_INVALID_ARG;
  if (g->edges > 0 && !g->nlist) return ECL_ERR_INVALID_ARG;
  if (g->nindex[0] != 0 || g->nindex[g->nodes] != g->edges) return ECL_ERR_FORMAT;
  for (int32_t v = 0; v < g->nodes; v++)
    if (g->nindex[v + 1] < g->nindex[v]) return ECL_ERR_FORMAT;
  for (int32_t j = 0; j < g->edges; j++)
    if ((uint32_t)g->nlist[j] >= (uint32_t)g->nodes) return ECL_ERR_FORMAT;
  return ECL_OK;
}

extern "C" int ecl_synthesize_weights(ecl_graph* g) {
  if (!g || !g->eweight || !g->nindex || g->nodes < 1) return ECL_ERR_INVALID_ARG;
  for (int32_t i = 0; i < g->nodes; i++) {
    for (int32_t j = g->nindex[i]; j < g->nindex[i + 1]; j++) {
      g->eweight[j] = ecl_synth_weight(i, g->nlist[j], g->nodes);
    }
  }
  return ECL_OK;
}

uint32_t ecl_sample_hash(uint32_t val) {
  // Integer mixing hash (two multiply-xorshift rounds with 0x45d9f3b), the
  // sampler of the reference heuristic.
  val = ((val >> 16) ^ val) * 0x45d9f3bu;
  val = ((val >> 16) ^ val) * 0x45d9f3bu;
  return (val >> 16) ^ val;
}

int ecl_heuristic_threshold_arrays(int32_t nodes, int32_t edges,
                                   const int32_t* eweight, int32_t* threshold,
                                   int32_t* filtered) {
  const int32_t avg_deg = edges / nodes;
  if (avg_deg < 4) {
    *filtered = 0;
    *threshold = INT32_MAX;
    return ECL_OK;
  }
  int32_t s[20];
  const int32_t ns = std::min(edges, 20);
  for (int32_t i = 0; i < ns; i++) s[i] = eweight[ecl_sample_hash((uint32_t)i) % (uint32_t)edges];
  std::sort(s, s + ns);
  const int32_t idx = std::min(19, (int)(3.0 * nodes * ns / edges));
  *threshold = s[idx];
  *filtered = 1;
  return ECL_OK;
}

extern "C" int ecl_heuristic_threshold(const ecl_graph* g, int32_t* threshold,
                                       int32_t* filtered) {
  if (!g || !threshold || !filtered || g->nodes < 1 || g->edges < 0)
    return ECL_ERR_INVALID_ARG;
  if (g->edges / g->nodes >= 4 && !g->eweight) return ECL_ERR_INVALID_ARG;
  return ecl_heuristic_threshold_arrays(g->nodes, g->edges, g->eweight, threshold, filtered);
}

extern "C" uint64_t ecl_forest_weight(const ecl_graph* g, const uint8_t* inMST) {
  uint64_t w = 0;
  if (!g || !inMST || !g->eweight) return 0;
  for (int32_t j = 0; j < g->edges; j++)
    if (inMST[j]) w += (uint64_t)(int64_t)g->eweight[j];
  return w;
}

extern "C" int ecl_verify(const ecl_graph* g, const uint8_t* a, const uint8_t* b,
                          int64_t counts[4], uint64_t* weight_a, uint64_t* weight_b) {
  if (!g || !a || !b) return 0;
  int64_t both = 0, neither = 0, only_a = 0, only_b = 0;
  uint64_t wa = 0, wb = 0;
  for (int32_t j = 0; j < g->edges; j++) {
    const bool x = a[j] != 0, y = b[j] != 0;
    both += x && y;
    neither += !x && !y;
    only_a += x && !y;
    only_b += !x && y;
    if (g->eweight) {
      if (x) wa += (uint64_t)(int64_t)g->eweight[j];
      if (y) wb += (uint64_t)(int64_t)g->eweight[j];
    }
  }
  if (counts) {
    counts[0] = both;
    counts[1] = neither;
    counts[2] = only_a;
    counts[3] = only_b;
  }
  if (weight_a) *weight_a = wa;
  if (weight_b) *weight_b = wb;
  return (wa == wb && only_a == 0 && only_b == 0) ? 1 : 0;
}
