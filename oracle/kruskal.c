/*
 * ORACLE -- test infrastructure only. Nothing in the product library links,
 * loads or calls this file; only the test suite, the smoke check and the
 * benchmark's CPU-baseline leg do, as the checker.
 *
 * A plain-C restatement of the reference artifact's minimum spanning forest
 * semantics (alexfallin/MST-Artifact-SC23):
 *
 *   oracle_mst        serial Kruskal of cpuMST (ECL-MST/ECL_MST.cu:82-124):
 *                     one-direction entries nlist[j] > v only (:97), ordered
 *                     by (weight, edge index j), union-find with path
 *                     compression (serial_find :55-67, serial_join :70-79),
 *                     inMST marked at index j (:112), early exit after
 *                     nodes-1 unions (:104-116). Two refinements make it the
 *                     oracle of the GPU path gpuMST<filter> (:265-362):
 *                     weights are ordered as uint32, because the GPU key is
 *                     ((ull)w << 32) | j (:221,:234); and when `filtered`,
 *                     light entries (w <= threshold, signed, :172) are
 *                     processed before heavy ones (w > threshold), mirroring
 *                     the two phases (:309-340). For non-negative weights
 *                     both refinements change nothing: the forest is the
 *                     unique MSF under (w, j) for every threshold.
 *   oracle_heuristic  threshold rule of main (:389-395 hash, :408, :432-440)
 *   oracle_verify     verify() (:365-386)
 *   oracle_synth      weight synthesis for weightless inputs (:410-419)
 *
 * Parity pin: tests/test_oracle.py compares oracle_mst with the reference's
 * own cpuMST, compiled from the reference sources into oracle/_ref by
 * oracle/Makefile, and with the committed fixtures in tests/golden/ that
 * tests/golden/make_golden.py generated from that compiled reference.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  uint64_t key; /* ((uint64)(uint32)w << 32) | j */
  int32_t a, b; /* endpoints v < n */
} oedge;

/* LSD radix sort of edges by key, 16-bit digits, 4 passes. */
static int sort_edges(oedge* e, int64_t cnt) {
  if (cnt < 2) return 0;
  oedge* tmp = (oedge*)malloc((size_t)cnt * sizeof(oedge));
  int64_t* hist = (int64_t*)malloc(65536 * sizeof(int64_t));
  if (!tmp || !hist) {
    free(tmp);
    free(hist);
    return -1;
  }
  oedge *src = e, *dst = tmp;
  for (int pass = 0; pass < 4; pass++) {
    const int sh = 16 * pass;
    memset(hist, 0, 65536 * sizeof(int64_t));
    for (int64_t i = 0; i < cnt; i++) hist[(src[i].key >> sh) & 0xFFFF]++;
    int64_t sum = 0;
    for (int d = 0; d < 65536; d++) {
      const int64_t c = hist[d];
      hist[d] = sum;
      sum += c;
    }
    for (int64_t i = 0; i < cnt; i++) dst[hist[(src[i].key >> sh) & 0xFFFF]++] = src[i];
    oedge* t = src;
    src = dst;
    dst = t;
  }
  /* four passes: the sorted data is back in e */
  free(tmp);
  free(hist);
  return 0;
}

static int32_t ofind(int32_t* parent, int32_t idx) {
  int32_t curr = parent[idx];
  if (curr != idx) {
    int32_t next, prev = idx;
    while (curr != (next = parent[curr])) {
      parent[prev] = next;
      prev = curr;
      curr = next;
    }
  }
  return curr;
}

/* Returns 0, or -1 on allocation failure / bad input. inMST gets edges bytes. */
int oracle_mst(int32_t nodes, int32_t edges, const int32_t* nindex, const int32_t* nlist,
               const int32_t* eweight, int32_t threshold, int32_t filtered, uint8_t* inMST,
               uint64_t* weight_out, int64_t* forest_edges_out) {
  if (nodes < 1 || edges < 0) return -1;
  memset(inMST, 0, (size_t)edges);
  int64_t one_dir = 0;
  for (int32_t v = 0; v < nodes; v++)
    for (int32_t j = nindex[v]; j < nindex[v + 1]; j++)
      if (nlist[j] > v) one_dir++;
  oedge* e = (oedge*)malloc((size_t)(one_dir > 0 ? one_dir : 1) * sizeof(oedge));
  int32_t* parent = (int32_t*)malloc((size_t)nodes * sizeof(int32_t));
  if (!e || !parent) {
    free(e);
    free(parent);
    return -1;
  }
  /* light entries first (or all entries when unfiltered), then heavy */
  int64_t nl = 0;
  for (int pass = 0; pass < 2; pass++) {
    for (int32_t v = 0; v < nodes; v++) {
      for (int32_t j = nindex[v]; j < nindex[v + 1]; j++) {
        const int32_t n = nlist[j];
        if (n <= v) continue;
        const int light = !filtered || eweight[j] <= threshold;
        if ((pass == 0) != (light != 0)) continue;
        e[nl].key = ((uint64_t)(uint32_t)eweight[j] << 32) | (uint32_t)j;
        e[nl].a = v;
        e[nl].b = n;
        nl++;
      }
    }
    if (pass == 0) one_dir = nl; /* remember the split */
  }
  const int64_t n_light = one_dir, n_all = nl;
  if (sort_edges(e, n_light) || sort_edges(e + n_light, n_all - n_light)) {
    free(e);
    free(parent);
    return -1;
  }
  for (int32_t i = 0; i < nodes; i++) parent[i] = i;
  int64_t count = nodes - 1, fe = 0;
  uint64_t w = 0;
  for (int64_t pos = 0; pos < n_all && count > 0; pos++) {
    const int32_t arep = ofind(parent, e[pos].a);
    const int32_t brep = ofind(parent, e[pos].b);
    if (arep != brep) {
      const int32_t j = (int32_t)(e[pos].key & 0xFFFFFFFFu);
      inMST[j] = 1;
      w += (uint64_t)(int64_t)eweight[j];
      fe++;
      if (arep > brep) parent[brep] = arep;
      else parent[arep] = brep;
      count--;
    }
  }
  free(e);
  free(parent);
  if (weight_out) *weight_out = w;
  if (forest_edges_out) *forest_edges_out = fe;
  return 0;
}

static uint32_t ohash(uint32_t val) {
  val = ((val >> 16) ^ val) * 0x45d9f3bu;
  val = ((val >> 16) ^ val) * 0x45d9f3bu;
  return (val >> 16) ^ val;
}

/* Threshold rule of main: filtered iff edges/nodes >= 4. */
void oracle_heuristic(int32_t nodes, int32_t edges, const int32_t* eweight, int32_t* threshold,
                      int32_t* filtered) {
  if (nodes < 1 || edges / nodes < 4) {
    *filtered = 0;
    *threshold = 0x7fffffff;
    return;
  }
  int32_t s[20];
  const int32_t ns = edges < 20 ? edges : 20;
  for (int32_t i = 0; i < ns; i++) s[i] = eweight[ohash((uint32_t)i) % (uint32_t)edges];
  for (int32_t i = 1; i < ns; i++) {
    const int32_t x = s[i];
    int32_t k = i - 1;
    while (k >= 0 && s[k] > x) {
      s[k + 1] = s[k];
      k--;
    }
    s[k + 1] = x;
  }
  int32_t idx = (int32_t)(3.0 * nodes * ns / edges);
  if (idx > 19) idx = 19;
  *filtered = 1;
  *threshold = s[idx];
}

/* verify(): returns 1 when no entry is in only one forest and the uint64
 * weights agree. counts: both, neither, only_a, only_b. */
int oracle_verify(int32_t edges, const int32_t* eweight, const uint8_t* a, const uint8_t* b,
                  int64_t* counts) {
  int64_t both = 0, neither = 0, oa = 0, ob = 0;
  uint64_t wa = 0, wb = 0;
  for (int32_t j = 0; j < edges; j++) {
    const int x = a[j] != 0, y = b[j] != 0;
    both += x && y;
    neither += !x && !y;
    oa += x && !y;
    ob += !x && y;
    if (x) wa += (uint64_t)(int64_t)eweight[j];
    if (y) wb += (uint64_t)(int64_t)eweight[j];
  }
  if (counts) {
    counts[0] = both;
    counts[1] = neither;
    counts[2] = oa;
    counts[3] = ob;
  }
  return (wa == wb && oa == 0 && ob == 0) ? 1 : 0;
}

/* Weight synthesis with the int32 wrap of i*k. */
void oracle_synth(int32_t nodes, const int32_t* nindex, const int32_t* nlist, int32_t* eweight) {
  for (int32_t i = 0; i < nodes; i++)
    for (int32_t j = nindex[i]; j < nindex[i + 1]; j++) {
      const int32_t prod = (int32_t)((uint32_t)i * (uint32_t)nlist[j]);
      int32_t w = 1 + prod % nodes;
      if (w < 0) w = -w;
      eweight[j] = w;
    }
}
