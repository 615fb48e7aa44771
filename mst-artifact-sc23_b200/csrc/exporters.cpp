// Text exporters for the other MST codes of the artifact: the PBBS weighted
// edge array (PBBS_CPU/inputs/ecl2pbbs_genweights.cpp:34-41) and the
// MatrixMarket file cuGraph reads (cuGraph_GPU/inputs/
// ecl2mtx_genweights_cugraph.cpp:37-50), byte for byte. The reference prints
// each weight as a float through printf ("%f" / "%.1f"). A float converted
// from an int32 is a whole number of magnitude at most 2^31, so its "%f" text
// is that integer followed by ".000000" (".0" for "%.1f"); the writers print
// it that way with an integer formatter. Lines are formatted in parallel, one
// row range per thread, and written in row order.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "ecl_mst.h"
#include "internal.h"

namespace {

// Decimal text of v appended at p; returns the new end.
char* put_int(char* p, int64_t v) {
  if (v < 0) {
    *p++ = '-';
    v = -v;
  }
  char tmp[24];
  int n = 0;
  do {
    tmp[n++] = (char)('0' + v % 10);
    v /= 10;
  } while (v);
  while (n) *p++ = tmp[--n];
  return p;
}

// The integer printf shows for float(w).
int64_t float_value(int32_t w) { return (int64_t)(float)w; }

enum class Fmt { kPbbs, kMtx };

// Text of rows [r0, r1) in `out`.
void format_rows(const ecl_graph* g, Fmt fmt, int32_t r0, int32_t r1, std::string& out) {
  const int64_t entries = (int64_t)g->nindex[r1] - g->nindex[r0];
  out.resize((size_t)std::max<int64_t>(entries, 0) * 48 + 64);
  char* p = &out[0];
  for (int32_t src = r0; src < r1; src++) {
    for (int32_t j = g->nindex[src]; j < g->nindex[src + 1]; j++) {
      const int32_t dst = g->nlist[j];
      const int32_t w = g->eweight ? g->eweight[j] : ecl_synth_weight(src, dst, g->nodes);
      if (fmt == Fmt::kPbbs) {
        p = put_int(p, src);
        *p++ = ' ';
        p = put_int(p, dst);
        *p++ = ' ';
        p = put_int(p, float_value(w));
        memcpy(p, ".000000\n", 8);
        p += 8;
      } else if (src > dst) {
        p = put_int(p, (int64_t)src + 1);
        *p++ = ' ';
        p = put_int(p, (int64_t)dst + 1);
        *p++ = ' ';
        p = put_int(p, float_value(w));
        memcpy(p, ".0\n", 3);
        p += 3;
      }
    }
  }
  out.resize((size_t)(p - out.data()));
}

int write_text(const ecl_graph* g, const char* path, Fmt fmt) {
  if (!g || !path) return ECL_ERR_INVALID_ARG;
  const int st = ecl_validate_graph(g);
  if (st) return st;
  FILE* f = fopen(path, "wb");
  if (!f) return ECL_ERR_IO;
  bool ok = true;
  if (fmt == Fmt::kPbbs) {
    ok = fputs("WeightedEdgeArray\n", f) >= 0;
  } else {
    ok = fprintf(f, "%%%%MatrixMarket matrix coordinate real symmetric\n%d %d %d\n", g->nodes, g->nodes,
                 g->edges / 2) > 0;
  }
  // Rounds of `threads` row ranges of about kChunk entries each.
  constexpr int64_t kChunk = 1 << 22;
  const unsigned hc = std::thread::hardware_concurrency();
  const int threads = (int)std::max(1u, std::min(hc ? hc : 1u, 64u));
  std::vector<std::string> text((size_t)threads);
  int32_t row = 0;
  while (ok && row < g->nodes) {
    std::vector<int32_t> cut(1, row);
    for (int t = 0; t < threads && cut.back() < g->nodes; t++) {
      const int64_t target = (int64_t)g->nindex[cut.back()] + kChunk;
      // first row whose start is past the target (at least one row per range)
      int32_t next = (int32_t)(std::upper_bound(g->nindex + cut.back() + 1, g->nindex + g->nodes, target) -
                               g->nindex);
      cut.push_back(std::min(next, g->nodes));
    }
    const int parts = (int)cut.size() - 1;
    std::vector<std::thread> pool;
    for (int t = 1; t < parts; t++) pool.emplace_back(format_rows, g, fmt, cut[t], cut[t + 1], std::ref(text[t]));
    format_rows(g, fmt, cut[0], cut[1], text[0]);
    for (auto& th : pool) th.join();
    for (int t = 0; t < parts && ok; t++) ok = fwrite(text[t].data(), 1, text[t].size(), f) == text[t].size();
    row = cut.back();
  }
  if (fclose(f) != 0) ok = false;
  return ok ? ECL_OK : ECL_ERR_IO;
}

}  // namespace

extern "C" int ecl_write_pbbs(const ecl_graph* g, const char* path) { return write_text(g, path, Fmt::kPbbs); }

extern "C" int ecl_write_mtx(const ecl_graph* g, const char* path) { return write_text(g, path, Fmt::kMtx); }
