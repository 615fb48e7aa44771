// Test harness around the UNMODIFIED reference ECL-MST/ECL_MST.cu (ORACLE,
// test infrastructure only). It is compiled by oracle/Makefile directly from
// the reference source tree, into oracle/_ref/ which is not committed; the
// reference file is included, not copied. `main` is renamed so that cpuMST
// (ECL_MST.cu:82-124) and gpuMST<filter> (:265-362) can be called as
// functions, and `printf` is redirected so the runtime line gpuMST prints
// (:345) is captured instead of written to stdout.
#include <algorithm>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <tuple>
#include <vector>
#include <sys/time.h>
#include <cuda.h>
#include <cuda_runtime.h>

static char g_ref_line[256];
static int ref_capture_printf(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  const int r = vsnprintf(g_ref_line, sizeof g_ref_line, fmt, ap);
  va_end(ap);
  return r;
}

#define main ecl_reference_main
#define printf ref_capture_printf
#include ECL_REF_SOURCE
#undef printf
#undef main

static ECLgraph as_graph(int nodes, int edges, const int* nindex, const int* nlist,
                         const int* eweight) {
  ECLgraph g;
  g.nodes = nodes;
  g.edges = edges;
  g.nindex = const_cast<int*>(nindex);
  g.nlist = const_cast<int*>(nlist);
  g.eweight = const_cast<int*>(eweight);
  return g;
}

extern "C" {

// cpuMST of the reference; inMST receives `edges` bytes.
int ref_cpu_mst(int nodes, int edges, const int* nindex, const int* nlist, const int* eweight,
                unsigned char* inMST) {
  const ECLgraph g = as_graph(nodes, edges, nindex, nlist, eweight);
  bool* r = cpuMST(g);
  for (int j = 0; j < edges; j++) inMST[j] = r[j] ? 1 : 0;
  delete[] r;
  return 0;
}

// The threshold choice of the reference main (ECL_MST.cu:408,432-444), using
// the reference's own hash().
void ref_threshold(int nodes, int edges, const int* eweight, int* filter, int* threshold) {
  const int avg_deg = edges / nodes;
  if (avg_deg >= 4) {
    int sorted_weights[20];
    const int num_samples = std::min(edges, 20);
    for (int i = 0; i < num_samples; i++) sorted_weights[i] = eweight[(hash(i) % edges)];
    std::sort(sorted_weights, sorted_weights + num_samples);
    *threshold = sorted_weights[std::min(19, (int)(3.0 * nodes * num_samples / edges))];
    *filter = 1;
  } else {
    *threshold = INT_MAX;
    *filter = 0;
  }
}

// gpuMST<filter>(g, threshold) of the reference on device 0; returns the
// runtime the reference measured and printed (seconds) in *seconds.
int ref_gpu_mst(int nodes, int edges, const int* nindex, const int* nlist, const int* eweight,
                int filter, int threshold, unsigned char* inMST, double* seconds) {
  const ECLgraph g = as_graph(nodes, edges, nindex, nlist, eweight);
  g_ref_line[0] = 0;
  bool* r = filter ? gpuMST<true>(g, threshold) : gpuMST<false>(g, threshold);
  for (int j = 0; j < edges; j++) inMST[j] = r[j] ? 1 : 0;
  delete[] r;
  if (seconds) *seconds = atof(g_ref_line);
  return 0;
}

}  // extern "C"
