// The plain ECL-MST: the UNMODIFIED reference ECL-MST/ECL_MST.cu rebuilt for
// sm_100a, compiled by baseline/Makefile straight from the reference source
// tree into baseline/_ref/ (not committed). It is the comparison target the
// benchmark reports beside the new kernels. `main` is renamed so gpuMST
// (ECL_MST.cu:265-362) can be called as a function, and `printf` is
// redirected so the runtime line gpuMST prints (:345) is captured.
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

static char g_plain_line[256];
static int plain_capture_printf(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  const int r = vsnprintf(g_plain_line, sizeof g_plain_line, fmt, ap);
  va_end(ap);
  return r;
}

#define main ecl_plain_main
#define printf plain_capture_printf
#include ECL_REF_SOURCE
#undef printf
#undef main

extern "C" {

// Threshold choice of the reference main (ECL_MST.cu:408,432-444).
void plain_threshold(int nodes, int edges, const int* eweight, int* filter, int* threshold) {
  if (edges / nodes >= 4) {
    int s[20];
    const int ns = std::min(edges, 20);
    for (int i = 0; i < ns; i++) s[i] = eweight[(hash(i) % edges)];
    std::sort(s, s + ns);
    *threshold = s[std::min(19, (int)(3.0 * nodes * ns / edges))];
    *filter = 1;
  } else {
    *threshold = INT_MAX;
    *filter = 0;
  }
}

// One gpuMST<filter> call; *seconds = the reference's own timed window.
int plain_gpu_mst(int nodes, int edges, const int* nindex, const int* nlist, const int* eweight,
                  int filter, int threshold, unsigned char* inMST, double* seconds) {
  ECLgraph g;
  g.nodes = nodes;
  g.edges = edges;
  g.nindex = const_cast<int*>(nindex);
  g.nlist = const_cast<int*>(nlist);
  g.eweight = const_cast<int*>(eweight);
  g_plain_line[0] = 0;
  bool* r = filter ? gpuMST<true>(g, threshold) : gpuMST<false>(g, threshold);
  if (inMST)
    for (int j = 0; j < edges; j++) inMST[j] = r[j] ? 1 : 0;
  delete[] r;
  if (seconds) *seconds = atof(g_plain_line);
  return 0;
}

}  // extern "C"
