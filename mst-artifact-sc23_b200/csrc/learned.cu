// Learned filter threshold and degree split (placeholder until the MLP lands).
#include <cuda_runtime.h>

#include "ecl_mst.h"

struct ecl_mst_ctx;
int ecl_learned_prepare(ecl_mst_ctx*, const ecl_graph*, cudaStream_t, void*) {
  return ECL_ERR_UNSUPPORTED;
}
