// March kernel variants of tile shape 2 (see march_host.cuh).
#include "march_host.cuh"

namespace fdmap {

int march_configure_s2(fdmap_gpu* h) { return march_configure_shape<2>(h); }
int march_launch_s2(fdmap_gpu* h, const StageArgs& a) { return march_launch_shape<2>(h, a); }
int march_batch_s2(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s) {
  return march_batch_shape<2>(proto, a, p, s);
}

}  // namespace fdmap
