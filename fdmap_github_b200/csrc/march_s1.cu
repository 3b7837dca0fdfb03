// March kernel variants of tile shape 1 (see march_host.cuh).
#include "march_host.cuh"

namespace fdmap {

int march_configure_s1(fdmap_gpu* h) { return march_configure_shape<1>(h); }
int march_launch_s1(fdmap_gpu* h, const StageArgs& a) { return march_launch_shape<1>(h, a); }
int march_batch_s1(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s) {
  return march_batch_shape<1>(proto, a, p, s);
}

}  // namespace fdmap
