// March kernel variants of tile shape 3 (see march_host.cuh).
#include "march_host.cuh"

namespace fdmap {

int march_configure_s3(fdmap_gpu* h) { return march_configure_shape<3>(h); }
int march_launch_s3(fdmap_gpu* h, const StageArgs& a) { return march_launch_shape<3>(h, a); }
int march_batch_s3(const fdmap_gpu* proto, const StageArgs& a, const BatchPlan& p, cudaStream_t s) {
  return march_batch_shape<3>(proto, a, p, s);
}

}  // namespace fdmap
