// walk_count_sum.cu -- walk kernels instantiated for the image of 'integrate' plus the segments per ray (first pass of
// the detailed projection).
#include "walk_kernels.cuh"

namespace vt {

int launch_count_sum(vt_cloud* cl, WalkIO& io, int kernel, cudaStream_t st) {
  return launch_sum<kOutCount>(cl, io, kernel, st);
}

}  // namespace vt
