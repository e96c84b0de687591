// walk_image_sum.cu -- walk kernels instantiated for the image of 'integrate'.
#include "walk_kernels.cuh"

namespace vt {

int launch_image_sum(vt_cloud* cl, WalkIO& io, int kernel, cudaStream_t st) {
  return launch_sum<kOutImage>(cl, io, kernel, st);
}

}  // namespace vt
