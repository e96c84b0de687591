// walk_fill.cu -- walk kernels instantiated for the CSR segment lists (second pass of the detailed projection).
#include "walk_kernels.cuh"

namespace vt {

int launch_fill(vt_cloud* cl, WalkIO& io, int kernel, cudaStream_t st) {
  return launch_walk_t<kSum, 1, kOutFill>(cl, io, kernel, st);
}

}  // namespace vt
