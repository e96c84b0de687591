// walk_count_vmm.cu -- walk kernels instantiated for the images of 'volume', 'max' and 'min' plus the segments per ray
// (first pass of the detailed projection).
#include "walk_kernels.cuh"

namespace vt {

int launch_count_vmm(vt_cloud* cl, WalkIO& io, int mode, int kernel, cudaStream_t st) {
  return launch_vmm<kOutCount>(cl, io, mode, kernel, st);
}

}  // namespace vt
