// walk_image_vmm.cu -- walk kernels instantiated for the images of 'volume', 'max' and 'min'.
#include "walk_kernels.cuh"

namespace vt {

int launch_image_vmm(vt_cloud* cl, WalkIO& io, int mode, int kernel, cudaStream_t st) {
  return launch_vmm<kOutImage>(cl, io, mode, kernel, st);
}

}  // namespace vt
