// walk_tape.cu -- walk kernels instantiated for the taped forward of 'integrate' and 'volume'.
#include "walk_kernels.cuh"

namespace vt {

int launch_tape(vt_cloud* cl, WalkIO& io, int mode, int kernel, cudaStream_t st) {
  if (mode == kVolume) return launch_walk_t<kVolume, 4, kOutTape>(cl, io, kernel, st);
  return launch_sum<kOutTape>(cl, io, kernel, st);
}

}  // namespace vt
