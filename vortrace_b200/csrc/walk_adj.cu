// walk_adj.cu -- walk kernels instantiated for the re-walk adjoint of 'integrate' and 'volume'.
#include "walk_kernels.cuh"

namespace vt {

int launch_adj(vt_cloud* cl, WalkIO& io, int mode, int kernel, cudaStream_t st) {
  if (mode == kVolume) return launch_walk_t<kVolume, 4, kOutAdj>(cl, io, kernel, st);
  return launch_sum<kOutAdj>(cl, io, kernel, st);
}

}  // namespace vt
