// walkio.h -- arguments of one walk launch (shared by the kernels in
// project.cu and the host entry points in api.cu).
#pragma once

#include <cstdint>

#include "../../include/vortrace_b200.h"
#include "common.cuh"

struct vt_cloud;

namespace vt {

// kOutTape: the image of 'integrate' or 'volume' plus one tape entry per segment
constexpr int kOutImage = 0, kOutCount = 1, kOutFill = 2, kOutAdj = 3, kOutTape = 4;

// One segment of a taped forward: the adjoint of 'integrate' needs only
// the cell (original-order internal id), the ray and the segment length.
struct TapeEntry {
  int32_t pid;
  int32_t ray;
  double ds;
};
// One segment of a taped 'volume' forward: the cell (tree index), the ray,
// the segment length, the transmittance in front of the segment and the
// composited colour up to and including it -- what the reverse-mode
// compositing adjoint needs besides the fields and the final colour.
struct TapeEntryV {
  int32_t cell;
  int32_t ray;
  double ds;
  double T;
  double P[3];
};
constexpr int kErrNonFinite = 16;

struct WalkDiag;

struct WalkIO {
  const double* starts;  // nrays x 3, device
  const double* ends;    // nrays x 3, device
  int64_t nrays;
  int nout;              // values per ray (3 for volume, else nfields)
  double* out;           // image: nrays x nout
  int64_t* counts;       // count: segments per ray
  const int64_t* offsets;  // fill: CSR offsets
  int64_t* seg_cell;
  double* seg_enter;
  double* seg_exit;
  const double* gout;    // adjoint: upstream gradient, nrays x nout
  const double* fwd;     // adjoint: forward output (volume)
  double* grad;          // adjoint: npart x nfields, accumulated
  DevStats* stats;
  unsigned long long* slow_q;  // handed-over rays: (ray << 24) | segments emitted
  int* gstack_id;              // global pending-point stacks of k_slow
  double* gstack_s;
  int gstack_cap;
  int slow_threads;
  int64_t max_iter;
  int local_cap;         // in-register stack entries per ray
  int cache_mode;        // batched kernel: 1 = neighbourhood cache on
  const int32_t* order;  // batched kernels: ray visiting order (NULL: 0..nrays-1)
  void* tape;            // kOutTape: entries [0, tape_cap) (TapeEntry, or TapeEntryV for volume)
  unsigned long long* tape_count;  // kOutTape: entries appended (may exceed tape_cap)
  unsigned long long tape_cap;
  WalkDiag* diag;
  int deferred;          // k_slow only, over the entries deferred for the
                         // reference-order tree (which is now built)
};

int run_walk(vt_cloud* cl, WalkIO& io, int out_kind, int mode, int kernel, cudaStream_t st,
             vt_stats* stats);

// Launchers of the walk kernels, one translation unit each (walk_*.cu):
// image / count (segments per ray) of 'integrate' and of the other
// reductions, CSR fill, taped forward ('integrate' or 'volume') and the
// re-walk adjoint ('integrate' or 'volume').
int launch_image_sum(vt_cloud* cl, WalkIO& io, int kernel, cudaStream_t st);
int launch_image_vmm(vt_cloud* cl, WalkIO& io, int mode, int kernel, cudaStream_t st);
int launch_count_sum(vt_cloud* cl, WalkIO& io, int kernel, cudaStream_t st);
int launch_count_vmm(vt_cloud* cl, WalkIO& io, int mode, int kernel, cudaStream_t st);
int launch_fill(vt_cloud* cl, WalkIO& io, int kernel, cudaStream_t st);
int launch_tape(vt_cloud* cl, WalkIO& io, int mode, int kernel, cudaStream_t st);
int launch_adj(vt_cloud* cl, WalkIO& io, int mode, int kernel, cudaStream_t st);

}  // namespace vt
