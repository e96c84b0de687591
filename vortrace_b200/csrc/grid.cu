// grid.cu -- pixel-centre ray grids generated on the device.
//
// Replaces the host-side ray generation of ProjectionCloud.grid_projection
// for grids without rotation (vortrace/grid.py:35-44 base grid, :100-192
// projection grid with center=None).  Each axis holds numpy.linspace over the
// pixel centres, evaluated with numpy's own steps (numpy/_core/function_base.py
// linspace: y = i*step + start, the last sample set to stop; i/div*delta when
// the step underflows to zero), so the rays are bit-identical to the host
// generator's: ray i*ny + j runs from (x_i, y_j, bounds[0]) to
// (x_i, y_j, bounds[1]).
#include "internal.h"

namespace vt {

namespace {

// one axis of numpy.linspace(start, stop, n) over the pixel centres of
// [lo, hi] in n pixels; the arithmetic is done in the host's IEEE double
// with the same operation order as the reference's generator
struct GridAxis {
  double start, stop, step, delta, div;
  int64_t n;
  int kind;  // 0: i*step + start; 1: (i/div)*delta + start; 2: 0*delta + start
};

GridAxis make_axis(double lo, double hi, int64_t n) {
  GridAxis a{};
  const double d = (hi - lo) / (double)n;  // vortrace/grid.py:39-40
  a.start = lo + 0.5 * d;
  a.stop = hi - 0.5 * d;
  a.n = n;
  a.delta = a.stop - a.start;
  a.div = (double)(n - 1);
  if (n - 1 > 0) {
    a.step = a.delta / a.div;
    a.kind = a.step == 0.0 ? 1 : 0;
  } else {
    a.kind = 2;
  }
  return a;
}

__device__ __forceinline__ double axis_at(const GridAxis& a, int64_t i) {
  if (a.n > 1 && i == a.n - 1) return a.stop;
  const double y = (double)i;
  double v;
  if (a.kind == 0) v = __dmul_rn(y, a.step);
  else if (a.kind == 1) v = __dmul_rn(__ddiv_rn(y, a.div), a.delta);
  else v = __dmul_rn(y, a.delta);
  return __dadd_rn(v, a.start);
}

__global__ void k_grid_rays(GridAxis ax, GridAxis ay, double z0, double z1, double* starts,
                            double* ends) {
  const int64_t n = ax.n * ay.n;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = r / ay.n, j = r - i * ay.n;
    const double x = axis_at(ax, i), y = axis_at(ay, j);
    starts[3 * r + 0] = x;
    starts[3 * r + 1] = y;
    starts[3 * r + 2] = z0;
    ends[3 * r + 0] = x;
    ends[3 * r + 1] = y;
    ends[3 * r + 2] = z1;
  }
}

}  // namespace

int launch_grid_rays(const double extent[4], uint64_t nx, uint64_t ny, const double bounds[2],
                     double* d_starts, double* d_ends, cudaStream_t st) {
  const GridAxis ax = make_axis(extent[0], extent[1], (int64_t)nx);
  const GridAxis ay = make_axis(extent[2], extent[3], (int64_t)ny);
  const int64_t n = (int64_t)(nx * ny);
  if (n == 0) return VT_OK;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (n + 255) / 256;
  const int blocks = (int)(want < 8LL * nsm ? want : 8LL * nsm);
  k_grid_rays<<<blocks, 256, 0, st>>>(ax, ay, bounds[0], bounds[1], d_starts, d_ends);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(VT_ERR_CUDA, std::string("grid ray kernel: ") + cudaGetErrorString(e));
  return VT_OK;
}

}  // namespace vt
