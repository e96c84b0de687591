// common.cuh -- device-side types shared by the tree build, the k-NN
// searches and the walk kernels of libvortrace_b200.
//
// HBM layout of a built cloud (all arrays in *tree order*: the order of the
// implicit tree's leaves, see tree_build.cu):
//   pts     double4[n]   (x, y, z, unused)            32 B / point, one sector
//   pts32   float4[n]    (p - origin) in FP32, w = 0  16 B / point
//   nodes   double2[L-1] {divlow | split dim in the two low mantissa bits
//                         (rounded up), divhigh}      16 B / internal node;
//                         one pad entry in front, so that the sibling pair
//                         2i+1, 2i+2 is one aligned 32-byte sector
//   nodes32 float2[L-1]  {divlow rounded up | dim, divhigh rounded down},
//                         relative to origin           8 B / internal node;
//                         allocated with one pad entry in front, so that the
//                         sibling pair 2i+1, 2i+2 is one aligned 16-byte chunk
//   perm    int32[n]     tree index -> internal (filtered) point id
//   fields  double[n*nf] per-point fields, tree order
// The tree is implicit: internal node i has children 2i+1 and 2i+2, the
// L = 2^depth leaves follow the L-1 internal nodes, and leaf j holds the
// points [(j*n)>>depth, ((j+1)*n)>>depth).
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

namespace vt {

// Constants of the reference walk (src/ray.cpp:8-12, :321)
constexpr double kTol = 1e-9;
constexpr double kParallelTol = 1e-12;
constexpr double kPerturbEps = 2 * kTol;
constexpr int kMaxPerturbCycles = 1000;
constexpr int kExpandK = 100;
constexpr int kMaxDepth = 30;  // internal tree levels supported

// status codes (include/vortrace_b200.h)
constexpr int kErrMaxIter = 10;
constexpr int kErrSplitBounds = 11;
constexpr int kErrBinSearch = 12;
constexpr int kErrPerturb = 13;
constexpr int kErrKnnExpand = 14;
constexpr int kErrStack = 15;
constexpr int kErrNonFiniteDist = 17;  // squared distances overflowed
constexpr int kErrPeriodicBisect = 18;  // no second cell on a periodic same-cell ray
// internal: the ray must be finished by the degenerate-geometry kernel
constexpr int kNeedSlow = 99;
// internal: a 1-NN query met an exact tie and the reference-order tree is
// not available in this kernel (or not built yet); the ray is finished by
// k_slow, after the tree is built if need be
constexpr int kNeedTie = 98;
// status: an exact tie could not be resolved in the reference's order
constexpr int kErrTie = 19;
// 1-NN result: exact tie at the nearest distance, not resolved
constexpr int kTieUnresolved = -2;

enum Mode { kSum = 0, kMax = 1, kMin = 2, kVolume = 3 };

// One node of the reference-order tree (tietree.cu): nanoflann's Node
// (include/nanoflann.hpp:755-768) with explicit child indices.  feat < 0: a
// leaf holding index-array slots [a, b); else split dimension `feat`,
// children a (values <= lo) and b (values >= hi).
struct __align__(16) TieNode {
  double lo, hi;
  int32_t feat, a, b, pad;
};
// deepest reference-order tree the tie-resolving search supports
constexpr int kTieMaxDepth = 96;
// points per SoA leaf block (DevCloud::leaf32)
#ifndef VT_LEAF_SLOTS
#define VT_LEAF_SLOTS 8
#endif
constexpr int kLeafSlots = VT_LEAF_SLOTS;

struct DevCloud {
  const double4* __restrict__ pts;
  const float4* __restrict__ pts32;
  const double2* __restrict__ nodes;
  const float2* __restrict__ nodes32;
  const int32_t* __restrict__ perm;
  // the negated pts32 values of each leaf as SoA blocks of kLeafSlots
  // points (-x[8], -y[8], -z[8]: 96 B, 3 sectors per leaf, -inf past the
  // leaf's end) for the guarded-FP32 leaf scans, which form q - p as the
  // packed sum q + (-p); NULL when a leaf holds more points
  const float4* __restrict__ leaf32;
  const double* __restrict__ fields;
  // tight FP32 boxes (of the pts32 values) of every heap node, internal
  // nodes first then leaves: node i in [0, 2L-1)
  const float4* __restrict__ boxlo;
  const float4* __restrict__ boxhi;
  int64_t n;
  int64_t nleaves;  // 2^depth
  int nf;
  int depth;
  double bblo[3], bbhi[3];  // tight box of all points (nanoflann root_bbox)
  double origin[3];         // frame of pts32 / nodes32
  float bblo32[3], bbhi32[3];  // root box in that frame, rounded outward
  float coord_err;          // bound on |pts32 - (p - origin)| per component
  // periodic domain (src/pointcloud.cpp:26-32): the subbox and its side lengths
  int periodic;
  double sub_lo[3], sub_hi[3], box[3];
  // reference-order tree (tietree.cu); NULL until an exact tie needs it
  const TieNode* __restrict__ tt_nodes;
  const double4* __restrict__ tt_pts;
  const int32_t* __restrict__ tt_tid;
  double tt_lo[3], tt_hi[3];  // its root box (computeBoundingBox)
};

// ---- FP64 arithmetic with the reference's rounding (no FMA contraction) --
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// nanoflann L2_Simple_Adaptor::evalMetric (include/nanoflann.hpp:432-439):
// ((0 + d0*d0) + d1*d1) + d2*d2, d = q - p.  0 + x == x exactly.
__device__ __forceinline__ double metric(double qx, double qy, double qz, double4 p) {
  double d0 = dsub(qx, p.x), d1 = dsub(qy, p.y), d2 = dsub(qz, p.z);
  return dadd(dadd(dmul(d0, d0), dmul(d1, d1)), dmul(d2, d2));
}

// read-only 32-byte point load (two 16-byte halves of one sector)
__device__ __forceinline__ double4 ldg_pt(const double4* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  const double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ int node_dim(double lo) {
  return (int)(__double_as_longlong(lo) & 3);
}
__device__ __forceinline__ int node_dim32(float lo) { return (int)(__float_as_uint(lo) & 3u); }

__device__ __forceinline__ void leaf_range(const DevCloud& c, int64_t leaf, int64_t& a,
                                           int64_t& b) {
  a = (leaf * c.n) >> c.depth;
  b = ((leaf + 1) * c.n) >> c.depth;
}

// FP32 squared distance from q to the box [lo, hi] (0 inside) and to a
// point, with the same rounding steps: for every FP32 point p inside the
// box each per-axis gap is at most |q - p| (FP32 subtraction is monotone),
// so box_dist32 <= pt_dist32 for all points of the box.
__device__ __forceinline__ float box_dist32(float q0, float q1, float q2, float4 lo, float4 hi) {
  const float a = q0 < lo.x ? __fsub_rn(lo.x, q0) : (q0 > hi.x ? __fsub_rn(q0, hi.x) : 0.f);
  const float b = q1 < lo.y ? __fsub_rn(lo.y, q1) : (q1 > hi.y ? __fsub_rn(q1, hi.y) : 0.f);
  const float c = q2 < lo.z ? __fsub_rn(lo.z, q2) : (q2 > hi.z ? __fsub_rn(q2, hi.z) : 0.f);
  return __fadd_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)), __fmul_rn(c, c));
}

__device__ __forceinline__ float pt_dist32(float q0, float q1, float q2, float4 p) {
  const float a = __fsub_rn(q0, p.x), b = __fsub_rn(q1, p.y), c = __fsub_rn(q2, p.z);
  return __fadd_rn(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b)), __fmul_rn(c, c));
}

// Per-launch counters (atomically accumulated, warp-aggregated).
struct DevStats {
  unsigned long long rays;
  unsigned long long crossings;
  unsigned long long queries;
  unsigned long long fp64_resolves;
  unsigned long long slow_rays;
  unsigned long long max_stack;
  unsigned long long first_error;  // (ray << 8) | code, ~0 when none
  unsigned long long slow_count;   // rays queued for the degenerate kernel
  unsigned long long next_ray;     // work-queue head of the batched kernel
  unsigned long long next_slow;    // work-queue head of the degenerate kernel
  unsigned long long search_steps;     // nodes (groups) the searches expanded
  unsigned long long fp64_checks;      // FP64 re-checks of FP32-passing points
  unsigned long long cache_refreshes;  // neighbourhood-cache refills (k_warp)
  unsigned long long cache_hits;       // split queries answered from the cache
  unsigned long long ties;             // 1-NN queries that met an exact tie
  unsigned long long tie_deferred;     // rays waiting for the reference-order tree
  unsigned long long recheck_queries;  // guarded-FP32 queries with >= 1 FP64 re-check
  unsigned long long fp32_queries;     // guarded-FP32 split queries
  // counters build: per-warp cycles before / in / after the split search of
  // a loop trip, and search-loop steps of the warps and of all their lanes
  unsigned long long trip_cycles[3];
  unsigned long long search_warp_steps, search_lane_steps;
};

// Sum a small per-lane value over the active lanes, one atomic per warp.
__device__ __forceinline__ void warp_add(unsigned long long* p, unsigned v) {
  unsigned mask = __activemask();
  unsigned s = __reduce_add_sync(mask, v);
  if ((int)(threadIdx.x & 31) == __ffs(mask) - 1 && s) atomicAdd(p, (unsigned long long)s);
}

__device__ __forceinline__ void warp_max(unsigned long long* p, unsigned v) {
  unsigned mask = __activemask();
  unsigned s = __reduce_max_sync(mask, v);
  if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) atomicMax(p, (unsigned long long)s);
}

}  // namespace vt
