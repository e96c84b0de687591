// tree_build.cu -- device build of the implicit, left-balanced k-d tree.
//
// Replaces PointCloud::buildTree / nanoflann buildIndex (src/pointcloud.cpp:
// 193-212, include/nanoflann.hpp:858-1003, 1190-1202).  The tree differs
// from nanoflann's by design (median splits, implicit layout); its k-NN
// answers are the same exact sets (see knn.cuh).
//
// Build, all on the device:
//   1. tight bounding box of the points (block reduction + 64-bit atomics
//      on order-preserving integer images of the coordinates);
//   2. 63-bit Morton codes in that box, radix sort -> spatially coherent
//      initial order;
//   3. for each level l = 0..depth-1 (2^l segments, segment k = points
//      [(k*n)>>l, ((k+1)*n)>>l)):
//        a. per-segment bounding boxes (warp-aggregated atomics),
//        b. split dimension = widest extent of the segment's points,
//        c. stable radix sort of (coordinate along the split dim) then a
//           stable radix sort of the segment ids: every segment is now
//           ordered along its own split dimension,
//        d. node k of the level: divlow = largest coordinate of the left
//           half, divhigh = smallest of the right half (split at the
//           median position ((2k+1)*n)>>(l+1));
//   4. tree-order copies: pts (double4), pts32 (float4 relative to the box
//      centre), fields, perm (tree index -> internal id), and the FP32
//      node copy rounded outward.
#include <cub/cub.cuh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace vt {

__device__ __forceinline__ unsigned long long ord_key(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __forceinline__ double ord_val(unsigned long long k) {
  unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
  return __longlong_as_double((long long)b);
}

__global__ void k_split_aos(const double* __restrict__ aos, int64_t n, double* x, double* y,
                            double* z, int32_t* perm) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = aos[3 * i];
  y[i] = aos[3 * i + 1];
  z[i] = aos[3 * i + 2];
  perm[i] = (int32_t)i;
}

// Per-segment min/max of x,y,z at level `lvl` (segments contiguous).  bb
// holds 6 ord keys per segment: min x,y,z (atomicMin) then max x,y,z.
__global__ void k_seg_bbox(const double* __restrict__ x, const double* __restrict__ y,
                           const double* __restrict__ z, int64_t n, int lvl,
                           unsigned long long* bb) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool valid = i < n;
  int64_t ii = valid ? i : n - 1;
  int64_t seg = ((((ii + 1) << lvl) - 1) / n);
  unsigned long long k[6];
  k[0] = k[3] = ord_key(x[ii]);
  k[1] = k[4] = ord_key(y[ii]);
  k[2] = k[5] = ord_key(z[ii]);
  unsigned full = __ballot_sync(0xffffffffu, true);
  int64_t seg0 = __shfl_sync(full, seg, 0);
  int64_t seg31 = __shfl_sync(full, seg, 31);
  if (seg0 == seg31) {
    // whole warp in one segment (padding lanes repeat the last point)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        unsigned long long a = __shfl_xor_sync(full, k[j], o);
        unsigned long long b = __shfl_xor_sync(full, k[j + 3], o);
        k[j] = a < k[j] ? a : k[j];
        k[j + 3] = b > k[j + 3] ? b : k[j + 3];
      }
    }
    if ((threadIdx.x & 31) == 0) {
      unsigned long long* p = bb + 6 * seg;
      for (int j = 0; j < 3; ++j) {
        atomicMin(p + j, k[j]);
        atomicMax(p + 3 + j, k[j + 3]);
      }
    }
  } else if (valid) {
    unsigned long long* p = bb + 6 * seg;
    for (int j = 0; j < 3; ++j) {
      atomicMin(p + j, k[j]);
      atomicMax(p + 3 + j, k[j + 3]);
    }
  }
}

__global__ void k_bb_init(unsigned long long* bb, int64_t nseg) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nseg) return;
  for (int j = 0; j < 3; ++j) {
    bb[6 * i + j] = ~0ULL;
    bb[6 * i + 3 + j] = 0ULL;
  }
}

// Split dimension per segment: widest point extent, lowest dim on ties.
__global__ void k_seg_dim(const unsigned long long* __restrict__ bb, int64_t nseg,
                          uint8_t* dim) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= nseg) return;
  int best = 0;
  double bw = -1.0;
  for (int j = 0; j < 3; ++j) {
    double w = ord_val(bb[6 * k + 3 + j]) - ord_val(bb[6 * k + j]);
    if (w > bw) {
      bw = w;
      best = j;
    }
  }
  dim[k] = (uint8_t)best;
}

__global__ void k_keys(const double* __restrict__ x, const double* __restrict__ y,
                       const double* __restrict__ z, int64_t n, int lvl,
                       const uint8_t* __restrict__ dim, unsigned long long* key, uint32_t* seg,
                       int32_t* val) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t s = ((((i + 1) << lvl) - 1) / n);
  int d = dim[s];
  double v = d == 0 ? x[i] : (d == 1 ? y[i] : z[i]);
  key[i] = ord_key(v);
  seg[i] = (uint32_t)s;
  val[i] = (int32_t)i;
}

__global__ void k_gather_seg(const uint32_t* __restrict__ seg, const int32_t* __restrict__ idx,
                             int64_t n, uint32_t* out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = seg[idx[i]];
}

__global__ void k_gather_pts(const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, const int32_t* __restrict__ perm,
                             const int32_t* __restrict__ idx, int64_t n, double* x2, double* y2,
                             double* z2, int32_t* perm2) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int32_t j = idx[i];
  x2[i] = x[j];
  y2[i] = y[j];
  z2[i] = z[j];
  perm2[i] = perm[j];
}

// smallest double >= v whose two low mantissa bits equal dim
__device__ double pack_dim_up(double v, int dim) {
  for (int it = 0; it < 8; ++it) {
    if ((int)(__double_as_longlong(v) & 3) == dim) return v;
    v = nextafter(v, __longlong_as_double(0x7ff0000000000000LL));
  }
  return v;
}
__device__ float pack_dim_up32(float v, int dim) {
  for (int it = 0; it < 8; ++it) {
    if ((int)(__float_as_uint(v) & 3u) == dim) return v;
    v = nextafterf(v, __int_as_float(0x7f800000));
  }
  return v;
}

// Nodes of level `lvl` from the points already ordered at this level.
__global__ void k_level_nodes(const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, int64_t n, int lvl,
                              const uint8_t* __restrict__ dim, double ox, double oy, double oz,
                              double2* nodes, float2* nodes32) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t nseg = 1LL << lvl;
  if (k >= nseg) return;
  int d = dim[k];
  int64_t m = ((2 * k + 1) * n) >> (lvl + 1);
  const double* c = d == 0 ? x : (d == 1 ? y : z);
  double o = d == 0 ? ox : (d == 1 ? oy : oz);
  double lo = c[m - 1], hi = c[m];
  int64_t node = (nseg - 1) + k;
  nodes[node] = make_double2(pack_dim_up(lo, d), hi);
  float lo32 = __double2float_ru(__dsub_rn(lo, o));
  float hi32 = __double2float_rd(__dsub_rn(hi, o));
  nodes32[node] = make_float2(pack_dim_up32(lo32, d), hi32);
}

__global__ void k_morton(const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, int64_t n, double lx, double ly,
                         double lz, double sx, double sy, double sz, unsigned long long* key,
                         int32_t* val) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  auto q = [](double v, double lo, double s) -> unsigned long long {
    double t = (v - lo) * s;
    t = fmin(fmax(t, 0.0), 2097151.0);
    return (unsigned long long)t;
  };
  auto spread = [](unsigned long long v) -> unsigned long long {
    v &= 0x1fffffULL;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
  };
  key[i] = spread(q(x[i], lx, sx)) | (spread(q(y[i], ly, sy)) << 1) |
           (spread(q(z[i], lz, sz)) << 2);
  val[i] = (int32_t)i;
}

__global__ void k_finalize(const double* __restrict__ x, const double* __restrict__ y,
                           const double* __restrict__ z, int64_t n, double ox, double oy,
                           double oz, double4* pts, float4* pts32) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a = x[i], b = y[i], c = z[i];
  pts[i] = make_double4(a, b, c, 0.0);
  pts32[i] = make_float4(__double2float_rn(__dsub_rn(a, ox)), __double2float_rn(__dsub_rn(b, oy)),
                         __double2float_rn(__dsub_rn(c, oz)), 0.f);
}

__global__ void k_fields_tree(const double* __restrict__ f_in, const int32_t* __restrict__ perm,
                              int64_t n, int nf, double* f_out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * nf) return;
  int64_t p = i / nf;
  int f = (int)(i - p * nf);
  f_out[i] = f_in[(int64_t)perm[p] * nf + f];
}

static inline unsigned nblk(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

// Tight boxes of the FP32 point copies: leaves from their points ...
// SoA leaf blocks of the negated FP32 points: block j = 6 float4 {-x[0..3],
// -x[4..7], -y[0..3], -y[4..7], -z[0..3], -z[4..7]} of leaf j, -inf past its
// end (negation is exact, and q + (-p) rounds as q - p).
__global__ void k_leaf_soa(const float4* __restrict__ pts32, int64_t n, int depth,
                           int64_t nleaves, float4* __restrict__ out) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= nleaves) return;
  const int64_t a = (j * n) >> depth, b = ((j + 1) * n) >> depth;
  float v[3][kLeafSlots];
  for (int k = 0; k < kLeafSlots; ++k) {
    const bool in = a + k < b;
    const float4 p = in ? pts32[a + k] : make_float4(0.f, 0.f, 0.f, 0.f);
    v[0][k] = in ? -p.x : -INFINITY;
    v[1][k] = in ? -p.y : -INFINITY;
    v[2][k] = in ? -p.z : -INFINITY;
  }
  constexpr int Q = kLeafSlots / 4;  // float4 per coordinate
  float4* o = out + j * 3 * Q;
  for (int d = 0; d < 3; ++d)
    for (int q = 0; q < Q; ++q)
      o[Q * d + q] = make_float4(v[d][4 * q], v[d][4 * q + 1], v[d][4 * q + 2], v[d][4 * q + 3]);
}

__global__ void k_leaf_boxes(const float4* __restrict__ pts32, int64_t n, int depth,
                             int64_t nleaves, float4* lo, float4* hi) {
  int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= nleaves) return;
  const int64_t a = (j * n) >> depth, b = ((j + 1) * n) >> depth;
  float4 l = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
  float4 h = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
  for (int64_t p = a; p < b; ++p) {
    const float4 v = pts32[p];
    l.x = fminf(l.x, v.x); l.y = fminf(l.y, v.y); l.z = fminf(l.z, v.z);
    h.x = fmaxf(h.x, v.x); h.y = fmaxf(h.y, v.y); h.z = fmaxf(h.z, v.z);
  }
  lo[nleaves - 1 + j] = l;
  hi[nleaves - 1 + j] = h;
}

// ... internal nodes of one level as the union of their children.
__global__ void k_level_boxes(int lvl, float4* lo, float4* hi) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= (1LL << lvl)) return;
  const int64_t i = (1LL << lvl) - 1 + k;
  const float4 a = lo[2 * i + 1], b = lo[2 * i + 2], c = hi[2 * i + 1], d = hi[2 * i + 2];
  lo[i] = make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), 0.f);
  hi[i] = make_float4(fmaxf(c.x, d.x), fmaxf(c.y, d.y), fmaxf(c.z, d.z), 0.f);
}

// valid_rgba over internal-order fields (src/pointcloud.cpp:167-179)
__global__ void k_rgba_check(const double* __restrict__ f, int64_t n, int* bad) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double r = f[4 * i], g = f[4 * i + 1], b = f[4 * i + 2], a = f[4 * i + 3];
  if (!(r >= 0.0 && r <= 1.0 && g >= 0.0 && g <= 1.0 && b >= 0.0 && b <= 1.0 && a >= 0.0))
    atomicOr(bad, 1);
}

// Replace the tree-order field array from internal-order values.
int upload_fields(vt_cloud* cl, const double* src, bool src_device, cudaStream_t st) {
  const int64_t n = (int64_t)cl->npart;
  const int nf = (int)cl->nfields;
  const int B = 256;
  DevBuf<double> fin;
  const double* dsrc = src;
  int rc;
  if (!src_device) {
    if ((rc = fin.alloc((size_t)n * nf))) return rc;
    VT_CUDA(cudaMemcpyAsync(fin.p, src, (size_t)n * nf * sizeof(double), cudaMemcpyHostToDevice,
                            st));
    dsrc = fin.p;
  }
  k_fields_tree<<<nblk((int64_t)n * nf, B), B, 0, st>>>(dsrc, cl->perm_d.p, n, nf,
                                                        cl->fields_d.p);
  VT_CUDA(cudaGetLastError());
  bool valid = false;
  if (nf == 4 && n > 0) {
    DevBuf<int> bad;
    if ((rc = bad.alloc(1))) return rc;
    VT_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    k_rgba_check<<<nblk(n, B), B, 0, st>>>(dsrc, n, bad.p);
    VT_CUDA(cudaGetLastError());
    int hb = 1;
    VT_CUDA(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    VT_CUDA(cudaStreamSynchronize(st));
    valid = hb == 0;
  } else {
    VT_CUDA(cudaStreamSynchronize(st));
  }
  cl->valid_rgba = valid;
  return VT_OK;
}

// Build the device tree of `cl` from its host points/fields.
// Tree-order point copies, node boxes, tree-order fields and the device
// view, from the permutation (tree index -> internal id), the node splits
// and the tree-ordered coordinates; shared by the build and the load of a
// saved tree.
static int finish_tree(vt_cloud* cl, int depth, const double lo[3], const double hi[3],
                       const double org[3], DevBuf<int32_t>& pa, DevBuf<double2>& nodes,
                       DevBuf<float2>& nodes32, const double* x, const double* y,
                       const double* z) {
  const int64_t n = (int64_t)cl->npart;
  const int nf = (int)cl->nfields;
  cudaStream_t st = cl->stream;
  const int B = 256;
  const int64_t nleaves = 1LL << depth;
  int rc;
#define VT_TRY(x)                      \
  do {                                 \
    if ((rc = (x)) != VT_OK) return rc; \
  } while (0)
  // tree-order copies
  DevBuf<double4> pts;
  DevBuf<float4> pts32;
  DevBuf<double> fields;
  VT_TRY(pts.alloc(n));
  VT_TRY(pts32.alloc(n));
  VT_TRY(fields.alloc((int64_t)n * nf));
  k_finalize<<<nblk(n, B), B, 0, st>>>(x, y, z, n, org[0], org[1], org[2], pts.p, pts32.p);
  DevBuf<float4> blo, bhi;
  // one pad entry in front (as the node arrays): sibling boxes 2i+1, 2i+2
  // share an aligned 32-byte sector
  VT_TRY(blo.alloc(2 * nleaves));
  VT_TRY(bhi.alloc(2 * nleaves));
  k_leaf_boxes<<<nblk(nleaves, B), B, 0, st>>>(pts32.p, n, depth, nleaves, blo.p + 1,
                                                bhi.p + 1);
  // SoA leaf blocks when every leaf fits kLeafSlots points
  DevBuf<float4> lsoa;
  if (((n + nleaves - 1) >> depth) <= kLeafSlots) {
    VT_TRY(lsoa.alloc((int64_t)(3 * kLeafSlots / 4) * nleaves));
    k_leaf_soa<<<nblk(nleaves, B), B, 0, st>>>(pts32.p, n, depth, nleaves, lsoa.p);
  }
  for (int l = depth - 1; l >= 0; --l)
    k_level_boxes<<<nblk(1LL << l, B), B, 0, st>>>(l, blo.p + 1, bhi.p + 1);
  {
    // fields: upload in internal order into the (now free) aos buffer, gather
    DevBuf<double> fin;
    VT_TRY(fin.alloc((int64_t)n * nf));
    VT_CUDA(cudaMemcpyAsync(fin.p, cl->fields.data(), (size_t)n * nf * sizeof(double),
                            cudaMemcpyHostToDevice, st));
    k_fields_tree<<<nblk((int64_t)n * nf, B), B, 0, st>>>(fin.p, pa.p, n, nf, fields.p);
    VT_CUDA(cudaGetLastError());
    VT_CUDA(cudaStreamSynchronize(st));
  }
  // largest |p - origin| component, for the FP32 error bounds
  double mext = 0.0;
  for (int j = 0; j < 3; ++j) mext = fmax(mext, fmax(fabs(hi[j] - org[j]), fabs(lo[j] - org[j])));

  cl->perm_d = std::move(pa);
  cl->pts_d = std::move(pts);
  cl->pts32_d = std::move(pts32);
  cl->nodes_d = std::move(nodes);
  cl->nodes32_d = std::move(nodes32);
  cl->fields_d = std::move(fields);
  cl->boxlo_d = std::move(blo);
  cl->boxhi_d = std::move(bhi);
  cl->leaf32_d = std::move(lsoa);
  DevCloud& v = cl->view;
  v.pts = cl->pts_d.p;
  v.pts32 = cl->pts32_d.p;
  v.nodes = cl->nodes_d.p + 1;  // after the pad entry
  v.nodes32 = cl->nodes32_d.p + 1;  // after the pad entry
  v.perm = cl->perm_d.p;
  v.fields = cl->fields_d.p;
  v.boxlo = cl->boxlo_d.p + 1;  // after the pad entry
  v.boxhi = cl->boxhi_d.p + 1;
  v.leaf32 = cl->leaf32_d.p;  // NULL when not built (leaves above kLeafSlots)
  v.n = n;
  v.nleaves = nleaves;
  v.nf = nf;
  v.depth = depth;
  for (int j = 0; j < 3; ++j) {
    v.bblo[j] = lo[j];
    v.bbhi[j] = hi[j];
    v.origin[j] = org[j];
    // outward-rounded FP32 root box (all pts32 lie inside it)
    v.bblo32[j] = std::nextafter((float)(lo[j] - org[j]), -INFINITY);
    v.bbhi32[j] = std::nextafter((float)(hi[j] - org[j]), INFINITY);
    v.bblo32[j] = std::nextafter(v.bblo32[j], -INFINITY);
    v.bbhi32[j] = std::nextafter(v.bbhi32[j], INFINITY);
  }
  // |fl32(p - o) - (p - o)| <= 2^-24 |p - o| (plus the FP64 subtraction)
  v.coord_err = (float)(mext * 6.0e-8 + 1e-300);
  v.periodic = cl->periodic ? 1 : 0;
  for (int j = 0; j < 3; ++j) {
    v.sub_lo[j] = cl->subbox[2 * j];
    v.sub_hi[j] = cl->subbox[2 * j + 1];
    v.box[j] = cl->subbox[2 * j + 1] - cl->subbox[2 * j];
  }
  return VT_OK;
#undef VT_TRY
}

int build_tree_device(vt_cloud* cl) {
  const int64_t n = (int64_t)cl->npart;
  cudaStream_t st = cl->stream;
  const int B = 256;
  int depth = 0;
  while (((n + (1LL << depth) - 1) >> depth) > cl->leaf_size) ++depth;
  if (depth > kMaxDepth) return set_error(VT_ERR_INVALID, "point cloud too large for the tree");
  const int64_t nleaves = 1LL << depth;
  const int64_t ninternal = nleaves - 1;

  DevBuf<double> ax, bx, ay, by, az, bz;
  DevBuf<int32_t> pa, pb, va, vb;
  DevBuf<unsigned long long> ka, kb, bb;
  DevBuf<uint32_t> sa, sb;
  DevBuf<uint8_t> dims;
  DevBuf<double> aos;
  int rc;
#define VT_TRY(x)                      \
  do {                                 \
    if ((rc = (x)) != VT_OK) return rc; \
  } while (0)
  VT_TRY(aos.alloc(3 * n));
  VT_TRY(ax.alloc(n)); VT_TRY(bx.alloc(n)); VT_TRY(ay.alloc(n)); VT_TRY(by.alloc(n));
  VT_TRY(az.alloc(n)); VT_TRY(bz.alloc(n));
  VT_TRY(pa.alloc(n)); VT_TRY(pb.alloc(n)); VT_TRY(va.alloc(n)); VT_TRY(vb.alloc(n));
  VT_TRY(ka.alloc(n)); VT_TRY(kb.alloc(n)); VT_TRY(sa.alloc(n)); VT_TRY(sb.alloc(n));
  VT_TRY(bb.alloc(6 * (nleaves > 1 ? nleaves / 2 : 1)));
  VT_TRY(dims.alloc(nleaves > 1 ? nleaves / 2 : 1));

  VT_CUDA(cudaMemcpyAsync(aos.p, cl->pts.data(), 3 * n * sizeof(double), cudaMemcpyHostToDevice,
                          st));
  k_split_aos<<<nblk(n, B), B, 0, st>>>(aos.p, n, ax.p, ay.p, az.p, pa.p);

  // CUB temporary storage: max over the sorts used
  size_t tmp_bytes = 0, t1 = 0, t2 = 0;
  VT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, ka.p, kb.p, va.p, vb.p, (int)n, 0, 64, st));
  VT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t2, sa.p, sb.p, va.p, vb.p, (int)n, 0, 32, st));
  tmp_bytes = t1 > t2 ? t1 : t2;
  DevBuf<uint8_t> tmp;
  VT_TRY(tmp.alloc(tmp_bytes));

  // 1. bounding box of all points (one segment)
  k_bb_init<<<1, 32, 0, st>>>(bb.p, 1);
  k_seg_bbox<<<nblk(n, B), B, 0, st>>>(ax.p, ay.p, az.p, n, 0, bb.p);
  unsigned long long hb[6];
  VT_CUDA(cudaMemcpyAsync(hb, bb.p, sizeof(hb), cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  double lo[3], hi[3];
  for (int j = 0; j < 3; ++j) {
    auto back = [](unsigned long long k) {
      unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
      double v;
      memcpy(&v, &b, 8);
      return v;
    };
    lo[j] = back(hb[j]);
    hi[j] = back(hb[3 + j]);
  }
  double org[3];
  for (int j = 0; j < 3; ++j) org[j] = 0.5 * (lo[j] + hi[j]);

  // 2. Morton order
  {
    double sc[3];
    for (int j = 0; j < 3; ++j) {
      double w = hi[j] - lo[j];
      sc[j] = w > 0 ? 2097151.0 / w : 0.0;
    }
    k_morton<<<nblk(n, B), B, 0, st>>>(ax.p, ay.p, az.p, n, lo[0], lo[1], lo[2], sc[0], sc[1],
                                       sc[2], ka.p, va.p);
    VT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, ka.p, kb.p, va.p, vb.p, (int)n, 0,
                                            63, st));
    k_gather_pts<<<nblk(n, B), B, 0, st>>>(ax.p, ay.p, az.p, pa.p, vb.p, n, bx.p, by.p, bz.p,
                                           pb.p);
    std::swap(ax.p, bx.p); std::swap(ay.p, by.p); std::swap(az.p, bz.p); std::swap(pa.p, pb.p);
  }

  DevBuf<double2> nodes;
  DevBuf<float2> nodes32;
  VT_TRY(nodes.alloc(ninternal + 2));  // pad entry in front, as nodes32
  // one leading pad entry: the children pair (2i+1, 2i+2) of every node
  // then sits in one 16-byte aligned chunk, so a node and its sibling (the
  // deferred child the search visits later) share a sector (+3% on the
  // walk against pairs that straddle sectors)
  VT_TRY(nodes32.alloc(ninternal + 2));

  // 3. levels
  for (int l = 0; l < depth; ++l) {
    const int64_t nseg = 1LL << l;
    k_bb_init<<<nblk(nseg, B), B, 0, st>>>(bb.p, nseg);
    k_seg_bbox<<<nblk(n, B), B, 0, st>>>(ax.p, ay.p, az.p, n, l, bb.p);
    k_seg_dim<<<nblk(nseg, B), B, 0, st>>>(bb.p, nseg, dims.p);
    k_keys<<<nblk(n, B), B, 0, st>>>(ax.p, ay.p, az.p, n, l, dims.p, ka.p, sa.p, va.p);
    VT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, ka.p, kb.p, va.p, vb.p, (int)n, 0,
                                            64, st));
    const int32_t* order = vb.p;
    if (l > 0) {
      k_gather_seg<<<nblk(n, B), B, 0, st>>>(sa.p, vb.p, n, sb.p);
      VT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, sb.p, sa.p, vb.p, va.p, (int)n, 0,
                                              l, st));
      order = va.p;
    }
    k_gather_pts<<<nblk(n, B), B, 0, st>>>(ax.p, ay.p, az.p, pa.p, order, n, bx.p, by.p, bz.p,
                                           pb.p);
    std::swap(ax.p, bx.p); std::swap(ay.p, by.p); std::swap(az.p, bz.p); std::swap(pa.p, pb.p);
    k_level_nodes<<<nblk(nseg, B), B, 0, st>>>(ax.p, ay.p, az.p, n, l, dims.p, org[0], org[1],
                                               org[2], nodes.p + 1, nodes32.p + 1);
  }
  VT_CUDA(cudaGetLastError());

  return finish_tree(cl, depth, lo, hi, org, pa, nodes, nodes32, ax.p, ay.p, az.p);
#undef VT_TRY
}

// ------------------------------------------------------- saved trees
// Blob: TreeBlobHeader, then perm (int32 x n), nodes (double2 x L-1) and
// nodes32 (float2 x L-1).  The boxes, the tree-order copies and the fields
// are rebuilt from the cloud's own points, which must be the ones the tree
// was built on: the header keeps a hash of them.
struct TreeBlobHeader {
  char magic[8];
  uint32_t version;
  uint32_t depth;
  uint64_t n;
  uint64_t leaf_size;
  double lo[3], hi[3], org[3];
  uint64_t points_hash;
};
static const char kTreeMagic[8] = {'V', 'T', 'B', '2', 'T', 'R', 'E', 'E'};

// 64-bit hash of the filtered points (word-wise multiply-xor).
static uint64_t points_hash(const std::vector<double>& p) {
  uint64_t h = 1469598103934665603ULL;
  for (double v : p) {
    uint64_t w;
    memcpy(&w, &v, 8);
    h = (h ^ w) * 1099511628211ULL;
    h ^= h >> 29;
  }
  return h;
}

__global__ void k_gather_aos(const double* __restrict__ aos, const int32_t* __restrict__ perm,
                             int64_t n, double* x, double* y, double* z) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t p = perm[i];
  x[i] = aos[3 * p];
  y[i] = aos[3 * p + 1];
  z[i] = aos[3 * p + 2];
}

uint64_t tree_blob_size(const vt_cloud* cl) {
  const int64_t ni = cl->view.nleaves - 1;
  return sizeof(TreeBlobHeader) + (uint64_t)cl->npart * 4 + (uint64_t)ni * (16 + 8);
}

int save_tree_blob(vt_cloud* cl, void* buf) {
  TreeBlobHeader hd;
  memcpy(hd.magic, kTreeMagic, 8);
  hd.version = 1;
  hd.depth = (uint32_t)cl->view.depth;
  hd.n = cl->npart;
  hd.leaf_size = (uint64_t)cl->leaf_size;
  for (int j = 0; j < 3; ++j) {
    hd.lo[j] = cl->view.bblo[j];
    hd.hi[j] = cl->view.bbhi[j];
    hd.org[j] = cl->view.origin[j];
  }
  hd.points_hash = points_hash(cl->pts);
  uint8_t* out = static_cast<uint8_t*>(buf);
  memcpy(out, &hd, sizeof(hd));
  out += sizeof(hd);
  const int64_t ni = cl->view.nleaves - 1;
  cudaStream_t st = cl->stream;
  VT_CUDA(cudaMemcpyAsync(out, cl->perm_d.p, cl->npart * 4, cudaMemcpyDeviceToHost, st));
  out += cl->npart * 4;
  if (ni > 0) {
    VT_CUDA(cudaMemcpyAsync(out, cl->view.nodes, ni * 16, cudaMemcpyDeviceToHost, st));
    out += ni * 16;
    VT_CUDA(cudaMemcpyAsync(out, cl->view.nodes32, ni * 8, cudaMemcpyDeviceToHost, st));
  }
  VT_CUDA(cudaStreamSynchronize(st));
  return VT_OK;
}

int load_tree_blob(vt_cloud* cl, const void* buf, uint64_t size) {
  TreeBlobHeader hd;
  if (size < sizeof(hd)) return set_error(VT_ERR_INVALID, "tree blob too short");
  memcpy(&hd, buf, sizeof(hd));
  if (memcmp(hd.magic, kTreeMagic, 8) != 0)
    return set_error(VT_ERR_INVALID, "not a libvortrace_b200 tree blob");
  if (hd.version != 1) return set_error(VT_ERR_INVALID, "unsupported tree blob version");
  const int64_t n = (int64_t)cl->npart;
  if (hd.n != (uint64_t)n || hd.depth > (uint32_t)kMaxDepth ||
      ((n + (1LL << hd.depth) - 1) >> hd.depth) > (int64_t)hd.leaf_size || hd.leaf_size < 1)
    return set_error(VT_ERR_INVALID, "tree blob does not fit this point cloud");
  const int depth = (int)hd.depth;
  const int64_t ni = (1LL << depth) - 1;
  if (size != sizeof(hd) + (uint64_t)n * 4 + (uint64_t)ni * 24)
    return set_error(VT_ERR_INVALID, "tree blob has the wrong size");
  if (hd.points_hash != points_hash(cl->pts))
    return set_error(VT_ERR_INVALID, "tree blob was built on other points");
  const uint8_t* in = static_cast<const uint8_t*>(buf) + sizeof(hd);
  cudaStream_t st = cl->stream;
  const int B = 256;
  int rc;
  DevBuf<int32_t> pa;
  DevBuf<double2> nodes;
  DevBuf<float2> nodes32;
  DevBuf<double> aos, x, y, z;
  if ((rc = pa.alloc(n)) || (rc = nodes.alloc(ni + 2)) ||
      (rc = nodes32.alloc(ni + 2)) || (rc = aos.alloc(3 * n)) || (rc = x.alloc(n)) ||
      (rc = y.alloc(n)) || (rc = z.alloc(n)))
    return rc;
  VT_CUDA(cudaMemcpyAsync(pa.p, in, n * 4, cudaMemcpyHostToDevice, st));
  in += n * 4;
  if (ni > 0) {
    VT_CUDA(cudaMemcpyAsync(nodes.p + 1, in, ni * 16, cudaMemcpyHostToDevice, st));
    in += ni * 16;
    VT_CUDA(cudaMemcpyAsync(nodes32.p + 1, in, ni * 8, cudaMemcpyHostToDevice, st));
  }
  VT_CUDA(cudaMemcpyAsync(aos.p, cl->pts.data(), 3 * n * sizeof(double), cudaMemcpyHostToDevice,
                          st));
  k_gather_aos<<<nblk(n, B), B, 0, st>>>(aos.p, pa.p, n, x.p, y.p, z.p);
  VT_CUDA(cudaGetLastError());
  cl->leaf_size = (int)hd.leaf_size;
  return finish_tree(cl, depth, hd.lo, hd.hi, hd.org, pa, nodes, nodes32, x.p, y.p, z.p);
}

}  // namespace vt
