// batched.cuh -- persistent walk kernel with bounded, guarded-FP32 k-NN.
//
// Same walk as walk_ray() (src/ray.cpp:187-430) restructured for SIMD
// efficiency:
//   * persistent grid (a multiple of the SM count); every lane owns one ray;
//     a warp takes the next 32 rays of the coherent ray order (io.order, see
//     sort_rays) from a global atomic queue once all its lanes are done, so
//     the 32 rays of a warp are spatial neighbours whose searches visit the
//     same nodes, and many projections / arbitrary rays share one launch;
//   * one loop trip = one walk iteration per lane, so all lanes issue the
//     same k-NN search code;
//   * the split-point query is a *bounded* 3-NN: the two cells c and n whose
//     bisector holds the split point are known, so the search starts with
//     radius^2 R = max(d_c, d_n) + 4*TOL.  Every walk decision depends only
//     on points with r^2 < R (proof in knn3_decision_valid), otherwise the
//     query is re-resolved with an unbounded FP64 search;
//   * guarded FP32: descent and distance tests run on FP32 copies (nodes32,
//     pts32) with outward-rounded bounds; a point passes the FP32 test if
//     f < thr64 + G where G bounds |f - d| (FP32 rounding of coordinates and
//     arithmetic); every passing point is re-checked with its FP64 distance
//     in the reference's operation order, so results are exact;
//   * the top tree levels live in shared memory;
//   * rare paths (parallel bisector fallback, Case 1a, 100-NN expansion) run
//     inline in non-inlined functions; a pending-point stack deeper than the
//     in-register one hands the ray to k_slow with the number of segments
//     already emitted.
#pragma once

namespace vt {

constexpr int kBatchStack = 32;
// resident blocks per SM the batched kernel is compiled for (register cap).
// The guarded-FP32 search is compiled twice.  Launches with many rays per
// resident thread run it at 9 blocks of 128 threads (56 registers): more
// warps hide more of the dependent load latency than the extra spills cost
// (clustered_2m, 1M rays, 5 / 7 / 8 / 9 / 10 / 12 blocks -> 1088 / 1131 /
// 1150 / 1156 / 1060 / 427 Mcrossings/s; nested_16m, 4M rays, 1172 / 1278 /
// 1327 / 1342 / 1240 / 460).  Launches with fewer rays than
// VT_BATCHED_WIDE_RAYS_PER_THREAD per resident thread of that occupancy run
// it at 5 blocks (96 registers): there each warp gets few batches, the
// launch's tail dominates and the faster thread wins (volume_2m, 262,144
// rays: 788 at 5 blocks, 674 at 9; uniform_100k, 16,384 rays: 180 / 171).
// The FP64 search runs best at 4 blocks (128 registers: 822 against 768 /
// 714 / 707 at 5 / 6 / 8 blocks on clustered_2m).
#ifndef VT_BATCHED_MINB
#define VT_BATCHED_MINB 9
#endif
#ifndef VT_BATCHED_MINB_FEW
#define VT_BATCHED_MINB_FEW 5
#endif
#ifndef VT_BATCHED_WIDE_RAYS_PER_THREAD
#define VT_BATCHED_WIDE_RAYS_PER_THREAD 3
#endif
#ifndef VT_BATCHED_MINB64
#define VT_BATCHED_MINB64 4
#endif
// points per batch of distances in a leaf scan of the FP32 search (leaves
// without SoA blocks) / of the FP64 search (0: one at a time)
#ifndef VT_LEAF_BATCH
#define VT_LEAF_BATCH 4
#endif
static_assert(VT_LEAF_BATCH > 0, "the FP32 leaf scan loads points in batches");
// 1: at a node just above the leaves both leaves are scanned in turn, the
// farther one without a stack entry
#ifndef VT_LEAF_PAIR
#define VT_LEAF_PAIR 1
#endif
// 1: the FP32 search keeps its newest stack entry in registers
#ifndef VT_STACK_TOP
#define VT_STACK_TOP 1
#endif
// 1: the SoA leaf scan re-checks its passing slots through a bit mask
#ifndef VT_LEAF_MASK
#define VT_LEAF_MASK 1
#endif
// 1: the FP32 leaf scans read the SoA leaf blocks (DevCloud::leaf32)
#ifndef VT_LEAF_SOA
#define VT_LEAF_SOA 1
#endif
#ifndef VT_LEAF_BATCH64
#define VT_LEAF_BATCH64 4
#endif
// 1: the launch statistics also count the tree nodes the searches visit
// (search_steps), the FP64 re-checks of FP32-passing points other than the
// two cells of the split (fp64_checks), the guarded-FP32 split queries
// (fp32_queries) and those among them with at least one such re-check
// (recheck_queries); off by default, the counters cost registers (a build
// of the library with them on is made beside the default one)
#ifndef VT_BATCHED_COUNTERS
#define VT_BATCHED_COUNTERS 0
#endif

// ---- node fetch (shared memory for the top levels) ----------------------
struct Fetch64 {
  const double2* __restrict__ sm;
  const double2* __restrict__ g;
  int nsm;
  __device__ __forceinline__ double2 operator()(int64_t i) const {
    return i < nsm ? sm[i] : __ldg(&g[i]);
  }
};
struct Fetch32 {
  const float2* __restrict__ sm;
  const float2* __restrict__ g;
  int nsm;
  __device__ __forceinline__ float2 operator()(int64_t i) const {
    return i < nsm ? sm[i] : __ldg(&g[i]);
  }
  __device__ __forceinline__ float2 operator()(int i) const {
    return i < nsm ? sm[i] : __ldg(&g[i]);
  }
};

// Exact FP64 search with node fetch functor (same algorithm as knn_exact64).
template <class List, class F>
__device__ __forceinline__ void knn64_fetch(const DevCloud& c, const F& fetch, double qx,
                                            double qy, double qz, double bound, List& res,
                                            unsigned& nvisit) {
  const double q[3] = {qx, qy, qz};
  double off[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (q[d] < c.bblo[d]) off[d] = dmul(dsub(q[d], c.bblo[d]), dsub(q[d], c.bblo[d]));
    if (q[d] > c.bbhi[d]) off[d] = dmul(dsub(q[d], c.bbhi[d]), dsub(q[d], c.bbhi[d]));
  }
  double thr = fmin(bound, res.worst());
  const int64_t ninternal = c.nleaves - 1;
  int node = 0;
  int sp = 0;
  int s_node[kMaxDepth + 2];
  float s_mind[kMaxDepth + 2];
  float s_off[kMaxDepth + 2][3];
  unsigned visits = 0;
  for (;;) {
    ++visits;
    if (node < ninternal) {
      const double2 nd = fetch(node);
      const int dim = node_dim(nd.x);
      const double val = q[dim];
      const double diff1 = dsub(val, nd.x);
      const double diff2 = dsub(val, nd.y);
      const int first = 2 * node + 1;
      int best, other;
      double cut;
      if (dadd(diff1, diff2) < 0) {
        best = first;
        other = first + 1;
        cut = dmul(diff2, diff2);
      } else {
        best = first + 1;
        other = first;
        cut = dmul(diff1, diff1);
      }
      const double o0 = dim == 0 ? cut : off[0];
      const double o1 = dim == 1 ? cut : off[1];
      const double o2 = dim == 2 ? cut : off[2];
      const double nm = dmul(dadd(dadd(o0, o1), o2), 0.9999999999999991);
      if (nm < thr) {
        s_node[sp] = other;
        s_mind[sp] = __double2float_rd(nm);
        s_off[sp][0] = __double2float_rd(o0);
        s_off[sp][1] = __double2float_rd(o1);
        s_off[sp][2] = __double2float_rd(o2);
        ++sp;
      }
      node = best;
      continue;
    }
    {
      int64_t a, b;
      leaf_range(c, node - ninternal, a, b);
#if VT_LEAF_BATCH64
      // FP64 distances of up to VT_LEAF_BATCH64 points first (their loads in
      // flight together), then the tests in point order
      for (int64_t p0 = a; p0 < b; p0 += VT_LEAF_BATCH64) {
        double db[VT_LEAF_BATCH64];
#pragma unroll
        for (int j = 0; j < VT_LEAF_BATCH64; ++j) {
          db[j] = __longlong_as_double(0x7ff0000000000000ULL);
          if (p0 + j < b) db[j] = metric(qx, qy, qz, ldg_pt(&c.pts[p0 + j]));
        }
#pragma unroll
        for (int j = 0; j < VT_LEAF_BATCH64; ++j) {
          if (db[j] < thr) {
            res.insert(db[j], (int)(p0 + j));
            thr = fmin(bound, res.worst());
          }
        }
      }
#else
      for (int64_t p = a; p < b; ++p) {
        const double d = metric(qx, qy, qz, ldg_pt(&c.pts[p]));
        if (d < thr) {
          res.insert(d, (int)p);
          thr = fmin(bound, res.worst());
        }
      }
#endif
    }
    bool found = false;
    while (sp > 0) {
      --sp;
      if ((double)s_mind[sp] < thr) {
        node = s_node[sp];
        off[0] = s_off[sp][0];
        off[1] = s_off[sp][1];
        off[2] = s_off[sp][2];
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  nvisit += visits;
}

// Guarded FP32 bounded search, top-down from the root (nanoflann's
// searchLevel order: nearer child first, the farther one deferred on a
// per-thread stack if its bound is below the threshold).  Accepts points
// with FP64 distance d < R, keeps the 3 nearest (stable insertion).  G
// (guard_band) bounds |f - d| for every point with d < R, where f is the
// FP32 distance from pts32; a point with f < thr64 + G is re-checked with
// its FP64 distance.  Node bounds are FP32 lower bounds of f for every
// point of a subtree: per-axis offsets to the split planes (nodes32:
// divlow rounded up, divhigh rounded down), summed with monotone rounding.
// dc/dn: the known FP64 distances of the cells cid/nid (no reload).
template <class F>
__device__ __forceinline__ void knn3_guarded(const DevCloud& c, const F& fetch, double qx,
                                             double qy, double qz, int cid, int nid, double dc,
                                             double dn, double R, double G, KnnList<3>& res,
                                             unsigned& nvisit, unsigned& nverify,
                                             unsigned& nqverify) {
  const float q0 = __double2float_rn(dsub(qx, c.origin[0]));
  const float q1 = __double2float_rn(dsub(qy, c.origin[1]));
  const float q2 = __double2float_rn(dsub(qz, c.origin[2]));
  res.clear();
  double thr64 = R;
  float thr32 = __double2float_ru(dadd(thr64, G));
  // per-axis offsets start at the squared distance to the cloud's box
  // (nanoflann's computeInitialDistances, include/nanoflann.hpp:1005-1022):
  // a query outside the box (rays that start or end outside the cloud)
  // prunes with it.  bblo32/bbhi32 are rounded outward and the offsets
  // rounded down, so they stay below every point's FP32 offset.
  float off[3];
  {
    const float qd[3] = {q0, q1, q2};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float t = 0.f;
      if (qd[d] < c.bblo32[d]) t = __fsub_rd(c.bblo32[d], qd[d]);
      else if (qd[d] > c.bbhi32[d]) t = __fsub_rd(qd[d], c.bbhi32[d]);
      off[d] = __fmul_rd(t, t);
    }
  }
  // 32-bit node and point indices (the tree holds < 2^31 points): the
  // 64-bit compares and address arithmetic cost 2% of the walk
  const int ninternal = (int)(c.nleaves - 1);
  int node = 0;
  int sp = 0;
  int s_node[kMaxDepth + 2];
  float s_off[kMaxDepth + 2][3];
  float s_mind[kMaxDepth + 2];
#if VT_STACK_TOP
  // the newest deferred subtree is kept in registers: a push followed by
  // its pop (the far sibling after the near subtree) touches no local memory
  bool tos = false;
  int tos_node = 0;
  float tos_mind = 0.f, tos_o0 = 0.f, tos_o1 = 0.f, tos_o2 = 0.f;
#endif
  unsigned visits = 0, ver = 0;
  for (;;) {
    ++visits;
    // the leaves to scan next: the current node if it is a leaf, or both
    // children of a node just above the leaves (the nearer first, the other
    // while its bound stays below the threshold: no stack entry for it)
    int leaf0 = -1, leaf1 = -1;
    float nm1 = 0.f;
    if (node < ninternal) {
      const float2 nd = fetch(node);
      const int first = 2 * node + 1;
      const int dim = node_dim32(nd.x);
      const float val = dim == 0 ? q0 : (dim == 1 ? q1 : q2);
      int best, other;
      float o;
      if (__fadd_rn(__fsub_rn(val, nd.x), __fsub_rn(val, nd.y)) < 0.f) {
        best = first;
        other = first + 1;
        o = nd.y > val ? __fsub_rn(nd.y, val) : 0.f;  // right child: p >= hi32
      } else {
        best = first + 1;
        other = first;
        o = val > nd.x ? __fsub_rn(val, nd.x) : 0.f;  // left child: p <= lo32
      }
      const float t = __fmul_rn(o, o);
      const float o0 = dim == 0 ? fmaxf(t, off[0]) : off[0];
      const float o1 = dim == 1 ? fmaxf(t, off[1]) : off[1];
      const float o2 = dim == 2 ? fmaxf(t, off[2]) : off[2];
      const float nm = __fadd_rn(__fadd_rn(o0, o1), o2);
      if (VT_LEAF_PAIR && first >= ninternal) {
        leaf0 = best - ninternal;
        if (nm < thr32) {
          leaf1 = other - ninternal;
          nm1 = nm;
        }
      } else {
        if (nm < thr32) {
#if VT_STACK_TOP
          if (tos) {
            s_node[sp] = tos_node;
            s_mind[sp] = tos_mind;
            s_off[sp][0] = tos_o0;
            s_off[sp][1] = tos_o1;
            s_off[sp][2] = tos_o2;
            ++sp;
          }
          tos = true;
          tos_node = other;
          tos_mind = nm;
          tos_o0 = o0;
          tos_o1 = o1;
          tos_o2 = o2;
#else
          s_node[sp] = other;
          s_mind[sp] = nm;
          s_off[sp][0] = o0;
          s_off[sp][1] = o1;
          s_off[sp][2] = o2;
          ++sp;
#endif
        }
        node = best;
        continue;
      }
    } else {
      leaf0 = node - ninternal;
    }
#pragma unroll 1
    for (int lt = 0; lt < 2; ++lt) {
      const int leaf = lt == 0 ? leaf0 : leaf1;
      if (leaf < 0 || (lt == 1 && !(nm1 < thr32))) break;
      int a, b;
      {
        int64_t a64, b64;
        leaf_range(c, leaf, a64, b64);
        a = (int)a64;
        b = (int)b64;
      }
      // a passing FP32 distance f of tree point p: FP64 re-check, insertion
      auto test_point = [&](int p, float f) {
        if (f < thr32) {
          double d;
          if (p == cid) d = dc;
          else if (p == nid) d = dn;
          else {
            d = metric(qx, qy, qz, ldg_pt(&c.pts[p]));
            ++ver;
          }
          if (d < thr64) {
            res.insert(d, p);
            thr64 = fmin(R, res.worst());
            thr32 = __double2float_ru(dadd(thr64, G));
          }
        }
      };
      if (VT_LEAF_SOA && c.leaf32) {
        // the leaf's SoA block: 3 * kLeafSlots / 4 independent 16-byte
        // loads (8 slots: six loads, three sectors); distances of all slots
        // first, then the tests in point order (slots past the leaf's end
        // hold -inf: their distance is +inf and never passes)
        constexpr int Q = kLeafSlots / 4;  // float4 per coordinate
        const float4* blk = c.leaf32 + (int64_t)leaf * (3 * Q);
        float4 v[3 * Q];
#pragma unroll
        for (int u = 0; u < 3 * Q; ++u) v[u] = __ldg(blk + u);
        // distances two slots at a time with the packed FP32 operations of
        // sm_100 (each half rounds as the scalar operation): e = q + (-p),
        // f = ((ex^2 + ey^2) + ez^2), the order of pt_dist32
        float fb[kLeafSlots];
        const float2 qx2 = make_float2(q0, q0), qy2 = make_float2(q1, q1),
                     qz2 = make_float2(q2, q2);
#pragma unroll
        for (int h = 0; h < kLeafSlots / 2; ++h) {
          const float4 X = v[h / 2], Y = v[Q + h / 2], Z = v[2 * Q + h / 2];
          const float2 px = (h & 1) ? make_float2(X.z, X.w) : make_float2(X.x, X.y);
          const float2 py = (h & 1) ? make_float2(Y.z, Y.w) : make_float2(Y.x, Y.y);
          const float2 pz = (h & 1) ? make_float2(Z.z, Z.w) : make_float2(Z.x, Z.y);
          const float2 ex = __fadd2_rn(qx2, px), ey = __fadd2_rn(qy2, py),
                       ez = __fadd2_rn(qz2, pz);
          const float2 f2 = __fadd2_rn(__fadd2_rn(__fmul2_rn(ex, ex), __fmul2_rn(ey, ey)),
                                       __fmul2_rn(ez, ez));
          fb[2 * h] = f2.x;
          fb[2 * h + 1] = f2.y;
        }
#if VT_LEAF_MASK
        // the slots under the threshold as a mask, then one FP64 re-check per
        // set bit in slot order: lanes re-check their t-th passing point
        // together.  A point that passed against the leaf's starting
        // threshold but not against a threshold lowered by an insertion
        // before it has f >= thr64 + G, hence d >= thr64, and the FP64 test
        // rejects it, as the one-by-one scan would have skipped it.
        unsigned pass = 0;
#pragma unroll
        for (int k = 0; k < kLeafSlots; ++k) pass |= (fb[k] < thr32 ? 1u : 0u) << k;
        while (pass) {
          const int k = __ffs(pass) - 1;
          pass &= pass - 1;
          const int p = a + k;
          double d;
          if (p == cid) d = dc;
          else if (p == nid) d = dn;
          else {
            d = metric(qx, qy, qz, ldg_pt(&c.pts[p]));
            ++ver;
          }
          if (d < thr64) {
            res.insert(d, p);
            thr64 = fmin(R, res.worst());
            thr32 = __double2float_ru(dadd(thr64, G));
          }
        }
#else
#pragma unroll
        for (int k = 0; k < kLeafSlots; ++k) test_point(a + k, fb[k]);
#endif
      } else {
        // the FP32 distances of up to VT_LEAF_BATCH points first (independent
        // loads in flight together), then the tests in point order
        for (int p0 = a; p0 < b; p0 += VT_LEAF_BATCH) {
          float fb[VT_LEAF_BATCH];
#pragma unroll
          for (int k = 0; k < VT_LEAF_BATCH; ++k) {
            fb[k] = __int_as_float(0x7f800000);
            if (p0 + k < b) fb[k] = pt_dist32(q0, q1, q2, __ldg(&c.pts32[p0 + k]));
          }
#pragma unroll
          for (int k = 0; k < VT_LEAF_BATCH; ++k) test_point(p0 + k, fb[k]);
        }
      }
    }
    bool found = false;
#if VT_STACK_TOP
    if (tos) {
      tos = false;
      if (tos_mind < thr32) {
        node = tos_node;
        off[0] = tos_o0;
        off[1] = tos_o1;
        off[2] = tos_o2;
        found = true;
      }
    }
    if (!found)
#endif
    while (sp > 0) {
      --sp;
      if (s_mind[sp] < thr32) {
        node = s_node[sp];
        off[0] = s_off[sp][0];
        off[1] = s_off[sp][1];
        off[2] = s_off[sp][2];
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  nvisit += visits;
  nverify += ver;
  nqverify += ver > 0;
}

// A bounded result B (all points with d < R, at most 3, exact order) gives
// the same walk decisions as the unbounded 3-NN T when:
//   * |B| == 3 (then B == T), or
//   * |B| >= 1 and fl(R - r2[0]) >= TOL and fl(r2[0] + TOL) < R: every
//     missing entry of T has r2 >= R, so by monotone rounding the loop
//     "r2[i] - r2[0] >= TOL" breaks at the same i and "r2[0] + TOL < r2[1]"
//     has the same truth value.
__device__ __forceinline__ bool knn3_decision_valid(const KnnList<3>& r, double R) {
  const int cnt = r.count();
  if (cnt == 3) return true;
  if (cnt == 0) return false;
  return dsub(R, r.r2[0]) >= kTol && dadd(r.r2[0], kTol) < R;
}

// G(R) bounds |f - d| for every point with d < R, where f is the FP32
// distance between the FP32 images of q and p (frame origin subtracted,
// each coordinate within e of the exact offset) and d the FP64 metric:
// X = 3.5 e sqrt(R) + 3 e^2 bounds the change of the squared distance from
// the coordinate errors, 6u (R + X) the FP32 rounding of the three
// subtractions, three squares and two additions (u = 2^-24), 1e-15 R the
// FP64 rounding of d, and the factor 1.02 leaves slack.
__device__ __forceinline__ double guard_band(double R, double e) {
  const double u = 5.9604644775390625e-08;  // 2^-24
  const double sr = sqrt(R);
  const double cross = 3.5 * e * sr + 3.0 * e * e;
  return 1.02 * (6.0 * u * (R + cross) + cross + 1e-15 * R);
}

// ------------------------------------------------- rare paths, not inlined
struct RareOut {
  double s;
  int rc, a, b;
  unsigned nq;
};

// Parallel-bisector fallback of the split point (src/ray.cpp:96-126).
static __device__ __noinline__ RareOut rare_split(const DevCloud& c, RayGeom g, int cur, int nxt,
                                           double cur_s, double nxt_s) {
  Search64 S(c);
  RareOut o{0.0, 0, 0, 0, 0u};
  o.rc = split_full(c, g, S, cur, nxt, cur_s, nxt_s, o.s);
  o.nq = S.nq;
  return o;
}

// Case 1a (src/ray.cpp:364-422): intermediate cells on both sides.
static __device__ __noinline__ RareOut rare_case1a(const DevCloud& c, RayGeom g, double x, double y,
                                            double z, int cur, int nxt) {
  Search64 S(c);
  int sc = try_along_ray(g, S, x, y, z, -1.0, cur, nxt);
  if (sc < 0) {
    const double ex = dmul(kPerturbEps, g.d[0]), ey = dmul(kPerturbEps, g.d[1]),
                 ez = dmul(kPerturbEps, g.d[2]);
    sc = perp_perturb(g, S, dsub(x, ex), dsub(y, ey), dsub(z, ez), cur, nxt);
  }
  int sn = -1;
  if (sc >= 0) {
    sn = try_along_ray(g, S, x, y, z, 1.0, cur, nxt);
    if (sn < 0) {
      const double ex = dmul(kPerturbEps, g.d[0]), ey = dmul(kPerturbEps, g.d[1]),
                   ez = dmul(kPerturbEps, g.d[2]);
      sn = perp_perturb(g, S, dadd(x, ex), dadd(y, ey), dadd(z, ez), cur, nxt);
    }
  }
  const int rc = (sc == kTieUnresolved || sn == kTieUnresolved) ? kNeedTie
                 : (sc < 0 || sn < 0)                             ? kErrPerturb
                                                                  : 0;
  RareOut o{0.0, rc, sc, sn, S.nq};
  return o;
}

// 100-NN classification (src/ray.cpp:319-338).
static __device__ __noinline__ RareOut rare_expand(const DevCloud& c, double x, double y, double z,
                                            int cur, int nxt) {
  bool has_c = false, has_n = false;
  unsigned v = 0;
  RareOut o{0.0, 0, 0, 0, 1u};
  o.rc = expand_classify(c, x, y, z, cur, nxt, has_c, has_n, v);
  o.a = has_c;
  o.b = has_n;
  return o;
}

// --------------------------------------------------------------- kernel
template <int MODE, int NF, int OUT, bool G32, int MINB>
__global__ void __launch_bounds__(128, MINB) k_batched(DevCloud c, WalkIO io, int nsm) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // stage the top tree levels
  if (G32) {
    // one pad entry in front, as in the global array: siblings share a
    // 16-byte pair
    float2* s = reinterpret_cast<float2*>(smem_raw) + 1;
    for (int i = threadIdx.x; i < nsm; i += blockDim.x) s[i] = c.nodes32[i];
  } else {
    double2* s = reinterpret_cast<double2*>(smem_raw) + 1;  // pad entry, as in HBM
    for (int i = threadIdx.x; i < nsm; i += blockDim.x) s[i] = c.nodes[i];
  }
  __syncthreads();
  const Fetch64 f64{reinterpret_cast<const double2*>(smem_raw) + 1, c.nodes, G32 ? 0 : nsm};
  const Fetch32 f32{reinterpret_cast<const float2*>(smem_raw) + 1, c.nodes32, G32 ? nsm : 0};

  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const double cerr = (double)c.coord_err;

  // per-lane ray state
  int64_t ray = -1;
  int phase = 0;  // 0 idle, 1 start query, 2 end query, 3 walking
  bool exhausted = false;
  RayGeom g;
  int c0 = -1, cur = -1, open_cell = -1, nxt = -1;
  double cur_s = 0.0, entry_s = 0.0, nxt_s = 0.0, s_split = 0.0;
  int64_t iter = 0;
  LocalStack<kBatchStack> st;
  st.set_cap(io.local_cap);
  st.clear();
  double q_err = 0.0;
  // sinks
  std::conditional_t<OUT == kOutTape, TapeReducer<MODE, NF, true>, Reducer<MODE, NF>> red;
  FillSink fill;
  AdjSink<MODE, NF> adj;
  // lane counters
  unsigned n_rays = 0, n_cross = 0, n_q = 0, n_res = 0, n_visit = 0, n_ver = 0, max_sp = 0;
  unsigned n_qver = 0, n_q32 = 0;

#if VT_BATCHED_COUNTERS
  // trip profile (lane 0): cycles before the search (refill + walk logic),
  // in the search, after it (apply + tape); search-loop steps of the
  // warp (its longest search per trip) and of all lanes
  unsigned long long cyc_pre = 0, cyc_search = 0, cyc_post = 0, wsteps = 0, lsteps = 0;
#endif
  for (;;) {
#if VT_BATCHED_COUNTERS
    const long long t_trip = clock64();
#endif
    // ---- refill idle lanes from the work queue
    // a warp takes 32 consecutive rays (of the coherent order) once all its
    // lanes are idle: neighbouring rays visit the same tree nodes, so the
    // lanes' searches stay convergent and share cache lines
    const bool want = __all_sync(FULL, phase == 0) && !exhausted;
    const unsigned need = __ballot_sync(FULL, want);
    if (need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(&io.stats->next_ray, (unsigned long long)__popc(need));
      base = __shfl_sync(FULL, base, leader);
      if (want) {
        const int64_t i = (int64_t)base + __popc(need & ((1u << lane) - 1));
        if (i < io.nrays) {
          const int64_t r = io.order ? (int64_t)io.order[i] : i;
          ray = r;
          ray_init(g, io.starts + 3 * r, io.ends + 3 * r);
          if (!ray_finite(g)) {
            report(io, r, kErrNonFinite);
          } else {
            phase = 1;
            ++n_rays;
            if (OUT == kOutImage || OUT == kOutCount || OUT == kOutTape)
              red.init(&c, io.out + r * io.nout);
            if constexpr (OUT == kOutTape) red.set_tape(&io, r, 0u);
            else if (OUT == kOutFill) fill.init(&c, io, r);
            else adj.init(&c, io, r, 0u);
            double m = 0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j)
              m = fmax(m, fmax(fabs(g.s[j] - c.origin[j]), fabs(g.e[j] - c.origin[j])));
            q_err = m * 6.0e-8 + cerr;
          }
        } else {
          exhausted = true;
        }
      }
    }
    if (__all_sync(FULL, phase == 0 && exhausted)) break;

    unsigned nseg_now = 0;
    auto nseg_of = [&]() -> unsigned {
      if (OUT == kOutImage || OUT == kOutCount || OUT == kOutTape) return red.nseg;
      if (OUT == kOutFill) return fill.nseg;
      return adj.nseg;
    };
    auto emit = [&](int cell, double a, double b) {
      if (OUT == kOutImage || OUT == kOutCount || OUT == kOutTape) red.seg(cell, a, b);
      else if (OUT == kOutFill) fill.seg(cell, a, b);
      else adj.seg(cell, a, b);
    };
    auto finish_ok = [&]() {
      if (OUT == kOutImage || OUT == kOutCount || OUT == kOutTape) {
        red.write(io.out + ray * io.nout);
        if (OUT == kOutCount) io.counts[ray] = red.nseg;
      }
      n_cross += nseg_of();
      max_sp = max(max_sp, (unsigned)st.maxsp);
      phase = 0;
    };
    auto fail = [&](int rc) {
      if (rc == kNeedSlow || rc == kNeedTie) hand_over(io, ray, nseg_of());
      else report(io, ray, rc);
      max_sp = max(max_sp, (unsigned)st.maxsp);
      phase = 0;
    };
    (void)nseg_now;

    // ---- prepare this lane's query
    int qkind = 0;  // 0 none, 1 nearest neighbour (FP64), 2 bounded 3-NN
    double qx = 0, qy = 0, qz = 0, dc = 0, dn = 0, R = 0;
    if (phase == 1) {
      qx = g.s[0]; qy = g.s[1]; qz = g.s[2];
      qkind = 1;
    } else if (phase == 2) {
      qx = g.e[0]; qy = g.e[1]; qz = g.e[2];
      qkind = 1;
    } else if (phase == 3) {
      for (;;) {
        if (++iter > io.max_iter) {
          fail(kErrMaxIter);
          break;
        }
        nxt = st.top_id();
        nxt_s = st.top_s();
        if (dsub(nxt_s, cur_s) < 1e-14) {  // zero-width skip
          st.pop();
          cur = nxt;
          cur_s = nxt_s;
          open_cell = cur;
          if (st.empty()) {
            emit(open_cell, entry_s, cur_s);
            finish_ok();
            break;
          }
          continue;
        }
        const double4 pc = ldg_pt(&c.pts[cur]);
        const double4 pn = ldg_pt(&c.pts[nxt]);
        double s = split_analytic(g, pc, pn);
        if (!(s < DBL_MAX * 0.5 && s >= cur_s - kTol && s <= nxt_s + kTol)) {
          // parallel bisector: bisection with nearest-neighbour queries
          const RareOut ro = rare_split(c, g, cur, nxt, cur_s, nxt_s);
          n_q += ro.nq;
          s = ro.s;
          if (ro.rc) {
            fail(ro.rc);
            break;
          }
          if (s < dsub(cur_s, kTol) || s > dadd(nxt_s, kTol)) {
            fail(kErrSplitBounds);
            break;
          }
        }
        {
          const double lo = dadd(cur_s, 1e-15), hi = dsub(nxt_s, 1e-15);
          s = (s < lo) ? lo : (hi < s) ? hi : s;
        }
        s_split = s;
        ray_point(g, s, qx, qy, qz);
        dc = metric(qx, qy, qz, pc);
        dn = metric(qx, qy, qz, pn);
        R = dadd(fmax(dc, dn), 4.0 * kTol);
        qkind = 2;
        break;
      }
    }

    // ---- search (lanes of one kind run the same code)
#if VT_BATCHED_COUNTERS
    const long long t_search = clock64();
    const unsigned visit0 = n_visit;
#endif
    KnnList<3> r;
    if (qkind == 1) {
      r.clear();
      ++n_q;
      knn64_fetch(c, f64, qx, qy, qz, pinf(), r, n_visit);
    } else if (qkind == 2) {
      ++n_q;
      if (G32) {
        const double G = guard_band(R, q_err);
        knn3_guarded(c, f32, qx, qy, qz, cur, nxt, dc, dn, R, G, r, n_visit, n_ver, n_qver);
        ++n_q32;
      } else {
        r.clear();
        knn64_fetch(c, f64, qx, qy, qz, R, r, n_visit);
      }
      if (!knn3_decision_valid(r, R)) {
        ++n_res;
        r.clear();
        knn64_fetch(c, f64, qx, qy, qz, pinf(), r, n_visit);
      }
    }

#if VT_BATCHED_COUNTERS
    const long long t_apply = clock64();
    {
      const unsigned my = qkind == 2 ? n_visit - visit0 : 0u;
      const unsigned mx = __reduce_max_sync(FULL, my);
      const unsigned sm = __reduce_add_sync(FULL, my);
      if (lane == 0) {
        wsteps += mx;
        lsteps += sm;
        cyc_pre += (unsigned long long)(t_search - t_trip);
        cyc_search += (unsigned long long)(t_apply - t_search);
      }
    }
#endif
    // ---- apply
    if (qkind != 0 && r.id[0] < 0) {
      fail(kErrNonFiniteDist);  // squared distances overflowed
    } else if (qkind == 1 && r.id[1] >= 0 && r.r2[1] == r.r2[0]) {
      fail(kNeedTie);  // exactly tied nearest cells: resolved in k_slow
    } else if (qkind == 1 && phase == 1) {
      c0 = r.id[0];
      phase = 2;
    } else if (qkind == 1 && phase == 2) {
      const int c1 = r.id[0];
      if (c0 == c1) {
        emit(c0, 0.0, g.len);
        finish_ok();
      } else {
        st.clear();
        st.push(c1, g.len);
        cur = c0;
        cur_s = 0.0;
        open_cell = c0;
        entry_s = 0.0;
        iter = 0;
        phase = 3;
      }
    } else if (qkind == 2) {
      bool has_c = false, has_n = false, three_eq = true;
#pragma unroll
      for (int i = 0; i < 3; i++) {
        if (dsub(r.r2[i], r.r2[0]) >= kTol) {
          three_eq = false;
          break;
        }
        if (r.id[i] == cur) has_c = true;
        if (r.id[i] == nxt) has_n = true;
      }
      bool expand_failed = false;
      if (three_eq && !has_c && !has_n) {
        const RareOut ro = rare_expand(c, qx, qy, qz, cur, nxt);
        n_q += ro.nq;
        if (ro.rc) {
          fail(ro.rc);
          expand_failed = true;
        }
        has_c = ro.a;
        has_n = ro.b;
      }
      if (expand_failed) {
      } else if (has_c || has_n) {
        emit(open_cell, entry_s, s_split);
        open_cell = nxt;
        entry_s = s_split;
        st.pop();
        cur = nxt;
        cur_s = nxt_s;
        if (st.empty()) {
          emit(open_cell, entry_s, cur_s);
          finish_ok();
        }
      } else if (dadd(r.r2[0], kTol) < r.r2[1]) {
        if (st.room() < 1) fail(kNeedSlow);
        else st.push(r.id[0], s_split);
      } else {
        const RareOut ro = rare_case1a(c, g, qx, qy, qz, cur, nxt);
        n_q += ro.nq;
        const int sc = ro.a, sn = ro.b;
        if (ro.rc) fail(ro.rc);
        else if (sc == sn) {
          if (st.room() < 1) fail(kNeedSlow);
          else st.push(sc, s_split);
        } else if (st.room() < 2) {
          fail(kNeedSlow);
        } else {
          st.push(sn, s_split);
          st.push(sc, s_split);
        }
      }
    }
    // every lane reaches the end of a trip: write this trip's tape entries
    if constexpr (OUT == kOutTape) red.flush_tape(io);
#if VT_BATCHED_COUNTERS
    __syncwarp();
    if (lane == 0) cyc_post += (unsigned long long)(clock64() - t_apply);
#endif
  }
  warp_add(&io.stats->rays, n_rays);
  warp_add(&io.stats->crossings, n_cross);
  warp_add(&io.stats->queries, n_q);
  warp_add(&io.stats->fp64_resolves, n_res);
  warp_max(&io.stats->max_stack, max_sp);
#if VT_BATCHED_COUNTERS
  warp_add(&io.stats->search_steps, n_visit);
  warp_add(&io.stats->fp64_checks, n_ver);
  warp_add(&io.stats->recheck_queries, n_qver);
  warp_add(&io.stats->fp32_queries, n_q32);
  if (lane == 0) {
    atomicAdd(&io.stats->trip_cycles[0], cyc_pre);
    atomicAdd(&io.stats->trip_cycles[1], cyc_search);
    atomicAdd(&io.stats->trip_cycles[2], cyc_post);
    atomicAdd(&io.stats->search_warp_steps, wsteps);
    atomicAdd(&io.stats->search_lane_steps, lsteps);
  }
#endif
}

// The register cap of the guarded-FP32 kernel for a launch of nrays rays on
// nsms SMs (see VT_BATCHED_MINB); the FP64 kernel has one.
inline int batched_minb(bool g32, int64_t nrays, int nsms) {
  if (!g32) return VT_BATCHED_MINB64;
  const int64_t wide = (int64_t)VT_BATCHED_WIDE_RAYS_PER_THREAD * nsms * VT_BATCHED_MINB * 128;
  return nrays >= wide ? VT_BATCHED_MINB : VT_BATCHED_MINB_FEW;
}

template <int MODE, int NF, int OUT>
int launch_batched(vt_cloud* cl, WalkIO& io, int kernel, cudaStream_t st) {
  const bool g32 = kernel == VT_KERNEL_THREAD_FP32;
  const int64_t ninternal = cl->view.nleaves - 1;
  int64_t want = (1LL << cl->smem_levels) - 1;
  int nsm = (int)(want < ninternal ? want : ninternal);
  if (nsm < 0) nsm = 0;
  const size_t smem = (size_t)(nsm + 1) * (g32 ? sizeof(float2) : sizeof(double2));
  const int B = 128;
  int dev = 0, nsms = 0;
  VT_CUDA(cudaGetDevice(&dev));
  VT_CUDA(cudaDeviceGetAttribute(&nsms, cudaDevAttrMultiProcessorCount, dev));
  const int minb = batched_minb(g32, io.nrays, nsms);
  auto kfun = !g32 ? k_batched<MODE, NF, OUT, false, VT_BATCHED_MINB64>
              : minb == VT_BATCHED_MINB ? k_batched<MODE, NF, OUT, true, VT_BATCHED_MINB>
                                        : k_batched<MODE, NF, OUT, true, VT_BATCHED_MINB_FEW>;
  if (smem > 48 * 1024)
    VT_CUDA(cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // a set (or tuned) occupancy above the kernel's register cap cannot be
  // resident: clamp it
  int per_sm = cl->blocks_per_sm < minb ? cl->blocks_per_sm : minb;
  if (per_sm <= 0) {
    VT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfun, B, smem));
    if (per_sm < 1) per_sm = 1;
  }
  int64_t blocks = (int64_t)nsms * per_sm;
  const int64_t need = (io.nrays + B - 1) / B;
  if (blocks > need) blocks = need > 0 ? need : 1;
  kfun<<<(unsigned)blocks, B, smem, st>>>(cl->view, io, nsm);
  return VT_OK;
}

}  // namespace vt
