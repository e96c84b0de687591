// knn.cuh -- exact k-nearest-neighbour searches over the implicit tree.
//
// Results must equal the reference's nanoflann k-NN (include/nanoflann.hpp
// 1221-1241 findNeighbors, 1346-1408 searchLevel, 175-201 addPoint):
//   * squared distances are evaluated with the reference's operation order
//     (metric() in common.cuh), so r2 values are bit-identical;
//   * the result list is sorted ascending and a new point with a distance
//     equal to a listed one goes after it (strict '>' shift), points are
//     accepted only when d < current worst;
//   * pruning only ever uses lower bounds of the distance to a subtree, so
//     the returned set is exactly the k nearest; only the order in which
//     exactly tied points are met differs from nanoflann's (other tree).
// A search can be given an initial bound: points with d >= bound are never
// accepted (the result then holds the k nearest among those closer than the
// bound).
#pragma once

#include "common.cuh"

namespace vt {

// Fixed-capacity sorted list, unrolled insertion (registers for small K).
template <int K>
struct KnnList {
  double r2[K];
  int id[K];
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      r2[j] = __longlong_as_double(0x7ff0000000000000ULL);  // +inf
      id[j] = -1;
    }
  }
  __device__ __forceinline__ double worst() const { return r2[K - 1]; }
  // Stable insertion of (d, p); requires d < worst().
  __device__ __forceinline__ void insert(double d, int p) {
#pragma unroll
    for (int j = K - 1; j > 0; --j) {
      const double a = r2[j - 1], b = r2[j];
      const int ia = id[j - 1];
      if (a > d) {
        r2[j] = a;
        id[j] = ia;
      } else if (b > d) {
        r2[j] = d;
        id[j] = p;
      }
    }
    if (r2[0] > d) {
      r2[0] = d;
      id[0] = p;
    }
  }
  __device__ __forceinline__ int count() const {
    int c = 0;
#pragma unroll
    for (int j = 0; j < K; ++j) c += (id[j] >= 0);
    return c;
  }
  __device__ __forceinline__ int capacity() const { return K; }
  __device__ __forceinline__ void clear(int) { clear(); }
  __device__ __forceinline__ void set_count(int) {}
};

// Runtime-k list for the rare large queries (k up to KMAX, local memory).
template <int KMAX>
struct KnnBig {
  double r2[KMAX];
  int id[KMAX];
  int k, cnt;
  __device__ __forceinline__ void clear(int kk) {
    k = kk;
    cnt = 0;
  }
  __device__ __forceinline__ double worst() const {
    return cnt == k ? r2[k - 1] : __longlong_as_double(0x7ff0000000000000ULL);
  }
  __device__ void insert(double d, int p) {
    int i = cnt;
    for (; i > 0; --i) {
      if (r2[i - 1] > d) {
        if (i < k) {
          r2[i] = r2[i - 1];
          id[i] = id[i - 1];
        }
      } else
        break;
    }
    if (i < k) {
      r2[i] = d;
      id[i] = p;
    }
    if (cnt < k) ++cnt;
  }
  __device__ __forceinline__ int count() const { return cnt; }
  __device__ __forceinline__ int capacity() const { return k; }
  __device__ __forceinline__ void set_count(int n) { cnt = n; }
};

// Depth-first, nearer-child-first exact search (nanoflann's traversal on the
// implicit tree).  Deferred far children are kept on a small stack with
// FP32 lower bounds (rounded down) of their per-dimension box offsets.
template <class List>
__device__ __noinline__ void knn_exact64(const DevCloud& c, double qx, double qy, double qz,
                                         double bound, List& res, unsigned& nvisit) {
  const double q[3] = {qx, qy, qz};
  // include/nanoflann.hpp:1005-1021 computeInitialDistances
  double off[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (q[d] < c.bblo[d]) off[d] = dmul(dsub(q[d], c.bblo[d]), dsub(q[d], c.bblo[d]));
    if (q[d] > c.bbhi[d]) off[d] = dmul(dsub(q[d], c.bbhi[d]), dsub(q[d], c.bbhi[d]));
  }
  double thr = fmin(bound, res.worst());
  const int64_t ninternal = c.nleaves - 1;
  int64_t node = 0;
  int sp = 0;
  int64_t s_node[kMaxDepth + 2];
  float s_mind[kMaxDepth + 2];
  float s_off[kMaxDepth + 2][3];
  unsigned visits = 0;
  for (;;) {
    ++visits;
    if (node < ninternal) {
      const double2 nd = __ldg(&c.nodes[node]);
      const int dim = node_dim(nd.x);
      const double val = q[dim];
      const double diff1 = dsub(val, nd.x);
      const double diff2 = dsub(val, nd.y);
      const int64_t first = 2 * node + 1;
      int64_t best, other;
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
      // lower bound of the squared distance from q to `other`'s region
      double o0 = dim == 0 ? cut : off[0];
      double o1 = dim == 1 ? cut : off[1];
      double o2 = dim == 2 ? cut : off[2];
      double nm = dmul(dadd(dadd(o0, o1), o2), 0.9999999999999991);
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
      for (int64_t p = a; p < b; ++p) {
        const double4 P = ldg_pt(&c.pts[p]);
        const double d = metric(qx, qy, qz, P);
        if (d < thr) {
          res.insert(d, (int)p);
          thr = fmin(bound, res.worst());
        }
      }
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

// k-NN on the reference-order tree (tietree.cu) with nanoflann's traversal
// state for state (include/nanoflann.hpp:1221-1241 findNeighbors,
// 1005-1021 computeInitialDistances, 1346-1408 searchLevel): per-dimension
// offsets dists[] updated as mindistsq + cut_dist - dists[idx] and restored
// on the way back, the far child visited when its bound is <= the current
// worst distance, a leaf's points tested against the worst distance read
// on entering the leaf.  The recursion runs on an explicit frame stack
// (state 0: descend into the nearer child; 1: decide the farther one;
// 2: restore dists[idx]).  Results are device-tree indices.  Returns false
// when the tree is deeper than the stack (refused when the tree is built).
template <class List>
__device__ __noinline__ bool knn_tieorder(const DevCloud& c, double qx, double qy, double qz,
                                          List& res) {
  const double q[3] = {qx, qy, qz};
  double dists[3] = {0.0, 0.0, 0.0};
  double distsq = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (q[i] < c.tt_lo[i]) {
      dists[i] = dmul(dsub(q[i], c.tt_lo[i]), dsub(q[i], c.tt_lo[i]));
      distsq = dadd(distsq, dists[i]);
    }
    if (q[i] > c.tt_hi[i]) {
      dists[i] = dmul(dsub(q[i], c.tt_hi[i]), dsub(q[i], c.tt_hi[i]));
      distsq = dadd(distsq, dists[i]);
    }
  }
  int f_node[kTieMaxDepth];
  int f_state[kTieMaxDepth];
  double f_md[kTieMaxDepth], f_dst[kTieMaxDepth];
  int sp = 0;
  f_node[0] = 0;
  f_state[0] = 0;
  f_md[0] = distsq;
  while (sp >= 0) {
    const TieNode nd = c.tt_nodes[f_node[sp]];
    if (nd.feat < 0) {
      const double worst = res.worst();
      for (int i = nd.a; i < nd.b; ++i) {
        const double d = metric(qx, qy, qz, c.tt_pts[i]);
        if (d < worst) res.insert(d, c.tt_tid[i]);
      }
      --sp;
      continue;
    }
    const int idx = nd.feat;
    const double val = q[idx];
    const double diff1 = dsub(val, nd.lo);
    const double diff2 = dsub(val, nd.hi);
    const bool left_first = dadd(diff1, diff2) < 0;
    if (f_state[sp] == 0) {
      f_state[sp] = 1;
      if (sp + 1 >= kTieMaxDepth) return false;
      f_node[sp + 1] = left_first ? nd.a : nd.b;
      f_state[sp + 1] = 0;
      f_md[sp + 1] = f_md[sp];
      ++sp;
      continue;
    }
    if (f_state[sp] == 1) {
      const double cut = left_first ? dmul(dsub(val, nd.hi), dsub(val, nd.hi))
                                    : dmul(dsub(val, nd.lo), dsub(val, nd.lo));
      const double dst = dists[idx];
      const double md = dsub(dadd(f_md[sp], cut), dst);
      dists[idx] = cut;
      f_dst[sp] = dst;
      f_state[sp] = 2;
      if (md <= res.worst()) {
        if (sp + 1 >= kTieMaxDepth) return false;
        f_node[sp + 1] = left_first ? nd.b : nd.a;
        f_state[sp + 1] = 0;
        f_md[sp + 1] = md;
        ++sp;
        continue;
      }
    }
    dists[idx] = f_dst[sp];
    --sp;
  }
  return true;
}

// PointCloud::minDistSqToBox (src/pointcloud.cpp:283-297)
__device__ __forceinline__ double min_dist_sq_to_box(const DevCloud& c, double x, double y,
                                                     double z) {
  const double q[3] = {x, y, z};
  double d2 = 0.0;
#pragma unroll
  for (int dim = 0; dim < 3; dim++) {
    const double lo = c.sub_lo[dim], hi = c.sub_hi[dim];
    if (q[dim] < lo) {
      const double d = dsub(lo, q[dim]);
      d2 = dadd(d2, dmul(d, d));
    } else if (q[dim] > hi) {
      const double d = dsub(q[dim], hi);
      d2 = dadd(d2, dmul(d, d));
    }
  }
  return d2;
}

// Periodic images of PointCloud::queryTreeK (src/pointcloud.cpp:308-368):
// `res` holds the k-NN of q itself; each of the 26 shifted queries whose
// distance to the domain is within the current k-th distance + TOL is
// searched too, and the results are merged: one entry per particle with
// its smallest distance, sorted ascending, truncated to k.  (Equal
// distances keep their merge order here; the reference's std::sort leaves
// their order unspecified.)  `L` is KnnList<K> or KnnBig<KMAX>.
template <int KMAX, bool TT, class L>
__device__ __noinline__ void knn_periodic_merge64(const DevCloud& c, double qx, double qy,
                                                  double qz, L& res, unsigned& nvisit) {
  const int k = res.capacity();
  double md[2 * KMAX];
  int mi[2 * KMAX];
  int mn = res.count();
  for (int i = 0; i < mn; i++) {
    md[i] = res.r2[i];
    mi[i] = res.id[i];
  }
  for (int ix = -1; ix <= 1; ix++) {
    for (int iy = -1; iy <= 1; iy++) {
      for (int iz = -1; iz <= 1; iz++) {
        if (ix == 0 && iy == 0 && iz == 0) continue;
        const double sx = dadd(qx, dmul((double)ix, c.box[0]));
        const double sy = dadd(qy, dmul((double)iy, c.box[1]));
        const double sz = dadd(qz, dmul((double)iz, c.box[2]));
        const double minD2 = min_dist_sq_to_box(c, sx, sy, sz);
        const double worst = mn >= k ? md[k - 1] : __longlong_as_double(0x7ff0000000000000ULL);
        if (minD2 > dadd(worst, kTol)) continue;
        L img;
        img.clear(k);
        if (TT) knn_tieorder(c, sx, sy, sz, img);
        else knn_exact64(c, sx, sy, sz, __longlong_as_double(0x7ff0000000000000ULL), img, nvisit);
        const int ni = img.count();
        for (int i = 0; i < ni; i++) {
          bool found = false;
          for (int m = 0; m < mn; m++) {
            if (mi[m] == img.id[i]) {
              md[m] = fmin(md[m], img.r2[i]);
              found = true;
              break;
            }
          }
          if (!found) {
            md[mn] = img.r2[i];
            mi[mn] = img.id[i];
            ++mn;
          }
        }
        // sort ascending (stable insertion sort) and truncate to k
        for (int a = 1; a < mn; a++) {
          const double d = md[a];
          const int id = mi[a];
          int b = a;
          for (; b > 0 && md[b - 1] > d; --b) {
            md[b] = md[b - 1];
            mi[b] = mi[b - 1];
          }
          md[b] = d;
          mi[b] = id;
        }
        if (mn > k) mn = k;
      }
    }
  }
  for (int i = 0; i < mn; i++) {
    res.r2[i] = md[i];
    res.id[i] = mi[i];
  }
  res.set_count(mn);
}

// The k-NN of the reference's queryTreeK: exact FP64 search, then, in code
// compiled with PER and on a periodic cloud, the periodic merge.  Kernels
// that never serve periodic clouds compile without it (PER = false), which
// keeps the merge out of their register allocation.  TT: every search runs
// on the reference-order tree (the caller checks that it is built), so
// exactly tied points come in the reference's order.
template <int KMAX, bool PER, class L, bool TT = false>
__device__ __forceinline__ void knn_query64(const DevCloud& c, double qx, double qy, double qz,
                                            L& res, unsigned& nvisit) {
  if (TT) knn_tieorder(c, qx, qy, qz, res);
  else knn_exact64(c, qx, qy, qz, __longlong_as_double(0x7ff0000000000000ULL), res, nvisit);
  if constexpr (PER) {
    if (c.periodic && res.count() > 0) knn_periodic_merge64<KMAX, TT>(c, qx, qy, qz, res, nvisit);
  }
}

// One search's nearest neighbour (tree index) and whether another point has
// exactly the same distance (then the reference's answer depends on its
// traversal order).  On the reference-order tree (TT) the answer is the
// reference's and `tie` is not set.
template <bool TT>
__device__ __forceinline__ void nn1_search(const DevCloud& c, double x, double y, double z,
                                           int& id, double& d, bool& tie, unsigned& nvisit) {
  if (TT) {
    KnnList<1> r;
    r.clear();
    knn_tieorder(c, x, y, z, r);
    id = r.id[0];
    d = r.r2[0];
    return;
  }
  KnnList<2> r;
  r.clear();
  knn_exact64(c, x, y, z, __longlong_as_double(0x7ff0000000000000ULL), r, nvisit);
  id = r.id[0];
  d = r.r2[0];
  tie = tie || (r.id[1] >= 0 && r.r2[1] == r.r2[0]);
}

// PointCloud::queryTree (src/pointcloud.cpp:300-306) with the periodic
// 27-image merge (:313-367) at k = 1: an image's nearest replaces the
// current one only when strictly closer (the reference's sort keeps the
// earlier of equal entries) and the same particle keeps its smaller
// distance.
template <bool PER, bool TT>
__device__ __forceinline__ int nn1_query(const DevCloud& c, double qx, double qy, double qz,
                                         bool& tie, unsigned& nvisit) {
  int id;
  double d;
  nn1_search<TT>(c, qx, qy, qz, id, d, tie, nvisit);
  if (id < 0) return -1;
  if constexpr (PER) {
    if (c.periodic) {
      for (int ix = -1; ix <= 1; ix++)
        for (int iy = -1; iy <= 1; iy++)
          for (int iz = -1; iz <= 1; iz++) {
            if (ix == 0 && iy == 0 && iz == 0) continue;
            const double sx = dadd(qx, dmul((double)ix, c.box[0]));
            const double sy = dadd(qy, dmul((double)iy, c.box[1]));
            const double sz = dadd(qz, dmul((double)iz, c.box[2]));
            if (min_dist_sq_to_box(c, sx, sy, sz) > dadd(d, kTol)) continue;
            int iid;
            double idd;
            nn1_search<TT>(c, sx, sy, sz, iid, idd, tie, nvisit);
            if (iid < 0) continue;
            if (iid == id) d = fmin(d, idd);
            else if (idd < d) {
              id = iid;
              d = idd;
            }
          }
    }
  }
  return id;
}

// Nearest neighbour (tree index) of q, the reference's answer: -1 when no
// distance is finite; when the nearest distance is exactly shared, the
// query is repeated on the reference-order tree if TIES and the tree is
// built, else kTieUnresolved.  `nties` counts queries that met a tie.
template <bool PER = false, bool TIES = false>
__device__ __forceinline__ int nn1_exact64(const DevCloud& c, double qx, double qy, double qz,
                                           unsigned& nvisit, unsigned* nties = nullptr) {
  bool tie = false;
  const int id = nn1_query<PER, false>(c, qx, qy, qz, tie, nvisit);
  if (!tie || id < 0) return id;
  if (nties) ++*nties;
  if (!TIES || !c.tt_nodes) return kTieUnresolved;
  bool unused = false;
  return nn1_query<PER, true>(c, qx, qy, qz, unused, nvisit);
}

}  // namespace vt
