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

// Convenience: nearest neighbour (tree index) of q.
__device__ __forceinline__ int nn1_exact64(const DevCloud& c, double qx, double qy, double qz,
                                           unsigned& nvisit) {
  KnnList<1> r;
  r.clear();
  knn_exact64(c, qx, qy, qz, __longlong_as_double(0x7ff0000000000000ULL), r, nvisit);
  return r.id[0];
}

}  // namespace vt
