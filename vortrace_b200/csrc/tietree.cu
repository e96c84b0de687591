// tietree.cu -- the reference-order tree: nanoflann's middle-split k-d tree
// over the same points, built on the host when an exact distance tie first
// needs it, so that a nearest-neighbour query whose nearest distance is
// shared by several generators returns the generator the reference returns.
//
// Why it exists.  The device tree (tree_build.cu) is a median-split implicit
// tree: its searches return exactly the reference's nearest distances, but
// when two or more points are exactly equidistant from a query (lattices,
// quantised coordinates, rays along Voronoi faces) the point listed first is
// the first one the traversal meets, and nanoflann meets them in another
// order.  The walk uses the identity of a tied nearest point only through
// its 1-NN queries (ray ends, the bisection fallback of the split point,
// the perpendicular perturbation of Case 1a, the periodic same-cell
// bisection); its 2-NN and 3-NN decisions compare distances and sets within
// TOLERANCE and do not depend on the order of exactly tied points.  So the
// walk kernels detect an exact tie at the nearest distance of a 1-NN query
// and resolve only that query on this tree, with nanoflann's traversal.
//
// Build: include/nanoflann.hpp (v1.3.2, vendored by the reference)
//   computeBoundingBox 1316-1336, divideTree 858-905, middleSplit_ 910-956,
//   computeMinMax 837-849, planeSplit 967-1003; leaf_max_size 10
//   (src/pointcloud.cpp:204).  The split rule and both in-place partitions
//   are the published algorithm step for step, because the order of the
//   index array inside each leaf is part of the tie order.  Subtrees below
//   the top levels are built on separate host threads (the index ranges are
//   disjoint); the node array is in pre-order with explicit child indices.
// Device layout (uploaded once per built tree):
//   tt_nodes  TieNode[nnodes]   32 B: {divlow, divhigh, divfeat (-1: leaf),
//                               child1 | left, child2 | right}
//   tt_pts    double4[n]        point of index-array slot i (x, y, z, -)
//   tt_tid    int32[n]          device-tree index of index-array slot i
#include <algorithm>
#include <chrono>
#include <cstring>
#include <iostream>
#include <thread>
#include <vector>

#include "internal.h"

namespace vt {

namespace {

struct Iv {
  double low, high;
};

struct TieBuild {
  const double* P;  // n x 3, internal order
  uint32_t* vind;
  size_t leaf_max = 10;

  double pt(size_t idx, int d) const { return P[idx * 3 + d]; }

  // include/nanoflann.hpp:837-849
  void min_max(const uint32_t* ind, size_t count, int e, double& mn, double& mx) const {
    mn = pt(ind[0], e);
    mx = pt(ind[0], e);
    for (size_t i = 1; i < count; ++i) {
      const double v = pt(ind[i], e);
      if (v < mn) mn = v;
      if (v > mx) mx = v;
    }
  }

  // include/nanoflann.hpp:967-1003: values < cutval to the front, then the
  // values == cutval after them (unsigned indices, as the reference's size_t)
  void plane_split(uint32_t* ind, size_t count, int f, double cutval, size_t& lim1,
                   size_t& lim2) const {
    size_t left = 0, right = count - 1;
    for (;;) {
      while (left <= right && pt(ind[left], f) < cutval) ++left;
      while (right && left <= right && pt(ind[right], f) >= cutval) --right;
      if (left > right || !right) break;
      std::swap(ind[left], ind[right]);
      ++left;
      --right;
    }
    lim1 = left;
    right = count - 1;
    for (;;) {
      while (left <= right && pt(ind[left], f) <= cutval) ++left;
      while (right && left <= right && pt(ind[right], f) > cutval) --right;
      if (left > right || !right) break;
      std::swap(ind[left], ind[right]);
      ++left;
      --right;
    }
    lim2 = left;
  }

  // include/nanoflann.hpp:910-956
  void middle_split(uint32_t* ind, size_t count, size_t& index, int& cutfeat, double& cutval,
                    const Iv* bbox) const {
    const double EPS = 0.00001;
    double max_span = bbox[0].high - bbox[0].low;
    for (int i = 1; i < 3; ++i) {
      const double span = bbox[i].high - bbox[i].low;
      if (span > max_span) max_span = span;
    }
    double max_spread = -1;
    cutfeat = 0;
    for (int i = 0; i < 3; ++i) {
      const double span = bbox[i].high - bbox[i].low;
      if (span > (1 - EPS) * max_span) {
        double mn, mx;
        min_max(ind, count, i, mn, mx);
        const double spread = mx - mn;
        if (spread > max_spread) {
          cutfeat = i;
          max_spread = spread;
        }
      }
    }
    const double split_val = (bbox[cutfeat].low + bbox[cutfeat].high) / 2;
    double mn, mx;
    min_max(ind, count, cutfeat, mn, mx);
    if (split_val < mn) cutval = mn;
    else if (split_val > mx) cutval = mx;
    else cutval = split_val;
    size_t lim1, lim2;
    plane_split(ind, count, cutfeat, cutval, lim1, lim2);
    if (lim1 > count / 2) index = lim1;
    else if (lim2 < count / 2) index = lim2;
    else index = count / 2;
  }

  // include/nanoflann.hpp:858-905.  Appends the subtree of vind[left, right)
  // to `out` in pre-order; `bbox` comes in as the box the reference passes
  // down and leaves as the tight box of the subtree's points.  Returns the
  // subtree's depth in nodes.  spawn > 0: the first child is built on a
  // separate thread.
  int divide(size_t left, size_t right, Iv* bbox, std::vector<TieNode>& out, int spawn) {
    const size_t me = out.size();
    out.push_back(TieNode{});
    if (right - left <= leaf_max) {
      out[me].feat = -1;
      out[me].a = (int32_t)left;
      out[me].b = (int32_t)right;
      for (int i = 0; i < 3; ++i) bbox[i].low = bbox[i].high = pt(vind[left], i);
      for (size_t k = left + 1; k < right; ++k)
        for (int i = 0; i < 3; ++i) {
          const double v = pt(vind[k], i);
          if (bbox[i].low > v) bbox[i].low = v;
          if (bbox[i].high < v) bbox[i].high = v;
        }
      return 1;
    }
    size_t idx;
    int cutfeat;
    double cutval;
    middle_split(vind + left, right - left, idx, cutfeat, cutval, bbox);
    Iv lb[3], rb[3];
    memcpy(lb, bbox, sizeof(lb));
    memcpy(rb, bbox, sizeof(rb));
    lb[cutfeat].high = cutval;
    rb[cutfeat].low = cutval;
    int d1 = 0, d2 = 0;
    int32_t c1, c2;
    if (spawn > 0 && right - left > 65536) {
      std::vector<TieNode> s1, s2;
      bool failed = false;
      std::thread t([&] {
        try {
          d1 = divide(left, left + idx, lb, s1, spawn - 1);
        } catch (...) {
          failed = true;
        }
      });
      try {
        d2 = divide(left + idx, right, rb, s2, spawn - 1);
      } catch (...) {
        t.join();
        throw;
      }
      t.join();
      if (failed) throw std::bad_alloc();
      c1 = (int32_t)out.size();
      append(out, s1);
      c2 = (int32_t)out.size();
      append(out, s2);
    } else {
      c1 = (int32_t)out.size();
      d1 = divide(left, left + idx, lb, out, 0);
      c2 = (int32_t)out.size();
      d2 = divide(left + idx, right, rb, out, 0);
    }
    TieNode& nd = out[me];
    nd.feat = cutfeat;
    nd.a = c1;
    nd.b = c2;
    nd.lo = lb[cutfeat].high;
    nd.hi = rb[cutfeat].low;
    for (int i = 0; i < 3; ++i) {
      bbox[i].low = std::min(lb[i].low, rb[i].low);
      bbox[i].high = std::max(lb[i].high, rb[i].high);
    }
    return 1 + std::max(d1, d2);
  }

  // a subtree built with indices relative to its own array, moved to the end
  // of `out`
  static void append(std::vector<TieNode>& out, const std::vector<TieNode>& sub) {
    const int32_t off = (int32_t)out.size();
    out.reserve(out.size() + sub.size());
    for (TieNode nd : sub) {
      if (nd.feat >= 0) {
        nd.a += off;
        nd.b += off;
      }
      out.push_back(nd);
    }
  }
};

}  // namespace

void drop_tie_tree(vt_cloud* cl) {
  cl->tt_nodes_d.reset();
  cl->tt_pts_d.reset();
  cl->tt_tid_d.reset();
  cl->tt_depth = 0;
  cl->tt_ms = 0.0;
  cl->view.tt_nodes = nullptr;
  cl->view.tt_pts = nullptr;
  cl->view.tt_tid = nullptr;
}

int build_tie_tree(vt_cloud* cl, cudaStream_t st) {
  if (cl->view.tt_nodes) return VT_OK;
  if (!cl->tree_built)
    return set_error(VT_ERR_RUNTIME, "There is currently no valid tree for this point cloud");
  const size_t n = (size_t)cl->npart;
  if (n == 0 || n > 0x7fffffffULL)
    return set_error(VT_ERR_INVALID, "reference-order tree: point count out of range");
  auto t0 = std::chrono::high_resolution_clock::now();
  std::vector<uint32_t> vind(n);
  for (size_t i = 0; i < n; ++i) vind[i] = (uint32_t)i;
  TieBuild b;
  b.P = cl->pts.data();
  b.vind = vind.data();
  // include/nanoflann.hpp:1316-1336 computeBoundingBox
  Iv box[3];
  for (int i = 0; i < 3; ++i) box[i].low = box[i].high = b.pt(0, i);
  for (size_t k = 1; k < n; ++k)
    for (int i = 0; i < 3; ++i) {
      const double v = b.pt(k, i);
      if (v < box[i].low) box[i].low = v;
      if (v > box[i].high) box[i].high = v;
    }
  std::vector<TieNode> nodes;
  nodes.reserve(n / 4 + 16);
  unsigned hw = std::thread::hardware_concurrency();
  int spawn = 0;
  while ((1u << spawn) < (hw ? hw : 1u) && spawn < 6) ++spawn;
  const int depth = b.divide(0, n, box, nodes, spawn);
  if (depth > kTieMaxDepth)
    return set_error(VT_ERR_RUNTIME,
                     "the reference-order tree of this cloud is " + std::to_string(depth) +
                         " levels deep; exact ties can be resolved up to " +
                         std::to_string(kTieMaxDepth) + " levels");
  if (nodes.size() > 0x7fffffffULL)
    return set_error(VT_ERR_RUNTIME, "reference-order tree: too many nodes");
  // device-tree index of every internal id (perm: tree index -> internal id)
  std::vector<int32_t> perm(n), inv(n);
  VT_CUDA(cudaMemcpyAsync(perm.data(), cl->perm_d.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                          st));
  VT_CUDA(cudaStreamSynchronize(st));
  for (size_t t = 0; t < n; ++t) inv[(size_t)perm[t]] = (int32_t)t;
  std::vector<double4> tp(n);
  std::vector<int32_t> tid(n);
  for (size_t i = 0; i < n; ++i) {
    const size_t k = vind[i];
    tp[i] = make_double4(cl->pts[3 * k], cl->pts[3 * k + 1], cl->pts[3 * k + 2], 0.0);
    tid[i] = inv[k];
  }
  DevBuf<TieNode> dn;
  DevBuf<double4> dp;
  DevBuf<int32_t> di;
  int rc;
  if ((rc = dn.alloc(nodes.size())) || (rc = dp.alloc(n)) || (rc = di.alloc(n))) return rc;
  VT_CUDA(cudaMemcpyAsync(dn.p, nodes.data(), nodes.size() * sizeof(TieNode),
                          cudaMemcpyHostToDevice, st));
  VT_CUDA(cudaMemcpyAsync(dp.p, tp.data(), n * sizeof(double4), cudaMemcpyHostToDevice, st));
  VT_CUDA(cudaMemcpyAsync(di.p, tid.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  VT_CUDA(cudaStreamSynchronize(st));
  cl->tt_nodes_d = std::move(dn);
  cl->tt_pts_d = std::move(dp);
  cl->tt_tid_d = std::move(di);
  cl->tt_depth = depth;
  DevCloud& v = cl->view;
  v.tt_nodes = cl->tt_nodes_d.p;
  v.tt_pts = cl->tt_pts_d.p;
  v.tt_tid = cl->tt_tid_d.p;
  for (int i = 0; i < 3; ++i) {
    v.tt_lo[i] = box[i].low;
    v.tt_hi[i] = box[i].high;
  }
  auto t1 = std::chrono::high_resolution_clock::now();
  cl->tt_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  if (verbose())
    std::cout << "Reference-order tree (" << nodes.size() << " nodes, depth " << depth
              << ") built in " << (long long)cl->tt_ms << " milliseconds." << std::endl;
  return VT_OK;
}

}  // namespace vt

extern "C" int vt_cloud_build_tie_tree(vt_cloud* cl) {
  using namespace vt;
  try {
    if (!cl) return set_error(VT_ERR_INVALID, "null cloud handle");
    std::lock_guard<std::mutex> lk(cl->mu);
    VT_CUDA(cudaSetDevice(cl->device));
    return build_tie_tree(cl, cl->stream);
  } catch (const std::bad_alloc&) {
    return set_error(VT_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception& e) {
    return set_error(VT_ERR_RUNTIME, e.what());
  }
}
