// walk.cuh -- the per-ray walk of vortrace (src/ray.cpp:187-430) on device.
//
// The reference keeps the ray as a linked list of RayPoints and only ever
// inserts right after the current point, so the list past the current point
// is a stack whose top is `next`: Case 1 pushes, Case 1a pushes sn then sc,
// Case 2 and the zero-width skip pop.  Segments come out in ray order and
// go straight into a sink (fused reduction, segment writer or adjoint), so
// no per-ray segment list exists.
//
// Cell ids inside the walk are tree indices (tree order); the map to the
// reference's internal ids (perm) is a bijection, so every equality test the
// walk makes is unchanged.  All FP64 expressions keep the reference's order.
#pragma once

#include "knn.cuh"

namespace vt {

struct RayGeom {
  double s[3], e[3], d[3];
  double len;
};

// Ray::Ray (src/ray.cpp:14-35)
__device__ __forceinline__ void ray_init(RayGeom& g, const double* st, const double* en) {
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    g.s[j] = st[j];
    g.e[j] = en[j];
    g.d[j] = dsub(en[j], st[j]);
  }
  double l = __dsqrt_rn(dadd(dadd(dmul(g.d[0], g.d[0]), dmul(g.d[1], g.d[1])),
                             dmul(g.d[2], g.d[2])));
#pragma unroll
  for (int j = 0; j < 3; ++j) g.d[j] = ddiv(g.d[j], l);
  g.len = l;
}

__device__ __forceinline__ bool ray_finite(const RayGeom& g) {
  bool ok = true;
#pragma unroll
  for (int j = 0; j < 3; ++j) ok = ok && isfinite(g.s[j]) && isfinite(g.e[j]);
  return ok;
}

// Ray::findSplitPointDistance(pos1, pos2) (src/ray.cpp:38-60)
__device__ __forceinline__ double split_analytic(const RayGeom& g, double4 p1, double4 p2) {
  const double n0 = dsub(p2.x, p1.x), n1 = dsub(p2.y, p1.y), n2 = dsub(p2.z, p1.z);
  const double q0 = dsub(dmul(0.5, dadd(p1.x, p2.x)), g.s[0]);
  const double q1 = dsub(dmul(0.5, dadd(p1.y, p2.y)), g.s[1]);
  const double q2 = dsub(dmul(0.5, dadd(p1.z, p2.z)), g.s[2]);
  const double ndp = dadd(dadd(dmul(n0, q0), dmul(n1, q1)), dmul(n2, q2));
  const double ndd = dadd(dadd(dmul(n0, g.d[0]), dmul(n1, g.d[1])), dmul(n2, g.d[2]));
  if (fabs(ndd) < kParallelTol) return DBL_MAX;
  return ddiv(ndp, ndd);
}

__device__ __forceinline__ void ray_point(const RayGeom& g, double s, double& x, double& y,
                                          double& z) {
  x = dadd(g.s[0], dmul(s, g.d[0]));
  y = dadd(g.s[1], dmul(s, g.d[1]));
  z = dadd(g.s[2], dmul(s, g.d[2]));
}

// Detail of a failing ray (filled only by the diagnosis launch).
struct WalkDiag {
  int code;
  int c, n;  // tree indices
  double s, s_lo, s_hi;
};

// ---------------------------------------------------------------- stacks
template <int CAP>
struct LocalStack {
  int id[CAP];
  double s[CAP];
  int sp, maxsp;
  int cap = CAP;  // usable entries (<= CAP)
  __device__ __forceinline__ void set_cap(int c) { cap = c < CAP ? (c > 1 ? c : 1) : CAP; }
  __device__ __forceinline__ void clear() { sp = maxsp = 0; }
  __device__ __forceinline__ bool full() const { return sp >= cap; }
  __device__ __forceinline__ bool empty() const { return sp == 0; }
  __device__ __forceinline__ void push(int i, double v) {
    id[sp] = i;
    s[sp] = v;
    ++sp;
    maxsp = max(maxsp, sp);
  }
  __device__ __forceinline__ void pop() { --sp; }
  __device__ __forceinline__ int top_id() const { return id[sp - 1]; }
  __device__ __forceinline__ double top_s() const { return s[sp - 1]; }
  __device__ __forceinline__ int room() const { return cap - sp; }
};

struct GlobalStack {
  int* id;
  double* s;
  int cap;
  int sp, maxsp;
  __device__ __forceinline__ void clear() { sp = maxsp = 0; }
  __device__ __forceinline__ bool empty() const { return sp == 0; }
  __device__ __forceinline__ void push(int i, double v) {
    id[sp] = i;
    s[sp] = v;
    ++sp;
    maxsp = max(maxsp, sp);
  }
  __device__ __forceinline__ void pop() { --sp; }
  __device__ __forceinline__ int top_id() const { return id[sp - 1]; }
  __device__ __forceinline__ double top_s() const { return s[sp - 1]; }
  __device__ __forceinline__ int room() const { return cap - sp; }
};

// ------------------------------------------------------- exact FP64 search
// Full-featured search policy (plain kernel and degenerate-geometry kernel);
// PER: also serves periodic clouds (periodic k-NN merge, minimum-image split
// points, same-cell bisection).  TIES: a 1-NN query whose nearest distance
// is exactly shared is answered on the reference-order tree when it is
// built; otherwise (and always without TIES) nn1 returns kTieUnresolved and
// the walk stops with kNeedTie.
template <bool PER, bool TIES = false>
struct Search64T {
  const DevCloud& c;
  unsigned nq = 0, nvisit = 0, nties = 0;
  static constexpr bool kPeriodic = PER;
  __device__ explicit Search64T(const DevCloud& cc) : c(cc) {}
  __device__ __forceinline__ int nn1(double x, double y, double z) {
    ++nq;
    return nn1_exact64<PER, TIES>(c, x, y, z, nvisit, &nties);
  }
  // 3-NN at a split point between cells cid and nid
  __device__ __forceinline__ int knn3(double x, double y, double z, int cid, int nid,
                                      KnnList<3>& r) {
    ++nq;
    r.clear();
    knn_query64<3, PER>(c, x, y, z, r, nvisit);
    return 0;
  }
  __device__ __forceinline__ void knn2(double x, double y, double z, KnnList<2>& r) {
    ++nq;
    r.clear();
    knn_query64<2, PER>(c, x, y, z, r, nvisit);
  }
  static constexpr bool kDefer = false;  // rare paths run inline
};
using Search64 = Search64T<false>;

// ------------------------------------------------------------------ walk
// Ray::findSplitPointDistance(cloud, id1, id2, s_lo, s_hi) (src/ray.cpp:64-127)
template <class S>
__device__ int split_full(const DevCloud& c, const RayGeom& g, S& srch, int id1, int id2,
                          double s_lo, double s_hi, double& s_out) {
  double4 p1 = ldg_pt(&c.pts[id1]);
  double4 p2 = ldg_pt(&c.pts[id2]);
  if (S::kPeriodic && c.periodic) {
    // minimum image of both generators about the segment's midpoint on the
    // ray (src/ray.cpp:71-86)
    const double s_ref = dmul(0.5, dadd(s_lo, s_hi));
    double a[3] = {p1.x, p1.y, p1.z}, b[3] = {p2.x, p2.y, p2.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double ref = dadd(g.s[d], dmul(s_ref, g.d[d]));
      const double half = dmul(c.box[d], 0.5);
      const double diff1 = dsub(a[d], ref);
      if (diff1 > half) a[d] = dsub(a[d], c.box[d]);
      else if (diff1 < -half) a[d] = dadd(a[d], c.box[d]);
      const double diff2 = dsub(b[d], ref);
      if (diff2 > half) b[d] = dsub(b[d], c.box[d]);
      else if (diff2 < -half) b[d] = dadd(b[d], c.box[d]);
    }
    p1 = make_double4(a[0], a[1], a[2], 0.0);
    p2 = make_double4(b[0], b[1], b[2], 0.0);
  }
  double s = split_analytic(g, p1, p2);
  if (s < DBL_MAX * 0.5 && s >= s_lo - kTol && s <= s_hi + kTol) {
    s_out = s;
    return 0;
  }
  if (S::kDefer) return kNeedSlow;
  double lo = s_lo, hi = s_hi;
  for (int it = 0; it < 64; ++it) {
    const double mid = dmul(0.5, dadd(lo, hi));
    double x, y, z;
    ray_point(g, mid, x, y, z);
    const int mc = srch.nn1(x, y, z);
    if (mc == kTieUnresolved) return kNeedTie;
    if (mc < 0) return kErrNonFiniteDist;
    if (mc != id1 && mc != id2) {
      s_out = mid;
      return 0;
    }
    if (mc == id1) lo = mid;
    else hi = mid;
    if (dsub(hi, lo) < 1e-12) {
      s_out = dmul(0.5, dadd(lo, hi));
      return 0;
    }
  }
  return kErrBinSearch;
}

// Ray::perpPerturbToFindCell (src/ray.cpp:129-185); returns -1 on failure,
// kTieUnresolved when a query met a tie it could not resolve.
template <class S>
__device__ int perp_perturb(const RayGeom& g, S& srch, double px, double py, double pz, int ex1,
                            int ex2) {
  const double is2 = ddiv(1.0, __dsqrt_rn(2.0));
  const double w[3][3] = {{is2, is2, 0.0}, {0.0, is2, is2}, {is2, 0.0, is2}};
  const double pos[3] = {px, py, pz};
  int cycle = 0;
  for (int bound = 1; cycle < kMaxPerturbCycles; bound++) {
    for (int a = -bound; a <= bound && cycle < kMaxPerturbCycles; a++) {
      for (int b = -bound; b <= bound && cycle < kMaxPerturbCycles; b++) {
        for (int cc = -bound; cc <= bound && cycle < kMaxPerturbCycles; cc++) {
          if (a == 0 && b == 0 && cc == 0) continue;
          if (abs(a) < bound && abs(b) < bound && abs(cc) < bound) continue;
          double pd[3];
#pragma unroll
          for (int j = 0; j < 3; j++)
            pd[j] = dadd(dadd(dmul((double)a, w[0][j]), dmul((double)b, w[1][j])),
                         dmul((double)cc, w[2][j]));
          double cr[3];
          cr[0] = dsub(dmul(g.d[1], pd[2]), dmul(g.d[2], pd[1]));
          cr[1] = dsub(dmul(g.d[2], pd[0]), dmul(g.d[0], pd[2]));
          cr[2] = dsub(dmul(g.d[0], pd[1]), dmul(g.d[1], pd[0]));
          const double mag =
              __dsqrt_rn(dadd(dadd(dmul(cr[0], cr[0]), dmul(cr[1], cr[1])), dmul(cr[2], cr[2])));
          if (mag < 1e-15) {
            cycle++;
            continue;
          }
#pragma unroll
          for (int j = 0; j < 3; j++) cr[j] = ddiv(cr[j], mag);
          double pt[3];
#pragma unroll
          for (int j = 0; j < 3; j++) pt[j] = dadd(pos[j], dmul(kPerturbEps, cr[j]));
          const int cell = srch.nn1(pt[0], pt[1], pt[2]);
          if (cell == kTieUnresolved) return kTieUnresolved;
          if (cell != ex1 && cell != ex2) return cell;
          cycle++;
        }
      }
    }
  }
  return -1;
}

// src/ray.cpp:374-384 (tryAlongRay); -1 when ambiguous
template <class S>
__device__ int try_along_ray(const RayGeom& g, S& srch, double px, double py, double pz,
                             double sign, int cid, int nid) {
  const double e = dmul(sign, kPerturbEps);
  double x = dadd(px, dmul(e, g.d[0]));
  double y = dadd(py, dmul(e, g.d[1]));
  double z = dadd(pz, dmul(e, g.d[2]));
  KnnList<2> r;
  srch.knn2(x, y, z, r);
  if (dadd(r.r2[0], kTol) < r.r2[1] && r.id[0] != cid && r.id[0] != nid) return r.id[0];
  return -1;
}

// 100-NN expansion (src/ray.cpp:319-338).  Returns 0 or kErrKnnExpand.
template <bool PER = false>
__device__ __noinline__ int expand_classify(const DevCloud& c, double x, double y, double z,
                                            int cid, int nid, bool& has_c, bool& has_n,
                                            unsigned& nvisit) {
  KnnBig<kExpandK> r;
  const int kb = (int)min((int64_t)kExpandK, c.n);
  r.clear(kb);
  knn_query64<kExpandK, PER>(c, x, y, z, r, nvisit);
  for (int i = 0; i < kb; i++) {
    if (dsub(r.r2[i], r.r2[0]) >= kTol) break;
    if (r.id[i] == cid) has_c = true;
    if (r.id[i] == nid) has_n = true;
    if (i == kb - 1 && !has_c && !has_n) return kErrKnnExpand;
  }
  return 0;
}

// Ray::walk (src/ray.cpp:187-430).  Emits segments in order to
// `sink.seg(cell, s_enter, s_exit)`.  Returns 0, an error code, kNeedSlow
// (search policy with kDefer, or a stack without room) or kNeedTie (a 1-NN
// query met an exact tie the search policy cannot resolve; every segment
// emitted before it is the reference's).
template <class S, class Stack, class Sink>
__device__ int walk_ray(const DevCloud& c, const RayGeom& g, int64_t max_iter, S& srch,
                        Stack& st, Sink& sink, WalkDiag* diag) {
  const int c0 = srch.nn1(g.s[0], g.s[1], g.s[2]);
  const int c1 = srch.nn1(g.e[0], g.e[1], g.e[2]);
  if (c0 == kTieUnresolved || c1 == kTieUnresolved) return kNeedTie;
  if (c0 < 0 || c1 < 0) return kErrNonFiniteDist;  // squared distances overflowed
  int open_cell = c0;
  double entry_s = 0.0;
  st.clear();
  st.push(c1, g.len);
  if (c0 == c1) {
    if (!(S::kPeriodic && c.periodic)) {
      sink.seg(c0, 0.0, g.len);
      return 0;
    }
    // periodic: sample the ray at dyadic fractions 1/2, 1/4, 3/4, 1/8, ...
    // for a point in another cell and walk towards it first
    // (src/ray.cpp:220-246)
    bool found = false;
    for (int level = 1; level <= 10 && !found; level++) {
      const int n = 1 << level;
      for (int i = 1; i < n && !found; i += 2) {
        const double mid_s = ddiv(dmul(g.len, (double)i), (double)n);
        double x, y, z;
        ray_point(g, mid_s, x, y, z);
        const int mc = srch.nn1(x, y, z);
        if (mc == kTieUnresolved) return kNeedTie;
        if (mc < 0) return kErrNonFiniteDist;
        if (mc != c0) {
          st.push(mc, mid_s);
          found = true;
        }
      }
    }
    if (!found) {
      if (diag) diag->code = kErrPeriodicBisect;
      return kErrPeriodicBisect;
    }
  }
  int cur = c0;
  double cur_s = 0.0;
  int64_t iteration = 0;
  for (;;) {
    if (++iteration > max_iter) {
      if (diag) diag->code = kErrMaxIter;
      return kErrMaxIter;
    }
    const int nxt = st.top_id();
    const double nxt_s = st.top_s();
    // zero-width skip (src/ray.cpp:266-274)
    if (dsub(nxt_s, cur_s) < 1e-14) {
      st.pop();
      cur = nxt;
      cur_s = nxt_s;
      open_cell = cur;
      if (st.empty()) break;
      continue;
    }
    double s;
    int rc = split_full(c, g, srch, cur, nxt, cur_s, nxt_s, s);
    if (rc) {
      if (diag) {
        diag->code = rc;
        diag->c = cur;
        diag->n = nxt;
      }
      return rc;
    }
    if (s < dsub(cur_s, kTol) || s > dadd(nxt_s, kTol)) {
      if (diag) {
        diag->code = kErrSplitBounds;
        diag->c = cur;
        diag->n = nxt;
        diag->s = s;
        diag->s_lo = cur_s;
        diag->s_hi = nxt_s;
      }
      return kErrSplitBounds;
    }
    {
      const double lo = dadd(cur_s, 1e-15), hi = dsub(nxt_s, 1e-15);
      s = (s < lo) ? lo : (hi < s) ? hi : s;
    }
    double x, y, z;
    ray_point(g, s, x, y, z);
    KnnList<3> r;
    rc = srch.knn3(x, y, z, cur, nxt, r);
    if (rc) return rc;
    if (r.id[0] < 0) return kErrNonFiniteDist;
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
    if (three_eq && !has_c && !has_n) {
      if (S::kDefer) return kNeedSlow;
      rc = expand_classify<S::kPeriodic>(c, x, y, z, cur, nxt, has_c, has_n, srch.nvisit);
      if (rc) {
        if (diag) diag->code = rc;
        return rc;
      }
    }
    if (has_c || has_n) {
      // Case 2: boundary between cur and nxt (src/ray.cpp:340-354)
      sink.seg(open_cell, entry_s, s);
      open_cell = nxt;
      entry_s = s;
      st.pop();
      cur = nxt;
      cur_s = nxt_s;
      if (st.empty()) break;
    } else if (dadd(r.r2[0], kTol) < r.r2[1]) {
      // Case 1: one cell strictly closest (src/ray.cpp:358-363)
      if (st.room() < 1) return kNeedSlow;
      st.push(r.id[0], s);
    } else {
      // Case 1a (src/ray.cpp:364-422)
      if (S::kDefer) return kNeedSlow;
      int sc = try_along_ray(g, srch, x, y, z, -1.0, cur, nxt);
      if (sc < 0) {
        const double ex = dmul(kPerturbEps, g.d[0]), ey = dmul(kPerturbEps, g.d[1]),
                     ez = dmul(kPerturbEps, g.d[2]);
        sc = perp_perturb(g, srch, dsub(x, ex), dsub(y, ey), dsub(z, ez), cur, nxt);
        if (sc == kTieUnresolved) return kNeedTie;
        if (sc < 0) {
          if (diag) diag->code = kErrPerturb;
          return kErrPerturb;
        }
      }
      int sn = try_along_ray(g, srch, x, y, z, 1.0, cur, nxt);
      if (sn < 0) {
        const double ex = dmul(kPerturbEps, g.d[0]), ey = dmul(kPerturbEps, g.d[1]),
                     ez = dmul(kPerturbEps, g.d[2]);
        sn = perp_perturb(g, srch, dadd(x, ex), dadd(y, ey), dadd(z, ez), cur, nxt);
        if (sn == kTieUnresolved) return kNeedTie;
        if (sn < 0) {
          if (diag) diag->code = kErrPerturb;
          return kErrPerturb;
        }
      }
      if (sc == sn) {
        if (st.room() < 1) return kNeedSlow;
        st.push(sc, s);
      } else {
        if (st.room() < 2) return kNeedSlow;
        st.push(sn, s);
        st.push(sc, s);
      }
    }
  }
  // close the last open cell at the ray end (src/ray.cpp:427)
  sink.seg(open_cell, entry_s, cur_s);
  return 0;
}

}  // namespace vt
