// warp.cuh -- the batched walk kernel: one warp per ray, warp-cooperative
// guarded-FP32 k-NN.
//
// The walk of src/ray.cpp:187-430 runs with warp-uniform control flow: every
// lane holds the same ray state, and only the k-NN searches and the field
// reductions spread work over the lanes.
//   * Work queue: lane 0 of a warp takes the next ray from a global atomic
//     counter; long and short rays, many projections and arbitrary rays share
//     one persistent launch.
//   * k-NN ("wide" traversal of the implicit binary tree): a step expands one
//     node into its descendants 5 levels down (32 nodes, contiguous in heap
//     order, one per lane).  Each lane loads its node's tight FP32 box with two
//     coalesced 128-bit loads and tests it against the threshold; a ballot
//     gives the survivors, the nearest continues and the rest go on a per-warp
//     stack in shared memory.  Leaf groups are expanded into their points,
//     spread over the lanes (warp prefix sum + per-lane binary search), tested
//     in FP32, and the few points that pass are re-checked with their FP64
//     distance in the reference's operation order and inserted in lane order.
//   * Guarded FP32: a point passes if f < thr64 + G, where G bounds the
//     FP32 error of f for every point with d < R; box distances use the same
//     rounding steps as f on box corners that are themselves FP32 point
//     values, so box pruning never drops a point that would pass.  The FP64
//     list is exact; only the order of exactly tied points can differ from
//     nanoflann's.
//   * Split queries are bounded by R = max(d_c, d_n) + 4 TOL (see
//     knn3_decision_valid); end-point queries start from the leaf found by
//     descending the split planes, then search bounded by its best distance.
//   * The pending-point stack of the walk also lives in shared memory (64
//     entries per warp); a deeper stack hands the ray to k_slow.
#pragma once

namespace vt {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = 4;
constexpr int kWSearchStack = 128;  // per-warp search stack entries
constexpr int kWWalkStack = 64;     // per-warp pending ray points
#ifndef VT_WARP_MINB
#define VT_WARP_MINB 4
#endif

__device__ __forceinline__ int depth_of(int v) { return 31 - __clz(v + 1); }

// FP32 acceptance threshold for FP64 threshold T: every point with d < T
// has FP32 distance f < T + G(T) (guard_band), rounded up.
__device__ __forceinline__ float thr32_of(double T, double qe) {
  return __double2float_ru(dadd(T, guard_band(T, qe)));
}

struct WarpQuery {
  double x, y, z;     // FP64 query
  float q0, q1, q2;   // FP32 frame
  double bound, G;    // accept d < bound; FP32 guard band at the bound
  double qe;          // FP32 coordinate error of this ray's queries
  int cid, nid;       // cells with known distances (or -1)
  double dc, dn;
};

// Test the points of the leaves in `mask` (group starting at heap node
// `gfirst`) and insert the ones with d < current threshold into L.
template <int K>
__device__ __forceinline__ void warp_leaves(const DevCloud& c, const int lane,
                                            const WarpQuery& Q, const unsigned mask,
                                            const int64_t gfirst, KnnList<K>& L, double& thr64,
                                            float& thr32, unsigned& nver) {
  const int64_t ninternal = c.nleaves - 1;
  int64_t a = 0;
  int cnt = 0;
  if ((mask >> lane) & 1u) {
    const int64_t j = gfirst + lane - ninternal;
    a = (j * c.n) >> c.depth;
    cnt = (int)((((j + 1) * c.n) >> c.depth) - a);
  }
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  const int total = __shfl_sync(kFull, incl, 31);
  for (int base = 0; base < total; base += 32) {
    const int kk = base + lane;
    int lo = 0, hi = 31;
#pragma unroll
    for (int it = 0; it < 5; ++it) {
      const int mid = (lo + hi) >> 1;
      const int vm = __shfl_sync(kFull, incl, mid);
      if (vm > kk) hi = mid;
      else lo = mid + 1;
    }
    const long long ao = __shfl_sync(kFull, (long long)a, lo);
    const int exo = __shfl_sync(kFull, incl - cnt, lo);
    const int64_t p = ao + (kk - exo);
    const bool act = kk < total;
    float f = __int_as_float(0x7f800000);
    if (act) f = pt_dist32(Q.q0, Q.q1, Q.q2, __ldg(&c.pts32[p]));
    const bool cand = act && f < thr32;
    unsigned cm = __ballot_sync(kFull, cand);
    if (!cm) continue;
    double d = 0.0;
    if (cand) {
      const int pi = (int)p;
      if (pi == Q.cid) d = Q.dc;
      else if (pi == Q.nid) d = Q.dn;
      else {
        d = metric(Q.x, Q.y, Q.z, ldg_pt(&c.pts[p]));
        ++nver;
      }
    }
    while (cm) {
      const int j = __ffs(cm) - 1;
      cm &= cm - 1;
      const double dj = __shfl_sync(kFull, d, j);
      const int pj = __shfl_sync(kFull, (int)p, j);
      if (dj < thr64) {
        L.insert(dj, pj);
        thr64 = fmin(Q.bound, L.worst());
        thr32 = thr32_of(thr64, Q.qe);
      }
    }
  }
}

// Warp-cooperative exact K-NN among points with d < Q.bound; L may hold
// results already (then `skip_leaf`, the leaf they came from, is skipped).
// Returns false if the per-warp stack overflowed (the result is then not
// trustworthy and the caller re-resolves the query).
// `start` >= 0 restricts the search to the subtree of that internal node
// (whose own box the caller has tested); -1 searches the whole tree.
template <int K>
__device__ __forceinline__ bool warp_knn(const DevCloud& c, const int lane, const WarpQuery& Q,
                         const int64_t skip_leaf, KnnList<K>& L, int* s_node, float* s_mind,
                         unsigned& nver, unsigned& nsteps, const int64_t start = -1) {
  const int D = c.depth;
  const int64_t ninternal = c.nleaves - 1;
  double thr64 = fmin(Q.bound, L.worst());
  float thr32 = thr32_of(thr64, Q.qe);
  int sp = 0;
  bool overflow = false;
  // group being tested: nodes [gfirst, gfirst + gm), leaves if gleaves
  int64_t gfirst;
  int gm;
  bool gleaves;
  if (start >= 0) {
    const int k = 63 - __clzll(start + 1);
    const int s = min(5, D - k);
    gfirst = ((start + 1) << s) - 1;
    gm = 1 << s;
    gleaves = (k + s == D);
  } else if (D == 0) {
    gfirst = 0;
    gm = 1;
    gleaves = true;
  } else {
    const int s = ((D - 1) % 5) + 1;  // so that every later step spans 5 levels
    gfirst = (1LL << s) - 1;
    gm = 1 << s;
    gleaves = (s == D);
  }
  for (;;) {
    ++nsteps;
    const int64_t node = gfirst + lane;
    float nm = __int_as_float(0x7f800000);
    bool surv = false;
    if (lane < gm) {
      nm = box_dist32(Q.q0, Q.q1, Q.q2, __ldg(&c.boxlo[node]), __ldg(&c.boxhi[node]));
      surv = nm < thr32 && !(gleaves && node - ninternal == skip_leaf);
    }
    const unsigned mask = __ballot_sync(kFull, surv);
    bool next = false;
    int v = 0;
    if (gleaves) {
      if (mask) warp_leaves<K>(c, lane, Q, mask, gfirst, L, thr64, thr32, nver);
    } else if (mask) {
      const unsigned key = surv ? __float_as_uint(nm) : 0xffffffffu;
      const unsigned kmin = __reduce_min_sync(kFull, key);
      const int w = __ffs(__ballot_sync(kFull, key == kmin)) - 1;
      const unsigned rest = mask & ~(1u << w);
      const int cnt = __popc(rest);
      if (sp + cnt > kWSearchStack) {
        overflow = true;
      } else if ((rest >> lane) & 1u) {
        const int e = sp + __popc(rest & ((1u << lane) - 1u));
        s_node[e] = (int)node;
        s_mind[e] = nm;
      }
      if (!overflow) sp += cnt;
      __syncwarp();
      v = (int)(gfirst + w);
      next = true;
    }
    if (!next) {
      while (sp > 0) {
        --sp;
        const float pm = s_mind[sp];
        if (pm < thr32) {
          v = s_node[sp];
          next = true;
          break;
        }
      }
      __syncwarp();
      if (!next) break;
    }
    const int k = depth_of(v);
    const int s = min(5, D - k);
    gfirst = ((int64_t)(v + 1) << s) - 1;
    gm = 1 << s;
    gleaves = (k + s == D);
  }
  return !overflow;
}

// Leaf reached by descending the split planes from the root (uniform loads).
__device__ __forceinline__ int64_t warp_descend_leaf(const DevCloud& c, float q0, float q1,
                                                     float q2) {
  const int64_t ninternal = c.nleaves - 1;
  int64_t v = 0;
  while (v < ninternal) {
    const float2 nd = __ldg(&c.nodes32[v]);
    const int dim = node_dim32(nd.x);
    const float val = dim == 0 ? q0 : (dim == 1 ? q1 : q2);
    v = __fadd_rn(__fsub_rn(val, nd.x), __fsub_rn(val, nd.y)) < 0.f ? 2 * v + 1 : 2 * v + 2;
  }
  return v - ninternal;
}

// Unbounded K-NN: the leaf on the split-plane path first (all its points
// are candidates), then a search bounded by the K-th best distance found.
template <int K>
__device__ __forceinline__ bool warp_knn_unbounded(const DevCloud& c, const int lane, WarpQuery Q, double qe,
                                   KnnList<K>& L, int* s_node, float* s_mind, unsigned& nver,
                                   unsigned& nsteps) {
  L.clear();
  const int64_t leaf = warp_descend_leaf(c, Q.q0, Q.q1, Q.q2);
  {
    const int64_t a = (leaf * c.n) >> c.depth;
    const int cnt = (int)((((leaf + 1) * c.n) >> c.depth) - a);
    for (int base = 0; base < cnt; base += 32) {
      const int kk = base + lane;
      double d = 0.0;
      if (kk < cnt) d = metric(Q.x, Q.y, Q.z, ldg_pt(&c.pts[a + kk]));
      const int m = min(32, cnt - base);
      for (int j = 0; j < m; ++j) {
        const double dj = __shfl_sync(kFull, d, j);
        if (dj < L.worst()) L.insert(dj, (int)(a + base + j));
      }
    }
  }
  Q.bound = __longlong_as_double(0x7ff0000000000000LL);
  Q.cid = Q.nid = -1;
  // the threshold never exceeds the K-th distance found in the leaf
  Q.G = guard_band(L.worst(), qe);
  return warp_knn<K>(c, lane, Q, leaf, L, s_node, s_mind, nver, nsteps);
}

// Guard band for unbounded queries: the FP32 error bound at the current
// threshold is re-derived when the threshold is known (G grows with R).
__device__ __forceinline__ void warp_query_setup(WarpQuery& Q, const DevCloud& c, double x,
                                                 double y, double z) {
  Q.x = x;
  Q.y = y;
  Q.z = z;
  Q.q0 = __double2float_rn(dsub(x, c.origin[0]));
  Q.q1 = __double2float_rn(dsub(y, c.origin[1]));
  Q.q2 = __double2float_rn(dsub(z, c.origin[2]));
}

// ------------------------------------------------- tube cache
// Consecutive split points of a ray lie on the ray and move forward (a
// query's s is never below the walk's current s), so one gather of the
// points around a stretch of the ray serves many queries.  A warp keeps a
// "capsule" of points:
//   every point p whose axial parameter t = (p - P_a).dir lies in [0, L]
//   and whose distance from the ray's line is < rho is in the cache,
// with P_a = start + s_a dir.  A split query at parameter s is answered
// from the cache when, after the scan, the final threshold
// T = min(bound, 3rd best distance) gives r = sqrt(T)(1 + 1e-12) + eps
// with r <= rho and s_a <= s - r and s + r <= s_a + L: every p with
// d64(q, p) <= T has |t(p) - (s - s_a)| <= |p - q| < r and a distance from
// the line below r <= rho, so it is cached, and the bounded 3-NN over the
// cache is the same exact set as over the tree.  The gather's membership
// test runs in FP64 on the FP64 points; eps covers FP64 rounding.
//
// The cache holds up to kCache points in gather (tree) order, split into
// chunks of 32 with a tight FP32 box per chunk; a scan tests the chunk
// boxes (one per lane), then visits the surviving chunks nearest first.
#ifndef VT_WARP_CACHE
#define VT_WARP_CACHE 256
#endif
constexpr int kCache = VT_WARP_CACHE;  // points per warp
constexpr int kChunks = kCache / 32;
static_assert(kCache % 32 == 0 && kChunks <= 32, "cache is 1..32 chunks of 32 points");

struct Capsule {
  double sa, L, rho;  // start parameter, guaranteed length and radius
  int count;          // cached points
  int total;          // points found in the requested capsule (>= count)
};

__device__ __forceinline__ bool capsule_covers(const Capsule& K, double s, double R,
                                               double eps) {
  const double r = sqrt(R) * (1.0 + 1e-12) + eps;
  const double t = s - K.sa;
  return r <= K.rho && t - r >= 0.0 && t + r <= K.L;
}

// Entry parameter of the segment P0 + t d, t in [t0, t1], into the box
// [lo, hi] inflated by w per axis, or +inf if it misses.  A point of the box
// within distance w of the line has its foot on the line inside the
// inflated box, so its axial parameter is at least the returned value (up
// to rounding); missing the inflated box means no point of the box lies
// within w of the segment.
__device__ __forceinline__ double seg_box_entry(const double P0[3], const double d[3],
                                                const double invd[3], double t0, double t1,
                                                float4 lo, float4 hi, double w) {
  const double l3[3] = {lo.x, lo.y, lo.z}, h3[3] = {hi.x, hi.y, hi.z};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double l = l3[j] - w - P0[j], h = h3[j] + w - P0[j];
    if (d[j] == 0.0) {
      if (l > 0.0 || h < 0.0) return pinf();
    } else {
      double a = l * invd[j], b = h * invd[j];
      if (a > b) {
        const double x = a;
        a = b;
        b = x;
      }
      t0 = fmax(t0, a);
      t1 = fmin(t1, b);
    }
  }
  return t0 <= t1 + 1e-9 ? t0 : pinf();
}

// float <-> int keys with the same order (finite values), for integer
// warp reductions of FP32 coordinates
__device__ __forceinline__ int ord_key(float f) {
  const int k = __float_as_int(f);
  return k >= 0 ? k : k ^ 0x7fffffff;
}
__device__ __forceinline__ float ord_val(int k) {
  return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff);
}

// Gather the capsule (start parameter sa, length L, radius rho) of ray g
// into `cache` and build the chunk boxes.  The traversal continues into the
// subtree the segment enters first; once the cache is full, the smallest
// axial parameter of a dropped point (tdrop) shortens the capsule to
// L' = tdrop - 2 eps, and subtrees entered beyond tdrop + eps are pruned (all
// their capsule points lie beyond L'), which bounds the work of a gather.
__device__ __forceinline__ Capsule warp_gather_capsule(const DevCloud& c, const int lane,
                                                       const RayGeom& g, double sa, double L,
                                                       double rho, double eps, float4* cache,
                                                       float4* cblo, float4* cbhi,
                                                       int* s_node, float* s_key,
                                                       unsigned& nver, unsigned& nsteps) {
  const int D = c.depth;
  const int64_t ninternal = c.nleaves - 1;
  double Pa[3], P0[3], invd[3];
  ray_point(g, sa, Pa[0], Pa[1], Pa[2]);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    P0[j] = Pa[j] - c.origin[j];  // frame of the node boxes
    invd[j] = g.d[j] != 0.0 ? 1.0 / g.d[j] : 0.0;
  }
  // node boxes bound the FP32 images; real points are within coord_err
  const double wbox = rho + (double)c.coord_err + eps;
  const double t_lo = -eps, t_hi = L + eps;
  const double rho2_in = rho * rho * (1.0 + 1e-12) + eps * eps;
  double tdrop = pinf();  // warp-uniform
  int count = 0;
  int sp = 0;
  bool lost = false;
  int64_t gfirst;
  int gm;
  bool gleaves;
  if (D == 0) {
    gfirst = 0;
    gm = 1;
    gleaves = true;
  } else {
    const int s = ((D - 1) % 5) + 1;
    gfirst = (1LL << s) - 1;
    gm = 1 << s;
    gleaves = (s == D);
  }
  for (;;) {
    ++nsteps;
    const int64_t node = gfirst + lane;
    double te = pinf();
    if (lane < gm)
      te = seg_box_entry(P0, g.d, invd, t_lo, t_hi, __ldg(&c.boxlo[node]),
                         __ldg(&c.boxhi[node]), wbox);
    const bool surv = te <= tdrop + eps;
    const unsigned mask = __ballot_sync(kFull, surv);
    bool next = false;
    int v = 0;
    if (gleaves) {
      if (mask) {
        int64_t a = 0;
        int cnt = 0;
        if (surv) {
          const int64_t j = node - ninternal;
          a = (j * c.n) >> D;
          cnt = (int)((((j + 1) * c.n) >> D) - a);
        }
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += t;
        }
        const int total = __shfl_sync(kFull, incl, 31);
        double tmin_drop = pinf();
        for (int base = 0; base < total; base += 32) {
          const int kk = base + lane;
          int lo = 0, hi = 31;
#pragma unroll
          for (int it = 0; it < 5; ++it) {
            const int mid = (lo + hi) >> 1;
            if (__shfl_sync(kFull, incl, mid) > kk) hi = mid;
            else lo = mid + 1;
          }
          const long long ao = __shfl_sync(kFull, (long long)a, lo);
          const int exo = __shfl_sync(kFull, incl - cnt, lo);
          const int64_t p = ao + (kk - exo);
          bool in = false;
          double tp = 0.0;
          if (kk < total) {
            const double4 P = ldg_pt(&c.pts[p]);
            const double ax = P.x - Pa[0], ay = P.y - Pa[1], az = P.z - Pa[2];
            tp = ax * g.d[0] + ay * g.d[1] + az * g.d[2];
            const double rx = ax - tp * g.d[0], ry = ay - tp * g.d[1], rz = az - tp * g.d[2];
            in = tp >= t_lo && tp <= t_hi && rx * rx + ry * ry + rz * rz < rho2_in;
            ++nver;
          }
          const unsigned im = __ballot_sync(kFull, in);
          const int pos = count + __popc(im & ((1u << lane) - 1u));
          if (in) {
            if (pos < kCache) {
              float4 P32 = __ldg(&c.pts32[p]);
              P32.w = __int_as_float((int)p);
              cache[pos] = P32;
            } else {
              tmin_drop = fmin(tmin_drop, tp);
            }
          }
          count += __popc(im);
        }
        if (count > kCache) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1)
            tmin_drop = fmin(tmin_drop, __shfl_xor_sync(kFull, tmin_drop, o));
          tdrop = fmin(tdrop, tmin_drop);
        }
      }
    } else if (mask) {
      // continue into the survivor entered first, remember the others
      const int key = surv ? ord_key(__double2float_rd(te)) : 0x7fffffff;
      const int kmin = __reduce_min_sync(kFull, key);
      const int w = __ffs(__ballot_sync(kFull, surv && key == kmin)) - 1;
      const unsigned rest = mask & ~(1u << w);
      const int cnt = __popc(rest);
      if (sp + cnt > kWSearchStack) {
        lost = true;  // subtrees not remembered: no guarantee
      } else {
        if ((rest >> lane) & 1u) {
          const int e = sp + __popc(rest & ((1u << lane) - 1u));
          s_node[e] = (int)node;
          s_key[e] = __double2float_rd(te);
        }
        sp += cnt;
      }
      __syncwarp();
      v = (int)(gfirst + w);
      next = true;
    }
    if (!next) {
      while (sp > 0) {
        --sp;
        if ((double)s_key[sp] <= tdrop + eps) {
          v = s_node[sp];
          next = true;
          break;
        }
      }
      __syncwarp();
      if (!next) break;
    }
    const int k = depth_of(v);
    const int s = min(5, D - k);
    gfirst = ((int64_t)(v + 1) << s) - 1;
    gm = 1 << s;
    gleaves = (k + s == D);
  }
  const int kept = count < kCache ? count : kCache;
  // tight FP32 box of each chunk of 32 cached points
  for (int k = 0; k * 32 < kept; ++k) {
    const int idx = k * 32 + lane;
    const bool h = idx < kept;
    float4 P = make_float4(0.f, 0.f, 0.f, 0.f);
    if (h) P = cache[idx];
    const int x0 = __reduce_min_sync(kFull, h ? ord_key(P.x) : 0x7fffffff);
    const int y0 = __reduce_min_sync(kFull, h ? ord_key(P.y) : 0x7fffffff);
    const int z0 = __reduce_min_sync(kFull, h ? ord_key(P.z) : 0x7fffffff);
    const int x1 = __reduce_max_sync(kFull, h ? ord_key(P.x) : (int)0x80000000);
    const int y1 = __reduce_max_sync(kFull, h ? ord_key(P.y) : (int)0x80000000);
    const int z1 = __reduce_max_sync(kFull, h ? ord_key(P.z) : (int)0x80000000);
    if (lane == 0) {
      cblo[k] = make_float4(ord_val(x0), ord_val(y0), ord_val(z0), 0.f);
      cbhi[k] = make_float4(ord_val(x1), ord_val(y1), ord_val(z1), 0.f);
    }
  }
  __syncwarp();
  Capsule K;
  K.sa = sa;
  K.rho = rho;
  K.count = kept;
  K.total = count;
  K.L = lost ? -1.0 : fmin(L, tdrop - 2.0 * eps);
  return K;
}

// Bounded 3-NN over the cached points (same acceptance rule as warp_knn):
// chunk boxes first, then the surviving chunks nearest first.  The FP32
// guard band shrinks with the threshold: guard_band(T, qe) bounds the FP32
// error of every point with d < T.
__device__ __forceinline__ void warp_scan_cache(const DevCloud& c, const int lane,
                                                const WarpQuery& Q, const double qe,
                                                const float4* cache, const float4* cblo,
                                                const float4* cbhi, const int count,
                                                KnnList<3>& L, unsigned& nver) {
  L.clear();
  double thr64 = Q.bound;
  float thr32 = __double2float_ru(dadd(thr64, Q.G));
  const int nch = (count + 31) >> 5;
  float bd = __int_as_float(0x7f800000);
  if (lane < nch) bd = box_dist32(Q.q0, Q.q1, Q.q2, cblo[lane], cbhi[lane]);
  unsigned m = __ballot_sync(kFull, lane < nch && bd < thr32);
  while (m) {
    const unsigned key = ((m >> lane) & 1u) ? __float_as_uint(bd) : 0xffffffffu;
    const unsigned kmin = __reduce_min_sync(kFull, key);
    const int k = __ffs(__ballot_sync(kFull, key == kmin)) - 1;
    m &= ~(1u << k);
    const int idx = k * 32 + lane;
    bool cand = false;
    int p = -1;
    if (idx < count) {
      const float4 P = cache[idx];
      p = __float_as_int(P.w);
      cand = pt_dist32(Q.q0, Q.q1, Q.q2, P) < thr32;
    }
    unsigned cm = __ballot_sync(kFull, cand);
    if (cm) {
      double d = 0.0;
      if (cand) {
        if (p == Q.cid) d = Q.dc;
        else if (p == Q.nid) d = Q.dn;
        else {
          d = metric(Q.x, Q.y, Q.z, ldg_pt(&c.pts[p]));
          ++nver;
        }
      }
      bool changed = false;
      while (cm) {
        const int jj = __ffs(cm) - 1;
        cm &= cm - 1;
        const double dj = __shfl_sync(kFull, d, jj);
        const int pj = __shfl_sync(kFull, p, jj);
        if (dj < thr64) {
          L.insert(dj, pj);
          thr64 = fmin(Q.bound, L.worst());
          changed = true;
        }
      }
      if (changed) thr32 = __double2float_ru(dadd(thr64, guard_band(thr64, qe)));
    }
    m &= __ballot_sync(kFull, bd < thr32);
  }
}

// ------------------------------------------------------------------ sinks
// Lane-parallel reduction: lane f accumulates field f (f < nf <= 32) with
// the reference's sequence of operations per field.
template <int MODE>
struct WarpReducer {
  double acc, T;
  unsigned nseg;
  __device__ __forceinline__ void init() {
    nseg = 0;
    T = 1.0;
    acc = MODE == kMax ? -pinf() : (MODE == kMin ? pinf() : 0.0);
  }
  __device__ __forceinline__ void seg(const DevCloud& c, int lane, int cell, double a, double b) {
    ++nseg;
    const double ds = dsub(b, a);
    if (MODE == kVolume) {
      const double* F = c.fields + (int64_t)cell * 4;
      const double alpha = F[3];
      const double opac = dsub(1.0, exp(dmul(-alpha, ds)));
      if (lane < 3) acc = dadd(acc, dmul(dmul(T, F[lane]), opac));
      T = dmul(T, dsub(1.0, opac));
    } else if (lane < c.nf) {
      const double v = c.fields[(int64_t)cell * c.nf + lane];
      if (MODE == kSum) acc = dadd(acc, dmul(ds, v));
      else if (MODE == kMax) acc = v > acc ? v : acc;
      else acc = v < acc ? v : acc;
    }
  }
};

// Lane-parallel adjoint (see AdjSink): lane f scatters field f.
template <int MODE>
struct WarpAdj {
  double g, C, P, T;
  unsigned nseg, skip;
  __device__ __forceinline__ void init(const WalkIO& io, int lane, int64_t ray, unsigned sk) {
    nseg = 0;
    skip = sk;
    T = 1.0;
    P = 0.0;
    g = lane < io.nout ? io.gout[ray * io.nout + lane] : 0.0;
    C = (MODE == kVolume && lane < 3) ? io.fwd[ray * 3 + lane] : 0.0;
  }
  __device__ __forceinline__ void seg(const DevCloud& c, const WalkIO& io, int lane, int cell,
                                      double a, double b) {
    const bool emit = nseg >= skip;
    ++nseg;
    const double ds = dsub(b, a);
    const int64_t pid = c.perm[cell];
    if (MODE == kVolume) {
      const double* F = c.fields + (int64_t)cell * 4;
      const double alpha = F[3];
      const double e = exp(dmul(-alpha, ds));
      const double o = dsub(1.0, e);
      double term = 0.0;
      if (lane < 3) {
        const double Fk = F[lane];
        P = dadd(P, dmul(dmul(T, Fk), o));
        term = g * (T * Fk * e - (C - P));
        if (emit) atomicAdd(&io.grad[pid * 4 + lane], g * T * o);
      }
      term += __shfl_down_sync(kFull, term, 1);
      term += __shfl_down_sync(kFull, term, 2);
      if (emit && lane == 0) atomicAdd(&io.grad[pid * 4 + 3], ds * term);
      T = dmul(T, dsub(1.0, o));
    } else if (emit && lane < c.nf) {
      atomicAdd(&io.grad[pid * c.nf + lane], g * ds);
    }
  }
};

// --------------------------------------------------------------- kernel
template <int MODE, int OUT>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, VT_WARP_MINB) k_warp(DevCloud c, WalkIO io) {
  __shared__ int s_node_all[kWarpsPerBlock][kWSearchStack];
  __shared__ float s_mind_all[kWarpsPerBlock][kWSearchStack];
  __shared__ int w_id_all[kWarpsPerBlock][kWWalkStack];
  __shared__ double w_s_all[kWarpsPerBlock][kWWalkStack];
  __shared__ float4 cache_all[kWarpsPerBlock][kCache];
  __shared__ float4 cblo_all[kWarpsPerBlock][kChunks];
  __shared__ float4 cbhi_all[kWarpsPerBlock][kChunks];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  int* s_node = s_node_all[wib];
  float* s_mind = s_mind_all[wib];
  int* w_id = w_id_all[wib];
  double* w_s = w_s_all[wib];
  float4* cache = cache_all[wib];
  float4* cblo = cblo_all[wib];
  float4* cbhi = cbhi_all[wib];
  const double cerr = (double)c.coord_err;
  // capsule radius / local 3-NN radius, and length / radius (adapted per
  // warp so that a gather about fills the cache)
  const double cap_kappa = 2.0;
  double cap_lambda = 14.0;
  const bool use_cache = io.cache_mode != 0;
  unsigned n_rays = 0, n_cross = 0, n_q = 0, n_res = 0, n_ver = 0, n_steps = 0, max_sp = 0;
  unsigned n_refresh = 0, n_hit = 0;

  for (;;) {
    long long ray = 0;
    if (lane == 0) ray = (long long)atomicAdd(&io.stats->next_ray, 1ULL);
    ray = __shfl_sync(kFull, ray, 0);
    if (ray >= io.nrays) break;
    if (io.order) ray = io.order[ray];
    RayGeom g;
    ray_init(g, io.starts + 3 * ray, io.ends + 3 * ray);
    if (!ray_finite(g)) {
      if (lane == 0) report(io, ray, kErrNonFinite);
      continue;
    }
    ++n_rays;
    double qe = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j)
      qe = fmax(qe, fmax(fabs(g.s[j] - c.origin[j]), fabs(g.e[j] - c.origin[j])));
    qe = qe * 6.0e-8 + cerr;

    WarpReducer<MODE> red;
    WarpAdj<MODE> adj;
    unsigned fill_n = 0;
    int64_t fill_off = 0;
    if (OUT == kOutImage || OUT == kOutCount || OUT == kOutTape) red.init();
    else if (OUT == kOutFill) fill_off = io.offsets[ray];
    else adj.init(io, lane, ray, 0u);
    auto emit = [&](int cell, double a, double b) {
      if (OUT == kOutImage || OUT == kOutCount) red.seg(c, lane, cell, a, b);
      else if (OUT == kOutTape) {
        // the reducer, then lane 0 records the segment (for 'volume' with the
        // transmittance in front of it and the colour composited up to it)
        const double T0 = red.T;
        red.seg(c, lane, cell, a, b);
        if (MODE == kVolume) {
          const double p0 = __shfl_sync(kFull, red.acc, 0);
          const double p1 = __shfl_sync(kFull, red.acc, 1);
          const double p2 = __shfl_sync(kFull, red.acc, 2);
          if (lane == 0) tape_append(io, TapeEntryV{cell, (int)ray, dsub(b, a), T0, {p0, p1, p2}});
        } else if (lane == 0) {
          tape_append(io, TapeEntry{c.perm[cell], (int)ray, dsub(b, a)});
        }
      } else if (OUT == kOutFill) {
        if (lane == 0) {
          io.seg_cell[fill_off + fill_n] = c.perm[cell];
          io.seg_enter[fill_off + fill_n] = a;
          io.seg_exit[fill_off + fill_n] = b;
        }
        ++fill_n;
      } else adj.seg(c, io, lane, cell, a, b);
    };
    auto nseg_now = [&]() -> unsigned {
      return (OUT == kOutImage || OUT == kOutCount || OUT == kOutTape)
                 ? red.nseg
                 : (OUT == kOutFill ? fill_n : adj.nseg);
    };

    // ---- end cells: leaf on the split-plane path, then a bounded search
    WarpQuery Q;
    Q.qe = qe;
    // (2 nearest, so that an exact tie at the nearest distance is seen:
    // such a ray is handed to k_slow, which answers it in the reference's
    // order)
    auto nn_end = [&](double x, double y, double z) -> int {
      warp_query_setup(Q, c, x, y, z);
      KnnList<2> r1;
      r1.clear();
      const int64_t leaf = warp_descend_leaf(c, Q.q0, Q.q1, Q.q2);
      const int64_t a = (leaf * c.n) >> c.depth;
      const int cnt = (int)((((leaf + 1) * c.n) >> c.depth) - a);
      for (int base = 0; base < cnt; base += 32) {
        const int kk = base + lane;
        double d = 0.0;
        if (kk < cnt) d = metric(x, y, z, ldg_pt(&c.pts[a + kk]));
        const int m = min(32, cnt - base);
        for (int j = 0; j < m; ++j) {
          const double dj = __shfl_sync(kFull, d, j);
          if (dj < r1.worst()) r1.insert(dj, (int)(a + base + j));
        }
      }
      Q.bound = pinf();
      Q.G = guard_band(r1.worst(), qe);  // the threshold never exceeds it
      Q.cid = Q.nid = -1;
      Q.dc = Q.dn = 0.0;
      ++n_q;
      if (!warp_knn<2>(c, lane, Q, leaf, r1, s_node, s_mind, n_ver, n_steps)) {
        // search stack overflow: exact thread-level search by lane 0
        ++n_res;
        int id = -1;
        if (lane == 0) {
          unsigned v = 0;
          id = nn1_exact64(c, x, y, z, v);
        }
        return __shfl_sync(kFull, id, 0);
      }
      if (r1.id[0] >= 0 && r1.id[1] >= 0 && r1.r2[1] == r1.r2[0]) return kTieUnresolved;
      return r1.id[0];
    };
    const int c0 = nn_end(g.s[0], g.s[1], g.s[2]);
    const int c1 = nn_end(g.e[0], g.e[1], g.e[2]);
    if (c0 == kTieUnresolved || c1 == kTieUnresolved) {
      if (lane == 0) hand_over(io, ray, 0u);
      continue;
    }
    if (c0 < 0 || c1 < 0) {
      if (lane == 0) report(io, ray, kErrNonFiniteDist);
      continue;
    }
    // capsule cache of this ray (empty)
    Capsule cap;
    cap.sa = 0.0;
    cap.L = -1.0;
    cap.rho = 0.0;
    cap.count = 0;
    cap.total = 0;
    // absolute FP64 slack of the capsule tests (a few ulp of the coordinates)
    const double cap_eps = 1e-12 * (qe / 6.0e-8 + g.len + 1.0);
    int rc = 0;
    int cur = c0, open_cell = c0;
    double cur_s = 0.0, entry_s = 0.0;
    if (c0 == c1) {
      emit(c0, 0.0, g.len);
    } else {
      int sp = 1;
      if (lane == 0) {
        w_id[0] = c1;
        w_s[0] = g.len;
      }
      __syncwarp();
      int64_t iter = 0;
      for (;;) {
        if (++iter > io.max_iter) {
          rc = kErrMaxIter;
          break;
        }
        const int nxt = w_id[sp - 1];
        const double nxt_s = w_s[sp - 1];
        if (dsub(nxt_s, cur_s) < 1e-14) {  // zero-width skip
          --sp;
          cur = nxt;
          cur_s = nxt_s;
          open_cell = cur;
          if (sp == 0) break;
          continue;
        }
        const double4 pc = ldg_pt(&c.pts[cur]);
        const double4 pn = ldg_pt(&c.pts[nxt]);
        double s = split_analytic(g, pc, pn);
        if (!(s < DBL_MAX * 0.5 && s >= cur_s - kTol && s <= nxt_s + kTol)) {
          RareOut ro{0.0, 0, 0, 0, 0u};
          if (lane == 0) ro = rare_split(c, g, cur, nxt, cur_s, nxt_s);
          s = __shfl_sync(kFull, ro.s, 0);
          rc = __shfl_sync(kFull, ro.rc, 0);
          n_q += ro.nq;
          if (rc) break;
          if (s < dsub(cur_s, kTol) || s > dadd(nxt_s, kTol)) {
            rc = kErrSplitBounds;
            break;
          }
        }
        {
          const double lo = dadd(cur_s, 1e-15), hi = dsub(nxt_s, 1e-15);
          s = (s < lo) ? lo : (hi < s) ? hi : s;
        }
        double x, y, z;
        ray_point(g, s, x, y, z);
        warp_query_setup(Q, c, x, y, z);
        Q.dc = metric(x, y, z, pc);
        Q.dn = metric(x, y, z, pn);
        Q.cid = cur;
        Q.nid = nxt;
        Q.bound = dadd(fmax(Q.dc, Q.dn), 4.0 * kTol);
        Q.G = guard_band(Q.bound, qe);
        KnnList<3> r;
        r.clear();
        ++n_q;
        bool good;
        bool hit = false;
        if (use_cache && cap.L > 0.0 && s > cap.sa && s < cap.sa + cap.L) {
          warp_scan_cache(c, lane, Q, qe, cache, cblo, cbhi, cap.count, r, n_ver);
          if (capsule_covers(cap, s, fmin(Q.bound, r.worst()), cap_eps)) {
            good = true;
            hit = true;
            ++n_hit;
          }
        }
        if (!hit) {
          r.clear();  // a scan that missed leaves partial results
          good = warp_knn<3>(c, lane, Q, -1, r, s_node, s_mind, n_ver, n_steps);
        }
        if (!good || !knn3_decision_valid(r, Q.bound)) {
          ++n_res;
          good = warp_knn_unbounded<3>(c, lane, Q, qe, r, s_node, s_mind, n_ver, n_steps);
          if (!good) {
            // exact thread-level search by lane 0, broadcast
            KnnList<3> t;
            t.clear();
            if (lane == 0) {
              unsigned v = 0;
              knn_exact64(c, x, y, z, pinf(), t, v);
            }
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              r.r2[j] = __shfl_sync(kFull, t.r2[j], 0);
              r.id[j] = __shfl_sync(kFull, t.id[j], 0);
            }
          }
        }
        if (r.id[0] < 0) {
          rc = kErrNonFiniteDist;
          break;
        }
        if (use_cache && !hit) {
          // Re-gather around the walk's current point when this query is
          // local (its ball would lie in the new capsule); far split points
          // of the bisection phase do not move the capsule.
          const double rloc = sqrt(fmin(Q.bound, r.worst()));
          const double rho = cap_kappa * rloc;
          const double len = cap_lambda * rho;
          if (rho > 0.0 && s - cur_s + rloc + rho <= len) {
            cap = warp_gather_capsule(c, lane, g, cur_s - rho, len, rho, cap_eps, cache, cblo,
                                      cbhi, s_node, s_mind, n_ver, n_steps);
            ++n_refresh;
            if (cap.total > kCache)
              cap_lambda = fmax(2.0 * cap_kappa + 2.0, cap_lambda * 0.8);
            else if (cap.total < (kCache * 3) / 4)
              cap_lambda = fmin(400.0, cap_lambda * fmin(2.0, (0.85 * kCache) / fmax(1.0, (double)cap.total)));
          }
        }
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
          RareOut ro{0.0, 0, 0, 0, 0u};
          if (lane == 0) ro = rare_expand(c, x, y, z, cur, nxt);
          rc = __shfl_sync(kFull, ro.rc, 0);
          has_c = __shfl_sync(kFull, ro.a, 0);
          has_n = __shfl_sync(kFull, ro.b, 0);
          ++n_q;
          if (rc) break;
        }
        if (has_c || has_n) {
          emit(open_cell, entry_s, s);
          open_cell = nxt;
          entry_s = s;
          --sp;
          cur = nxt;
          cur_s = nxt_s;
          if (sp == 0) break;
        } else if (dadd(r.r2[0], kTol) < r.r2[1]) {
          if (sp >= kWWalkStack || sp >= io.local_cap) {
            rc = kNeedSlow;
            break;
          }
          if (lane == 0) {
            w_id[sp] = r.id[0];
            w_s[sp] = s;
          }
          ++sp;
          __syncwarp();
        } else {
          RareOut ro{0.0, 0, 0, 0, 0u};
          if (lane == 0) ro = rare_case1a(c, g, x, y, z, cur, nxt);
          rc = __shfl_sync(kFull, ro.rc, 0);
          const int sc = __shfl_sync(kFull, ro.a, 0), sn = __shfl_sync(kFull, ro.b, 0);
          n_q += ro.nq;
          if (rc) break;
          const int need = sc == sn ? 1 : 2;
          if (sp + need > kWWalkStack || sp + need > io.local_cap) {
            rc = kNeedSlow;
            break;
          }
          if (lane == 0) {
            if (sc == sn) {
              w_id[sp] = sc;
              w_s[sp] = s;
            } else {
              w_id[sp] = sn;
              w_s[sp] = s;
              w_id[sp + 1] = sc;
              w_s[sp + 1] = s;
            }
          }
          sp += need;
          __syncwarp();
        }
        max_sp = max(max_sp, (unsigned)sp);
      }
      if (rc == 0) emit(open_cell, entry_s, cur_s);
    }
    if (rc == 0) {
      if (OUT == kOutImage || OUT == kOutCount || OUT == kOutTape) {
        if (lane < io.nout) io.out[ray * io.nout + lane] = red.acc;
        if (OUT == kOutCount && lane == 0) io.counts[ray] = red.nseg;
      }
      n_cross += nseg_now();
    } else if (lane == 0) {
      if (rc == kNeedSlow || rc == kNeedTie) hand_over(io, ray, nseg_now());
      else report(io, ray, rc);
    }
    __syncwarp();
  }
  if (lane == 0) {
    atomicAdd(&io.stats->rays, (unsigned long long)n_rays);
    atomicAdd(&io.stats->crossings, (unsigned long long)n_cross);
    atomicAdd(&io.stats->queries, (unsigned long long)n_q);
    atomicAdd(&io.stats->fp64_resolves, (unsigned long long)n_res);
    atomicMax(&io.stats->max_stack, (unsigned long long)max_sp);
    atomicAdd(&io.stats->search_steps, (unsigned long long)n_steps);
    atomicAdd(&io.stats->fp64_checks, (unsigned long long)n_ver);
    atomicAdd(&io.stats->cache_refreshes, (unsigned long long)n_refresh);
    atomicAdd(&io.stats->cache_hits, (unsigned long long)n_hit);
  }
}

template <int MODE, int OUT>
int launch_warp(vt_cloud* cl, WalkIO& io, cudaStream_t st) {
  const int B = kWarpsPerBlock * 32;
  int dev = 0, nsms = 0;
  VT_CUDA(cudaGetDevice(&dev));
  VT_CUDA(cudaDeviceGetAttribute(&nsms, cudaDevAttrMultiProcessorCount, dev));
  int per_sm = cl->blocks_per_sm;
  if (per_sm <= 0) {
    VT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_warp<MODE, OUT>, B, 0));
    if (per_sm < 1) per_sm = 1;
  }
  int64_t blocks = (int64_t)nsms * per_sm;
  const int64_t need = (io.nrays + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (blocks > need) blocks = need > 0 ? need : 1;
  k_warp<MODE, OUT><<<(unsigned)blocks, B, 0, st>>>(cl->view, io);
  return VT_OK;
}

}  // namespace vt
