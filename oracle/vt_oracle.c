/*
 * vt_oracle.c -- CPU restatement of vortrace's exact Voronoi ray walk.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (vortrace_b200/) links,
 * loads or calls this file; it is the checker that the CUDA path is compared
 * against, and the "port" CPU baseline of bench.py.  It is pinned against the
 * reference itself (oracle/_ref, compiled from the reference's sources by
 * oracle/build_ref.sh) and against the reference's golden projection.
 *
 * What is restated, with the reference location each part follows
 * (paths are within the gusbeane/vortrace project):
 *   - kD-tree build: nanoflann v1.3.2 as vendored in include/nanoflann.hpp
 *       divideTree        include/nanoflann.hpp:858-905
 *       middleSplit_      include/nanoflann.hpp:910-956
 *       planeSplit        include/nanoflann.hpp:967-1003
 *       computeMinMax     include/nanoflann.hpp:837-849
 *       computeBoundingBox include/nanoflann.hpp:1316-1336
 *     with leaf_max_size 10 (src/pointcloud.cpp:204).  The tree is rebuilt
 *     with the same split rule so that exact-tie answers (lattices) come out
 *     in the same order as the reference's.
 *   - k-NN search: findNeighbors/searchLevel/KNNResultSet::addPoint/
 *     L2_Simple_Adaptor::evalMetric/computeInitialDistances
 *       include/nanoflann.hpp:1221-1241, 1346-1408, 175-201, 432-445, 1005-1021
 *   - the walk: Ray::Ray, findSplitPointDistance (both overloads),
 *     perpPerturbToFindCell, Ray::walk      src/ray.cpp:14-35, 38-127, 129-185, 187-430
 *   - reductions: reduce_sum/max/min/volume_render  src/reduction.cpp:8-83
 *   - the per-ray driver: Projection::makeProjection /
 *     makeDetailedProjection                src/projection.cpp:26-144
 * Periodic mode (src/pointcloud.cpp:313-367, src/ray.cpp:71-86,220-246) is
 * not restated.
 *
 * Floating point: every FP64 expression keeps the reference's operation
 * order; build with -ffp-contract=off so no FMA is formed.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define VTO_TOLERANCE 1e-9              /* src/ray.cpp:8 */
#define VTO_PARALLEL_BISECTOR_TOL 1e-12 /* src/ray.cpp:9 */
#define VTO_MAX_ITERATIONS 100000       /* src/ray.cpp:10 */
#define VTO_PERTURBATION_EPS (2 * VTO_TOLERANCE) /* src/ray.cpp:11 */
#define VTO_MAX_PERTURBATION_CYCLES 1000 /* src/ray.cpp:12 */
#define VTO_K_EXPAND 100                /* src/ray.cpp:321 */
#define VTO_NONE ((size_t)-1)

/* status codes (same meaning as the product's VT_ERR_* codes) */
enum {
  VTO_OK = 0,
  VTO_ERR_INVALID = 1,
  VTO_ERR_MAX_ITER = 10,
  VTO_ERR_SPLIT_BOUNDS = 11,
  VTO_ERR_BINSEARCH = 12,
  VTO_ERR_PERTURB = 13,
  VTO_ERR_KNN_EXPAND = 14,
  VTO_ERR_NOMEM = 20
};

/* reduction modes, src/../include/mytypes.hpp:14 */
enum { VTO_SUM = 0, VTO_MAX = 1, VTO_MIN = 2, VTO_VOLUME = 3 };

typedef struct { double low, high; } vto_iv;

typedef struct {
  int64_t child1, child2; /* -1 for both: leaf */
  int divfeat;
  size_t left, right;     /* leaf: vind range [left, right) */
  double divlow, divhigh;
} vto_node;

typedef struct {
  double *pts; /* own copy, n x 3 */
  size_t n;
  size_t leaf_max;
  size_t *vind;
  vto_node *nodes;
  size_t nnodes, cap;
  int64_t root;
  vto_iv root_bbox[3];
} vto_tree;

static inline double P(const vto_tree *t, size_t idx, int d) { return t->pts[idx * 3 + d]; }

/* Work counters of the k-NN searches (per thread; summed by vto_project):
 * queries, tree nodes visited (searchLevel calls), leaves visited, point
 * distance evaluations.  They define the algorithmic bytes per crossing of
 * the reference's own search (used for the roofline of the GPU kernels). */
static __thread unsigned long long tl_cnt[4];
static unsigned long long g_cnt[4];

/* ------------------------------------------------------------------ build */

static int64_t alloc_node(vto_tree *t) {
  if (t->nnodes == t->cap) {
    size_t nc = t->cap ? t->cap * 2 : 1024;
    vto_node *nn = (vto_node *)realloc(t->nodes, nc * sizeof(vto_node));
    if (!nn) return -1;
    t->nodes = nn;
    t->cap = nc;
  }
  memset(&t->nodes[t->nnodes], 0, sizeof(vto_node));
  return (int64_t)t->nnodes++;
}

/* include/nanoflann.hpp:837-849 */
static void compute_min_max(const vto_tree *t, const size_t *ind, size_t count, int e,
                            double *mn, double *mx) {
  *mn = P(t, ind[0], e);
  *mx = P(t, ind[0], e);
  for (size_t i = 1; i < count; ++i) {
    double v = P(t, ind[i], e);
    if (v < *mn) *mn = v;
    if (v > *mx) *mx = v;
  }
}

/* include/nanoflann.hpp:967-1003: two in-place partitions, the first moving
 * values < cutval to the front, the second moving values == cutval next. */
static void plane_split(const vto_tree *t, size_t *ind, size_t count, int cutfeat, double cutval,
                        size_t *lim1, size_t *lim2) {
  size_t left = 0, right = count - 1;
  for (;;) {
    while (left <= right && P(t, ind[left], cutfeat) < cutval) ++left;
    while (right && left <= right && P(t, ind[right], cutfeat) >= cutval) --right;
    if (left > right || !right) break;
    size_t tmp = ind[left]; ind[left] = ind[right]; ind[right] = tmp;
    ++left;
    --right;
  }
  *lim1 = left;
  right = count - 1;
  for (;;) {
    while (left <= right && P(t, ind[left], cutfeat) <= cutval) ++left;
    while (right && left <= right && P(t, ind[right], cutfeat) > cutval) --right;
    if (left > right || !right) break;
    size_t tmp = ind[left]; ind[left] = ind[right]; ind[right] = tmp;
    ++left;
    --right;
  }
  *lim2 = left;
}

/* include/nanoflann.hpp:910-956 */
static void middle_split(const vto_tree *t, size_t *ind, size_t count, size_t *index,
                         int *cutfeat, double *cutval, const vto_iv *bbox) {
  const double EPS = 0.00001;
  double max_span = bbox[0].high - bbox[0].low;
  for (int i = 1; i < 3; ++i) {
    double span = bbox[i].high - bbox[i].low;
    if (span > max_span) max_span = span;
  }
  double max_spread = -1;
  *cutfeat = 0;
  for (int i = 0; i < 3; ++i) {
    double span = bbox[i].high - bbox[i].low;
    if (span > (1 - EPS) * max_span) {
      double mn, mx;
      compute_min_max(t, ind, count, i, &mn, &mx);
      double spread = mx - mn;
      if (spread > max_spread) {
        *cutfeat = i;
        max_spread = spread;
      }
    }
  }
  double split_val = (bbox[*cutfeat].low + bbox[*cutfeat].high) / 2;
  double mn, mx;
  compute_min_max(t, ind, count, *cutfeat, &mn, &mx);
  if (split_val < mn) *cutval = mn;
  else if (split_val > mx) *cutval = mx;
  else *cutval = split_val;
  size_t lim1, lim2;
  plane_split(t, ind, count, *cutfeat, *cutval, &lim1, &lim2);
  if (lim1 > count / 2) *index = lim1;
  else if (lim2 < count / 2) *index = lim2;
  else *index = count / 2;
}

/* include/nanoflann.hpp:858-905.  bbox is in/out: on return it holds the
 * tight box of the node's points. */
static int64_t divide_tree(vto_tree *t, size_t left, size_t right, vto_iv *bbox) {
  int64_t ni = alloc_node(t);
  if (ni < 0) return -1;
  if ((right - left) <= t->leaf_max) {
    t->nodes[ni].child1 = t->nodes[ni].child2 = -1;
    t->nodes[ni].left = left;
    t->nodes[ni].right = right;
    for (int i = 0; i < 3; ++i) {
      bbox[i].low = P(t, t->vind[left], i);
      bbox[i].high = P(t, t->vind[left], i);
    }
    for (size_t k = left + 1; k < right; ++k) {
      for (int i = 0; i < 3; ++i) {
        if (bbox[i].low > P(t, t->vind[k], i)) bbox[i].low = P(t, t->vind[k], i);
        if (bbox[i].high < P(t, t->vind[k], i)) bbox[i].high = P(t, t->vind[k], i);
      }
    }
  } else {
    size_t idx;
    int cutfeat;
    double cutval;
    middle_split(t, t->vind + left, right - left, &idx, &cutfeat, &cutval, bbox);
    t->nodes[ni].divfeat = cutfeat;
    vto_iv left_bbox[3], right_bbox[3];
    memcpy(left_bbox, bbox, sizeof(left_bbox));
    left_bbox[cutfeat].high = cutval;
    int64_t c1 = divide_tree(t, left, left + idx, left_bbox);
    memcpy(right_bbox, bbox, sizeof(right_bbox));
    right_bbox[cutfeat].low = cutval;
    int64_t c2 = divide_tree(t, left + idx, right, right_bbox);
    if (c1 < 0 || c2 < 0) return -1;
    t->nodes[ni].child1 = c1;
    t->nodes[ni].child2 = c2;
    t->nodes[ni].divlow = left_bbox[cutfeat].high;
    t->nodes[ni].divhigh = right_bbox[cutfeat].low;
    for (int i = 0; i < 3; ++i) {
      bbox[i].low = left_bbox[i].low < right_bbox[i].low ? left_bbox[i].low : right_bbox[i].low;
      bbox[i].high = left_bbox[i].high > right_bbox[i].high ? left_bbox[i].high : right_bbox[i].high;
    }
  }
  return ni;
}

void vto_tree_free(vto_tree *t) {
  if (!t) return;
  free(t->pts);
  free(t->vind);
  free(t->nodes);
  free(t);
}

/* Build over n points (AoS x,y,z).  src/pointcloud.cpp:193-212 and
 * include/nanoflann.hpp:1190-1202. */
vto_tree *vto_tree_build(const double *pts, size_t n, size_t leaf_max) {
  if (n == 0) return NULL;
  vto_tree *t = (vto_tree *)calloc(1, sizeof(vto_tree));
  if (!t) return NULL;
  t->n = n;
  t->leaf_max = leaf_max;
  t->pts = (double *)malloc(n * 3 * sizeof(double));
  t->vind = (size_t *)malloc(n * sizeof(size_t));
  if (!t->pts || !t->vind) { vto_tree_free(t); return NULL; }
  memcpy(t->pts, pts, n * 3 * sizeof(double));
  for (size_t i = 0; i < n; ++i) t->vind[i] = i;
  for (int i = 0; i < 3; ++i) t->root_bbox[i].low = t->root_bbox[i].high = P(t, 0, i);
  for (size_t k = 1; k < n; ++k)
    for (int i = 0; i < 3; ++i) {
      if (P(t, k, i) < t->root_bbox[i].low) t->root_bbox[i].low = P(t, k, i);
      if (P(t, k, i) > t->root_bbox[i].high) t->root_bbox[i].high = P(t, k, i);
    }
  t->root = divide_tree(t, 0, n, t->root_bbox);
  if (t->root < 0) { vto_tree_free(t); return NULL; }
  return t;
}

size_t vto_tree_nnodes(const vto_tree *t) { return t ? t->nnodes : 0; }

/* ----------------------------------------------------------------- search */

typedef struct {
  size_t *ids;
  double *dists;
  size_t capacity, count;
} vto_result;

/* include/nanoflann.hpp:157-163 */
static inline void result_init(vto_result *r, size_t *ids, double *dists, size_t k) {
  r->ids = ids;
  r->dists = dists;
  r->capacity = k;
  r->count = 0;
  if (k) dists[k - 1] = DBL_MAX;
}

/* include/nanoflann.hpp:175-201: stable insertion, shift only on strict > */
static inline void result_add(vto_result *r, double dist, size_t index) {
  size_t i;
  for (i = r->count; i > 0; --i) {
    if (r->dists[i - 1] > dist) {
      if (i < r->capacity) {
        r->dists[i] = r->dists[i - 1];
        r->ids[i] = r->ids[i - 1];
      }
    } else
      break;
  }
  if (i < r->capacity) {
    r->dists[i] = dist;
    r->ids[i] = index;
  }
  if (r->count < r->capacity) r->count++;
}

static inline double worst_dist(const vto_result *r) { return r->dists[r->capacity - 1]; }

/* include/nanoflann.hpp:432-439: ((0 + d0*d0) + d1*d1) + d2*d2 with d = q - p */
static inline double eval_metric(const vto_tree *t, const double *q, size_t idx) {
  double result = 0.0;
  for (int i = 0; i < 3; ++i) {
    const double diff = q[i] - P(t, idx, i);
    result += diff * diff;
  }
  return result;
}

/* include/nanoflann.hpp:1346-1408 */
static void search_level(const vto_tree *t, vto_result *r, const double *vec, int64_t ni,
                         double mindistsq, double *dists) {
  const vto_node *node = &t->nodes[ni];
  tl_cnt[1]++;
  if (node->child1 < 0 && node->child2 < 0) {
    tl_cnt[2]++;
    tl_cnt[3] += node->right - node->left;
    double wd = worst_dist(r);
    for (size_t i = node->left; i < node->right; ++i) {
      size_t index = t->vind[i];
      double dist = eval_metric(t, vec, index);
      if (dist < wd) result_add(r, dist, index);
    }
    return;
  }
  int idx = node->divfeat;
  double val = vec[idx];
  double diff1 = val - node->divlow;
  double diff2 = val - node->divhigh;
  int64_t best, other;
  double cut_dist;
  if ((diff1 + diff2) < 0) {
    best = node->child1;
    other = node->child2;
    cut_dist = (val - node->divhigh) * (val - node->divhigh);
  } else {
    best = node->child2;
    other = node->child1;
    cut_dist = (val - node->divlow) * (val - node->divlow);
  }
  search_level(t, r, vec, best, mindistsq, dists);
  double dst = dists[idx];
  mindistsq = mindistsq + cut_dist - dst;
  dists[idx] = cut_dist;
  /* epsError = 1 + 0.0f (SearchParams default eps) */
  if (mindistsq * (double)1.0f <= worst_dist(r)) search_level(t, r, vec, other, mindistsq, dists);
  dists[idx] = dst;
}

/* knnSearch: include/nanoflann.hpp:1252-1259 + findNeighbors :1221-1241.
 * Returns the number of valid results.  Unfilled r2 slots: the last one is
 * DBL_MAX (KNNResultSet::init), the others are left untouched. */
size_t vto_knn(const vto_tree *t, const double *q, size_t k, size_t *ids, double *r2) {
  vto_result r;
  result_init(&r, ids, r2, k);
  if (!t || t->n == 0 || k == 0) return 0;
  tl_cnt[0]++;
  double dists[3] = {0.0, 0.0, 0.0};
  double distsq = 0.0;
  for (int i = 0; i < 3; ++i) {
    if (q[i] < t->root_bbox[i].low) {
      dists[i] = (q[i] - t->root_bbox[i].low) * (q[i] - t->root_bbox[i].low);
      distsq += dists[i];
    }
    if (q[i] > t->root_bbox[i].high) {
      dists[i] = (q[i] - t->root_bbox[i].high) * (q[i] - t->root_bbox[i].high);
      distsq += dists[i];
    }
  }
  search_level(t, &r, q, t->root, distsq, dists);
  return r.count;
}

/* batch helper for tests: nq queries, k each; missing entries get id -1 and
 * r2 = DBL_MAX */
void vto_knn_batch(const vto_tree *t, const double *q, size_t nq, size_t k, int64_t *ids,
                   double *r2) {
#pragma omp parallel
  {
    size_t *tid = (size_t *)malloc(k * sizeof(size_t));
    double *tr2 = (double *)malloc(k * sizeof(double));
#pragma omp for schedule(static)
    for (long long i = 0; i < (long long)nq; ++i) {
      size_t cnt = vto_knn(t, q + 3 * i, k, tid, tr2);
      for (size_t j = 0; j < k; ++j) {
        ids[i * k + j] = j < cnt ? (int64_t)tid[j] : -1;
        r2[i * k + j] = j < cnt ? tr2[j] : DBL_MAX;
      }
    }
    free(tid);
    free(tr2);
  }
}

static size_t query1(const vto_tree *t, const double *q) {
  size_t id = VTO_NONE;
  double r2;
  vto_knn(t, q, 1, &id, &r2);
  return id;
}

/* ------------------------------------------------------------------- walk */

typedef struct { size_t tree_id, next; double s; } vto_raypt;  /* include/ray.hpp:26-36 */
typedef struct { size_t cell_id; double s_enter, s_exit; } vto_seg; /* include/ray.hpp:14-19 */

typedef struct {
  vto_raypt *pts;
  size_t npts, cap_pts;
  vto_seg *segs;
  size_t nsegs, cap_segs;
  /* error detail */
  int err;
  char msg[256];
} vto_ws;

static int ws_push_pt(vto_ws *w, size_t tree_id, size_t next, double s) {
  if (w->npts == w->cap_pts) {
    size_t nc = w->cap_pts ? w->cap_pts * 2 : 1024;
    vto_raypt *np = (vto_raypt *)realloc(w->pts, nc * sizeof(vto_raypt));
    if (!np) return -1;
    w->pts = np;
    w->cap_pts = nc;
  }
  w->pts[w->npts].tree_id = tree_id;
  w->pts[w->npts].next = next;
  w->pts[w->npts].s = s;
  w->npts++;
  return 0;
}

static int ws_push_seg(vto_ws *w, size_t cell, double a, double b) {
  if (w->nsegs == w->cap_segs) {
    size_t nc = w->cap_segs ? w->cap_segs * 2 : 1024;
    vto_seg *ns = (vto_seg *)realloc(w->segs, nc * sizeof(vto_seg));
    if (!ns) return -1;
    w->segs = ns;
    w->cap_segs = nc;
  }
  w->segs[w->nsegs].cell_id = cell;
  w->segs[w->nsegs].s_enter = a;
  w->segs[w->nsegs].s_exit = b;
  w->nsegs++;
  return 0;
}

typedef struct {
  double start[3], end[3], dir[3];
  double len;
} vto_ray;

/* src/ray.cpp:14-35 */
static void ray_init(vto_ray *r, const double *a, const double *b) {
  for (int j = 0; j < 3; ++j) {
    r->start[j] = a[j];
    r->end[j] = b[j];
    r->dir[j] = b[j] - a[j];
  }
  double s = sqrt(r->dir[0] * r->dir[0] + r->dir[1] * r->dir[1] + r->dir[2] * r->dir[2]);
  r->dir[0] /= s;
  r->dir[1] /= s;
  r->dir[2] /= s;
  r->len = s;
}

/* src/ray.cpp:38-60 */
double vto_split_point_distance(const double *start, const double *dir, const double *p1,
                                const double *p2) {
  double ppl[3], norm[3];
  norm[0] = p2[0] - p1[0];
  norm[1] = p2[1] - p1[1];
  norm[2] = p2[2] - p1[2];
  ppl[0] = 0.5 * (p1[0] + p2[0]) - start[0];
  ppl[1] = 0.5 * (p1[1] + p2[1]) - start[1];
  ppl[2] = 0.5 * (p1[2] + p2[2]) - start[2];
  double ndp = norm[0] * ppl[0] + norm[1] * ppl[1] + norm[2] * ppl[2];
  double ndd = norm[0] * dir[0] + norm[1] * dir[1] + norm[2] * dir[2];
  if (fabs(ndd) < VTO_PARALLEL_BISECTOR_TOL) return DBL_MAX;
  return ndp / ndd;
}

/* src/ray.cpp:64-127 (non-periodic) */
static double split_full(const vto_tree *t, const vto_ray *r, size_t id1, size_t id2, double s_lo,
                         double s_hi, vto_ws *w) {
  const double *p1 = t->pts + id1 * 3, *p2 = t->pts + id2 * 3;
  double s = vto_split_point_distance(r->start, r->dir, p1, p2);
  if (s < DBL_MAX * 0.5 && s >= s_lo - VTO_TOLERANCE && s <= s_hi + VTO_TOLERANCE) return s;
  double lo = s_lo, hi = s_hi;
  for (int it = 0; it < 64; ++it) {
    double mid_s = 0.5 * (lo + hi);
    double mid_pt[3];
    for (int j = 0; j < 3; ++j) mid_pt[j] = r->start[j] + mid_s * r->dir[j];
    size_t mc = query1(t, mid_pt);
    if (mc != id1 && mc != id2) return mid_s;
    if (mc == id1) lo = mid_s;
    else hi = mid_s;
    if (hi - lo < 1e-12) return 0.5 * (lo + hi);
  }
  w->err = VTO_ERR_BINSEARCH;
  snprintf(w->msg, sizeof(w->msg),
           "Binary search did not converge for split point between cells %zu and %zu", id1, id2);
  return NAN;
}

/* src/ray.cpp:129-185 */
static size_t perp_perturb(const vto_tree *t, const vto_ray *r, const double *pos, size_t ex1,
                           size_t ex2, vto_ws *w) {
  const double INV_SQRT2 = 1.0 / sqrt(2.0);
  const double wv[3][3] = {{INV_SQRT2, INV_SQRT2, 0.0}, {0.0, INV_SQRT2, INV_SQRT2},
                           {INV_SQRT2, 0.0, INV_SQRT2}};
  int cycle = 0;
  for (int bound = 1; cycle < VTO_MAX_PERTURBATION_CYCLES; bound++) {
    for (int a = -bound; a <= bound && cycle < VTO_MAX_PERTURBATION_CYCLES; a++) {
      for (int b = -bound; b <= bound && cycle < VTO_MAX_PERTURBATION_CYCLES; b++) {
        for (int c = -bound; c <= bound && cycle < VTO_MAX_PERTURBATION_CYCLES; c++) {
          if (a == 0 && b == 0 && c == 0) continue;
          if (abs(a) < bound && abs(b) < bound && abs(c) < bound) continue;
          double pdir[3];
          for (int j = 0; j < 3; j++) pdir[j] = a * wv[0][j] + b * wv[1][j] + c * wv[2][j];
          double cd[3];
          cd[0] = r->dir[1] * pdir[2] - r->dir[2] * pdir[1];
          cd[1] = r->dir[2] * pdir[0] - r->dir[0] * pdir[2];
          cd[2] = r->dir[0] * pdir[1] - r->dir[1] * pdir[0];
          double mag = sqrt(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
          if (mag < 1e-15) { cycle++; continue; }
          for (int j = 0; j < 3; j++) cd[j] /= mag;
          double pert[3];
          for (int j = 0; j < 3; j++) pert[j] = pos[j] + VTO_PERTURBATION_EPS * cd[j];
          size_t cell = query1(t, pert);
          if (cell != ex1 && cell != ex2) return cell;
          cycle++;
        }
      }
    }
  }
  w->err = VTO_ERR_PERTURB;
  snprintf(w->msg, sizeof(w->msg),
           "Perturbation did not resolve degenerate split point after %d cycles",
           VTO_MAX_PERTURBATION_CYCLES);
  return VTO_NONE;
}

/* src/ray.cpp:374-384: along-ray perturbation, unambiguous result or NONE */
static size_t try_along_ray(const vto_tree *t, const vto_ray *r, const double *pos, double sign,
                            size_t c, size_t n) {
  double pert[3];
  for (int j = 0; j < 3; j++) pert[j] = pos[j] + sign * VTO_PERTURBATION_EPS * r->dir[j];
  size_t p_ids[2];
  double p_r2[2];
  vto_knn(t, pert, 2, p_ids, p_r2);
  if (p_r2[0] + VTO_TOLERANCE < p_r2[1] && p_ids[0] != c && p_ids[0] != n) return p_ids[0];
  return VTO_NONE;
}

/* src/ray.cpp:187-430 (non-periodic).  Returns 0 or an error code; the
 * segments are in w->segs. */
static int ray_walk(const vto_tree *t, const vto_ray *r, vto_ws *w) {
  size_t current, next, ctree_id, ntree_id;
  double s, pos[3];
  w->nsegs = 0;
  w->npts = 0;
  w->err = 0;
  if (ws_push_pt(w, VTO_NONE, 1, 0.0) || ws_push_pt(w, VTO_NONE, VTO_NONE, r->len))
    return VTO_ERR_NOMEM;
  w->pts[0].tree_id = query1(t, r->start);
  w->pts[1].tree_id = query1(t, r->end);
  size_t open_cell = w->pts[0].tree_id;
  double entry_s = w->pts[0].s;
  if (w->pts[0].tree_id == w->pts[1].tree_id) {
    if (ws_push_seg(w, w->pts[0].tree_id, w->pts[0].s, w->pts[1].s)) return VTO_ERR_NOMEM;
    return 0;
  }
  current = 0;
  ctree_id = w->pts[current].tree_id;
  next = w->pts[current].next;
  ntree_id = w->pts[next].tree_id;
  size_t iteration = 0;
  int not_done = 1;
  while (not_done) {
    if (++iteration > VTO_MAX_ITERATIONS) {
      snprintf(w->msg, sizeof(w->msg), "Ray walk exceeded maximum iteration count");
      return w->err = VTO_ERR_MAX_ITER;
    }
    if (w->pts[next].s - w->pts[current].s < 1e-14) {
      current = next;
      ctree_id = w->pts[current].tree_id;
      open_cell = ctree_id;
      next = w->pts[current].next;
      if (next == VTO_NONE) not_done = 0;
      else ntree_id = w->pts[next].tree_id;
      continue;
    }
    s = split_full(t, r, ctree_id, ntree_id, w->pts[current].s, w->pts[next].s, w);
    if (w->err) return w->err;
    if (s < w->pts[current].s - VTO_TOLERANCE || s > w->pts[next].s + VTO_TOLERANCE) {
      snprintf(w->msg, sizeof(w->msg),
               "Split point outside segment bounds: s=%f not in (%f, %f) for cells %zu and %zu", s,
               w->pts[current].s, w->pts[next].s, ctree_id, ntree_id);
      return w->err = VTO_ERR_SPLIT_BOUNDS;
    }
    {
      /* std::clamp(s, lo, hi) == (s < lo) ? lo : (hi < s) ? hi : s */
      double lo = w->pts[current].s + 1e-15, hi = w->pts[next].s - 1e-15;
      s = (s < lo) ? lo : (hi < s) ? hi : s;
    }
    for (int j = 0; j < 3; j++) pos[j] = r->start[j] + s * r->dir[j];

    size_t ids[3] = {VTO_NONE, VTO_NONE, VTO_NONE};
    double r2v[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
    vto_knn(t, pos, 3, ids, r2v);
    int has_c = 0, has_n = 0, three_eq = 1;
    for (int i = 0; i < 3; i++) {
      if (r2v[i] - r2v[0] >= VTO_TOLERANCE) { three_eq = 0; break; }
      if (ids[i] == ctree_id) has_c = 1;
      if (ids[i] == ntree_id) has_n = 1;
    }
    if (three_eq && !has_c && !has_n) {
      size_t k_big = VTO_K_EXPAND < t->n ? VTO_K_EXPAND : t->n;
      size_t ids_big[VTO_K_EXPAND];
      double r2_big[VTO_K_EXPAND];
      vto_knn(t, pos, k_big, ids_big, r2_big);
      for (size_t i = 0; i < k_big; i++) {
        if (r2_big[i] - r2_big[0] >= VTO_TOLERANCE) break;
        if (ids_big[i] == ctree_id) has_c = 1;
        if (ids_big[i] == ntree_id) has_n = 1;
        if (i == k_big - 1 && !has_c && !has_n) {
          snprintf(w->msg, sizeof(w->msg),
                   "Could not resolve split point classification after expanding to %d-NN. This "
                   "should be very unlikely; consider increasing TOLERANCE or K_EXPAND.",
                   VTO_K_EXPAND);
          return w->err = VTO_ERR_KNN_EXPAND;
        }
      }
    }
    if (has_c || has_n) {
      if (ws_push_seg(w, open_cell, entry_s, s)) return VTO_ERR_NOMEM;
      open_cell = ntree_id;
      entry_s = s;
      current = w->pts[current].next;
      ctree_id = w->pts[current].tree_id;
      next = w->pts[current].next;
      if (next == VTO_NONE) not_done = 0;
      else ntree_id = w->pts[next].tree_id;
    } else {
      if (r2v[0] + VTO_TOLERANCE < r2v[1]) {
        if (ws_push_pt(w, ids[0], next, s)) return VTO_ERR_NOMEM;
        next = w->npts - 1;
        w->pts[current].next = next;
        ntree_id = ids[0];
      } else {
        size_t sc = try_along_ray(t, r, pos, -1.0, ctree_id, ntree_id);
        if (sc == VTO_NONE) {
          double pc[3];
          for (int j = 0; j < 3; j++) pc[j] = pos[j] - VTO_PERTURBATION_EPS * r->dir[j];
          sc = perp_perturb(t, r, pc, ctree_id, ntree_id, w);
          if (w->err) return w->err;
        }
        size_t sn = try_along_ray(t, r, pos, 1.0, ctree_id, ntree_id);
        if (sn == VTO_NONE) {
          double pn[3];
          for (int j = 0; j < 3; j++) pn[j] = pos[j] + VTO_PERTURBATION_EPS * r->dir[j];
          sn = perp_perturb(t, r, pn, ctree_id, ntree_id, w);
          if (w->err) return w->err;
        }
        if (sc == sn) {
          if (ws_push_pt(w, sc, next, s)) return VTO_ERR_NOMEM;
          next = w->npts - 1;
          w->pts[current].next = next;
          ntree_id = sc;
        } else {
          size_t sn_idx = w->npts;
          if (ws_push_pt(w, sn, next, s)) return VTO_ERR_NOMEM;
          size_t sc_idx = w->npts;
          if (ws_push_pt(w, sc, sn_idx, s)) return VTO_ERR_NOMEM;
          w->pts[current].next = sc_idx;
          next = sc_idx;
          ntree_id = sc;
        }
      }
    }
  }
  if (ws_push_seg(w, open_cell, entry_s, w->pts[current].s)) return VTO_ERR_NOMEM;
  return 0;
}

/* src/reduction.cpp:8-83; out has nout = (mode==VOLUME ? 3 : nf) values */
static void reduce(const vto_ws *w, const double *fields, size_t nf, int mode, double *out) {
  if (mode == VTO_SUM) {
    for (size_t f = 0; f < nf; f++) out[f] = 0.0;
    for (size_t i = 0; i < w->nsegs; i++) {
      double ds = w->segs[i].s_exit - w->segs[i].s_enter;
      for (size_t f = 0; f < nf; f++) out[f] += ds * fields[w->segs[i].cell_id * nf + f];
    }
  } else if (mode == VTO_MAX) {
    for (size_t f = 0; f < nf; f++) out[f] = -INFINITY;
    for (size_t i = 0; i < w->nsegs; i++)
      for (size_t f = 0; f < nf; f++) {
        double v = fields[w->segs[i].cell_id * nf + f];
        if (v > out[f]) out[f] = v;
      }
  } else if (mode == VTO_MIN) {
    for (size_t f = 0; f < nf; f++) out[f] = INFINITY;
    for (size_t i = 0; i < w->nsegs; i++)
      for (size_t f = 0; f < nf; f++) {
        double v = fields[w->segs[i].cell_id * nf + f];
        if (v < out[f]) out[f] = v;
      }
  } else {
    double T = 1.0;
    double color[3] = {0.0, 0.0, 0.0};
    for (size_t i = 0; i < w->nsegs; i++) {
      size_t c = w->segs[i].cell_id;
      double alpha = fields[c * nf + 3];
      double ds = w->segs[i].s_exit - w->segs[i].s_enter;
      double opacity = 1.0 - exp(-alpha * ds);
      for (size_t k = 0; k < 3; k++) color[k] += T * fields[c * nf + k] * opacity;
      T *= (1.0 - opacity);
    }
    for (int k = 0; k < 3; k++) out[k] = color[k];
  }
}

/* counters of the last vto_project call: queries, nodes, leaves, points */
void vto_last_counters(unsigned long long *out) {
  for (int j = 0; j < 4; ++j) out[j] = g_cnt[j];
}

/*
 * Project nrays rays (src/projection.cpp:26-144).
 *   out:        nrays * nout values (nout = 3 for VOLUME, else nf)
 *   seg_counts: optional, nrays entries (segments per ray)
 *   offsets:    optional, nrays+1 CSR offsets; when given together with
 *               cell_ids/s_enter/s_exit, segments are written there.
 *   nthreads:   OpenMP threads (<=0: runtime default)
 * Returns 0, or the error code of the lowest-index failing ray, whose index
 * and message are stored in *err_ray / errmsg.
 */
int vto_project(const vto_tree *t, const double *fields, size_t nf, int valid_rgba,
                const double *starts, const double *ends, size_t nrays, int mode, double *out,
                int64_t *seg_counts, const int64_t *offsets, int64_t *cell_ids, double *s_enter,
                double *s_exit, int nthreads, int64_t *err_ray, char *errmsg, size_t errlen) {
  if (mode == VTO_VOLUME) {
    if (nf != 4) {
      if (errmsg) snprintf(errmsg, errlen,
                           "VolumeRender requires exactly 4 fields (R, G, B, alpha), got %zu", nf);
      return VTO_ERR_INVALID;
    }
    if (!valid_rgba) {
      if (errmsg) snprintf(errmsg, errlen,
                           "Volume rendering requires R, G, B values in [0, 1] and alpha >= 0");
      return VTO_ERR_INVALID;
    }
  }
  size_t nout = mode == VTO_VOLUME ? 3 : nf;
  int64_t first_bad = -1;
  int first_code = 0;
  char first_msg[256] = {0};
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
  nthreads = 1;
#endif
  for (int j = 0; j < 4; ++j) g_cnt[j] = 0;
#pragma omp parallel num_threads(nthreads)
  {
    vto_ws w;
    memset(&w, 0, sizeof(w));
    for (int j = 0; j < 4; ++j) tl_cnt[j] = 0;
#pragma omp for schedule(dynamic, 256)
    for (long long i = 0; i < (long long)nrays; ++i) {
      vto_ray r;
      ray_init(&r, starts + 3 * i, ends + 3 * i);
      int rc = ray_walk(t, &r, &w);
      if (rc) {
#pragma omp critical
        {
          if (first_bad < 0 || i < first_bad) {
            first_bad = i;
            first_code = rc;
            memcpy(first_msg, w.msg, sizeof(first_msg));
          }
        }
        continue;
      }
      reduce(&w, fields, nf, mode, out + i * nout);
      if (seg_counts) seg_counts[i] = (int64_t)w.nsegs;
      if (offsets && cell_ids) {
        int64_t o = offsets[i];
        for (size_t j = 0; j < w.nsegs; ++j) {
          cell_ids[o + j] = (int64_t)w.segs[j].cell_id;
          s_enter[o + j] = w.segs[j].s_enter;
          s_exit[o + j] = w.segs[j].s_exit;
        }
      }
    }
    free(w.pts);
    free(w.segs);
    for (int j = 0; j < 4; ++j) {
#pragma omp atomic
      g_cnt[j] += tl_cnt[j];
    }
  }
  if (first_bad >= 0) {
    if (err_ray) *err_ray = first_bad;
    if (errmsg) snprintf(errmsg, errlen, "%s", first_msg);
    return first_code;
  }
  return 0;
}
