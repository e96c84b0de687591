// project.cu -- host side of the walk launches, fused reductions, segment
// output, adjoint.
//
// Replaces Projection::makeProjection / makeDetailedProjection
// (src/projection.cpp:26-144), Ray::integrate (src/ray.cpp:432-442) and the
// reductions (src/reduction.cpp:8-96).  The walk kernels themselves
// (k_plain, k_batched, k_warp, k_slow) live in walk_kernels.cuh and are
// instantiated by walk_*.cu; this file holds
//   k_diag    re-walks the first failing ray alone to recover the numbers of
//             the reference's error message;
//   the ray sort, the walk sequence (counters, kernels, handed-over rays,
//   failure reporting), CUDA graphs of a walk, the tape scatter kernels,
//   Slice / BruteProjection sampling, the k-NN test hook and the
//   projection without allocation.
// Output kinds: image (reduction per ray), count (image + segments per
// ray), fill (CSR segments), tape, adjoint (scatter-add of field gradients).
#include <cub/cub.cuh>

#include <chrono>
#include <cstdio>
#include <memory>
#include <type_traits>

#include "internal.h"
#include "walk_kernels.cuh"

namespace vt {

// ------------------------------------------------------------- k_diag
__global__ void k_diag(DevCloud c, WalkIO io, int64_t ray) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  GlobalStack st;
  st.id = io.gstack_id;
  st.s = io.gstack_s;
  st.cap = io.gstack_cap;
  RayGeom g;
  ray_init(g, io.starts + 3 * ray, io.ends + 3 * ray);
  io.diag->code = 0;
  if (!ray_finite(g)) {
    io.diag->code = kErrNonFinite;
    return;
  }
  Search64T<true, true> S(c);  // serves periodic and non-periodic clouds
  NullSink ns;
  int rc = walk_ray(c, g, io.max_iter, S, st, ns, io.diag);
  if (rc == kNeedSlow) rc = kErrStack;
  io.diag->code = rc;
  if (rc) {
    io.diag->c = io.diag->c >= 0 ? c.perm[io.diag->c] : -1;
    io.diag->n = io.diag->n >= 0 ? c.perm[io.diag->n] : -1;
  }
}

// -------------------------------------------------------------- k_knn
// PointCloud::queryTree(q, k).  TT = false: the device tree, searched for
// k + 1 neighbours so that an exact tie inside the list or across its end
// is seen (then *tie is set and the host repeats the queries with TT = true,
// on the reference-order tree, which lists tied points in the reference's
// order).
template <bool TT>
__global__ void k_knn(DevCloud c, const double* __restrict__ q, int64_t nq, int k, int64_t* ids,
                      double* r2, unsigned* tie) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nq) return;
  KnnBig<129> r;
  r.clear(TT ? k : (int)min((int64_t)k + 1, c.n));
  unsigned v = 0;
  knn_query64<129, true, KnnBig<129>, TT>(c, q[3 * i], q[3 * i + 1], q[3 * i + 2], r, v);
  if (!TT) {
    bool t = false;
    for (int j = 0; j + 1 < r.cnt && j < k; ++j) t = t || r.r2[j] == r.r2[j + 1];
    if (t) atomicOr(tie, 1u);
  }
  for (int j = 0; j < k; ++j) {
    const bool ok = j < r.cnt;
    ids[i * k + j] = ok ? (int64_t)c.perm[r.id[j]] : -1;
    r2[i * k + j] = ok ? r.r2[j] : DBL_MAX;
  }
}

}  // namespace vt

namespace vt {

static std::string fmt_double(double v) {
  // std::to_string(double) formatting ("%f"), as in the reference's message
  char buf[64];
  snprintf(buf, sizeof(buf), "%f", v);
  return buf;
}

// The walk kernels of one output kind and reduction (walk_*.cu).
static int launch_kind(vt_cloud* cl, WalkIO& io, int out_kind, int mode, int kernel,
                       cudaStream_t st) {
  switch (out_kind) {
    case kOutImage:
      return mode == kSum ? launch_image_sum(cl, io, kernel, st)
                          : launch_image_vmm(cl, io, mode, kernel, st);
    case kOutCount:
      return mode == kSum ? launch_count_sum(cl, io, kernel, st)
                          : launch_count_vmm(cl, io, mode, kernel, st);
    case kOutFill: return launch_fill(cl, io, kernel, st);
    case kOutTape:
      if (mode != kSum && mode != kVolume)
        return set_error(VT_ERR_INVALID, "a tape is recorded for 'integrate' and 'volume' only");
      return launch_tape(cl, io, mode, kernel, st);
    default:
      if (mode != kSum && mode != kVolume)
        return set_error(VT_ERR_INVALID, "adjoint is defined for 'integrate' and 'volume' only");
      return launch_adj(cl, io, mode, kernel, st);
  }
}

// Enqueue one walk on `st`: counters reset, then the kernels.  No host
// synchronisation, so the sequence can be captured into a CUDA graph.
static int enqueue_walk(vt_cloud* cl, WalkIO& io, int out_kind, int mode, int kernel,
                        cudaStream_t st) {
  // periodic clouds: the periodic k-NN merge and minimum-image split points
  // live in the exact FP64 walk of the one-ray-per-thread kernel
  if (cl->periodic) {
    kernel = VT_KERNEL_PLAIN_FP64;
    io.order = nullptr;
  }
  io.max_iter = cl->max_iter;
  io.local_cap = cl->local_stack;
  io.cache_mode = cl->cache_mode;
  io.diag = nullptr;
  VT_CUDA(cudaMemsetAsync(io.stats, 0, sizeof(DevStats), st));
  VT_CUDA(cudaMemsetAsync(&io.stats->first_error, 0xff, sizeof(unsigned long long), st));
  return launch_kind(cl, io, out_kind, mode, kernel, st);
}

static int finish_walk(vt_cloud* cl, WalkIO& io, const DevStats& hs, float ms, cudaStream_t st,
                       vt_stats* stats, WalkDiag* d_diag);

// One walk launch (+ handed-over rays) on scratch already placed in `io`
// (stats, hand-over queue, global stacks); turns a per-ray failure into the
// reference's error message.  `d_diag`: device scratch for the diagnosis of
// a failing ray (NULL: allocated on demand).  `timed`: CUDA events around
// the launches for vt_stats.walk_ms.
// Rays deferred by k_slow for the reference-order tree (an exact tie at the
// nearest distance of a 1-NN query, tietree.cu): build the tree if it is not
// there (unless the caller cannot allocate: then an error naming
// vt_cloud_build_tie_tree), run k_slow over the deferred rays and re-read
// the counters into `hs`.
static int complete_deferred(vt_cloud* cl, WalkIO& io, int out_kind, int mode, cudaStream_t st,
                             bool may_alloc, DevStats& hs) {
  if (hs.tie_deferred == 0) return VT_OK;
  if (!cl->view.tt_nodes) {
    if (!may_alloc)
      return set_error(VT_ERR_RUNTIME,
                       "an exact distance tie needs the reference-order tree, which this call "
                       "does not allocate: build it first with vt_cloud_build_tie_tree");
    const int rc = build_tie_tree(cl, st);
    if (rc) return rc;
  }
  io.deferred = 1;
  const int rc = launch_kind(cl, io, out_kind, mode, VT_KERNEL_AUTO, st);
  io.deferred = 0;
  if (rc) return rc;
  VT_CUDA(cudaMemcpyAsync(&hs, io.stats, sizeof(DevStats), cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  return VT_OK;
}

static int run_walk_on(vt_cloud* cl, WalkIO& io, int out_kind, int mode, int kernel,
                       cudaStream_t st, vt_stats* stats, WalkDiag* d_diag, bool timed,
                       bool may_alloc = true) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (timed) {
    VT_CUDA(cudaEventCreate(&e0));
    VT_CUDA(cudaEventCreate(&e1));
    VT_CUDA(cudaEventRecord(e0, st));
  }
  const int rc = enqueue_walk(cl, io, out_kind, mode, kernel, st);
  if (rc) {
    if (timed) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    }
    return rc;
  }
  if (timed) VT_CUDA(cudaEventRecord(e1, st));
  DevStats hs;
  VT_CUDA(cudaMemcpyAsync(&hs, io.stats, sizeof(DevStats), cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f;
  if (timed) {
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  const int rc2 = complete_deferred(cl, io, out_kind, mode, st, may_alloc, hs);
  if (rc2) return rc2;
  return finish_walk(cl, io, hs, ms, st, stats, d_diag);
}

// Counters of a finished walk into `stats`; the reference's message when a
// ray failed (the first failing ray is re-walked alone by k_diag).
static int finish_walk(vt_cloud* cl, WalkIO& io, const DevStats& hs, float ms, cudaStream_t st,
                       vt_stats* stats, WalkDiag* d_diag) {
  if (hs.rays > 0) cl->cross_per_ray = (double)hs.crossings / (double)hs.rays;
  if (stats) {
    stats->rays = hs.rays;
    stats->crossings = hs.crossings;
    stats->queries = hs.queries;
    stats->fp64_resolves = hs.fp64_resolves;
    stats->slow_rays = hs.slow_rays;
    stats->max_stack = hs.max_stack;
    stats->walk_ms = ms;
    stats->search_steps = hs.search_steps;
    stats->fp64_checks = hs.fp64_checks;
    stats->cache_refreshes = hs.cache_refreshes;
    stats->cache_hits = hs.cache_hits;
    stats->ties = hs.ties;
    stats->fp32_queries = hs.fp32_queries;
    stats->fp64_check_queries = hs.recheck_queries;
    for (int i = 0; i < 3; ++i) stats->trip_cycles[i] = hs.trip_cycles[i];
    stats->search_warp_steps = hs.search_warp_steps;
    stats->search_lane_steps = hs.search_lane_steps;
  }
  if (hs.first_error != ~0ULL) {
    const int64_t ray = (int64_t)(hs.first_error >> 8);
    const int code = (int)(hs.first_error & 0xff);
    // re-walk the failing ray alone for the message details
    DevBuf<WalkDiag> dg;
    if (!d_diag) {
      if (dg.alloc(1)) return VT_ERR_NOMEM;
      d_diag = dg.p;
    }
    WalkDiag hd{0, -1, -1, 0.0, 0.0, 0.0};
    VT_CUDA(cudaMemcpyAsync(d_diag, &hd, sizeof(hd), cudaMemcpyHostToDevice, st));
    io.diag = d_diag;
    k_diag<<<1, 1, 0, st>>>(cl->view, io, ray);
    VT_CUDA(cudaGetLastError());
    VT_CUDA(cudaMemcpyAsync(&hd, d_diag, sizeof(hd), cudaMemcpyDeviceToHost, st));
    VT_CUDA(cudaStreamSynchronize(st));
    io.diag = nullptr;
    std::string msg;
    switch (code) {
      case kErrMaxIter: msg = "Ray walk exceeded maximum iteration count"; break;
      case kErrSplitBounds:
        msg = "Split point outside segment bounds: s=" + fmt_double(hd.s) + " not in (" +
              fmt_double(hd.s_lo) + ", " + fmt_double(hd.s_hi) + ") for cells " +
              std::to_string(hd.c) + " and " + std::to_string(hd.n);
        break;
      case kErrBinSearch:
        msg = "Binary search did not converge for split point between cells " +
              std::to_string(hd.c) + " and " + std::to_string(hd.n);
        break;
      case kErrPerturb:
        msg = "Perturbation did not resolve degenerate split point after " +
              std::to_string(kMaxPerturbCycles) + " cycles";
        break;
      case kErrKnnExpand:
        msg = "Could not resolve split point classification after expanding to " +
              std::to_string(kExpandK) +
              "-NN. This should be very unlikely; consider increasing TOLERANCE or K_EXPAND.";
        break;
      case kErrStack:
        msg = "Ray walk exceeded the pending-point stack capacity (" +
              std::to_string(io.gstack_cap) + ")";
        break;
      case kErrNonFinite:
        return set_error(VT_ERR_INVALID,
                         "Ray endpoints must be finite (ray " + std::to_string(ray) + ")");
      case kErrNonFiniteDist:
        return set_error(VT_ERR_INVALID, "Squared distances overflow for ray " +
                                             std::to_string(ray) + ": coordinates too large");
      case kErrPeriodicBisect:
        msg = "Could not find intermediate cell by bisection along periodic ray";
        break;
      case kErrTie:
        msg = "an exact distance tie could not be resolved in the reference's order";
        break;
      default: msg = "ray walk failed with code " + std::to_string(code); break;
    }
    return set_error(code, msg);
  }
  return VT_OK;
}

// ------------------------------------------------------- ray ordering
// The batched kernels walk the rays in a coherent order: sorted by a 64-bit
// key of the quantized direction (5 bits per component, bits 48-62) and the
// Morton code of the ray's midpoint in the cloud's box (16 bits per axis,
// bits 0-47).  Parallel rays of a projection grid then run as compact 2D
// tiles, so the 32 rays of a warp cross the same cells.  Non-finite rays
// sort last.  Results are written at each ray's own index.
__device__ __forceinline__ unsigned long long spread3(unsigned v) {
  unsigned long long x = v & 0xffffu;
  x = (x | (x << 16)) & 0x0000ff0000ffULL;
  x = (x | (x << 8)) & 0x00f00f00f00fULL;
  x = (x | (x << 4)) & 0x0c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x249249249249ULL;
  return x;
}

__global__ void k_ray_keys(const double* __restrict__ S, const double* __restrict__ E,
                           int64_t n, DevCloud c, unsigned long long* keys, int32_t* idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s[3], e[3], d[3];
  bool ok = true;
  double len2 = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    s[j] = S[3 * i + j];
    e[j] = E[3 * i + j];
    d[j] = e[j] - s[j];
    len2 += d[j] * d[j];
    ok = ok && isfinite(s[j]) && isfinite(e[j]);
  }
  unsigned long long key = ~0ULL;
  if (ok) {
    const double inv = len2 > 0.0 ? 1.0 / sqrt(len2) : 0.0;
    unsigned long long dq = 0, mc = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double u = (d[j] * inv + 1.0) * 15.5;
      dq = (dq << 5) | (unsigned long long)(u < 0.0 ? 0 : (u > 31.0 ? 31 : (int)u));
      const double ext = c.bbhi[j] - c.bblo[j];
      double m = ext > 0.0 ? ((0.5 * (s[j] + e[j]) - c.bblo[j]) / ext) * 65535.0 : 0.0;
      m = m < 0.0 ? 0.0 : (m > 65535.0 ? 65535.0 : m);
      mc |= spread3((unsigned)m) << j;
    }
    key = (dq << 48) | mc;
  }
  keys[i] = key;
  idx[i] = (int32_t)i;
}

// ------------------------------------------------ longest batches first
// A warp walks 32 consecutive rays of the coherent order and takes the next
// 32 only when all of them are done, so a launch ends when the warp that
// drew the most expensive late batch ends.  Rays through dense regions cross
// several times more cells than rays through the outskirts, and the coherent
// order interleaves them, so with a few batches per warp (a 512x512 image:
// 2.8 per resident warp) the last quarter of the launch runs a fraction of
// the warps.  The batches are therefore handed out longest first (LPT
// scheduling): each ray's cost is estimated by the number of device-tree
// leaves whose tight box its segment crosses (an FP32 slab test per node,
// a small fraction of the walk's own node visits), a batch costs its most
// expensive ray, and the batches are sorted by decreasing cost class.  The
// order only changes when each ray is walked, never what is computed.
constexpr int kBatch = 32;

__global__ void k_ray_cost(const double* __restrict__ S, const double* __restrict__ E,
                           const int32_t* __restrict__ order, int64_t n, DevCloud c,
                           uint32_t* __restrict__ cost) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t r = order[i];
  float p0[3], inv[3];
  bool ok = true;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const double a = S[3 * r + j] - c.origin[j], b = E[3 * r + j] - c.origin[j];
    ok = ok && isfinite(a) && isfinite(b);
    p0[j] = (float)a;
    const float d = (float)(b - a);
    inv[j] = d != 0.f ? 1.f / d : 1e30f;
  }
  uint32_t count = 0;
  if (ok) {
    const int64_t ninternal = c.nleaves - 1;
    int64_t stack[kMaxDepth + 2];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const int64_t node = stack[--sp];
      const float4 lo = __ldg(&c.boxlo[node]), hi = __ldg(&c.boxhi[node]);
      // segment p0 + t (p1 - p0), t in [0, 1], against the box (slabs)
      float t0 = 0.f, t1 = 1.f;
      const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        float ta = (l[j] - p0[j]) * inv[j], tb = (h[j] - p0[j]) * inv[j];
        if (ta > tb) {
          const float t = ta;
          ta = tb;
          tb = t;
        }
        t0 = fmaxf(t0, ta);
        t1 = fminf(t1, tb);
      }
      if (!(t0 <= t1)) continue;
      if (node >= ninternal) {
        ++count;
      } else if (sp + 2 <= kMaxDepth + 2) {
        stack[sp++] = 2 * node + 2;
        stack[sp++] = 2 * node + 1;
      }
    }
  }
  cost[i] = count;
}

// Cost classes per doubling of the estimated cost: batches are sorted by
// class (the radix sort is stable, so each class keeps the coherent order:
// the warps running at the same time still share their region of the tree)
#ifndef VT_LPT_CLASSES_PER_DOUBLING
#define VT_LPT_CLASSES_PER_DOUBLING 1
#endif
// the reordering pays while each SM gets few batches; with many (large
// images) the tail is short and the coherent order's cache sharing between
// concurrent warps is worth more (measured on B200 with 20 resident warps
// per SM: +20% at 56 batches per SM, -1% at 221, -2% at 885; the threshold
// is kept in batches per SM)
constexpr int kLptMaxBatchesPerSm = 160;

// key of batch b (ascending sort = decreasing cost class); the partial last
// batch sorts last, so every other batch stays aligned to 32 queue slots
__global__ void k_batch_keys(const uint32_t* __restrict__ cost, int64_t n, int64_t nb,
                             uint32_t* __restrict__ keys, int32_t* __restrict__ idx) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int64_t a = b * kBatch, e = a + kBatch < n ? a + kBatch : n;
  uint32_t m = 0;
  for (int64_t i = a; i < e; ++i) m = max(m, cost[i]);
  const uint32_t cls = (uint32_t)(VT_LPT_CLASSES_PER_DOUBLING * log2f(1.0f + (float)m));
  keys[b] = e - a < kBatch ? 0xffffffffu : ~min(cls, 0xfffffffeu);
  idx[b] = (int32_t)b;
}

__global__ void k_permute_batches(const int32_t* __restrict__ order,
                                  const int32_t* __restrict__ bsorted, int64_t n,
                                  int32_t* __restrict__ out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  out[k] = order[(int64_t)bsorted[k / kBatch] * kBatch + k % kBatch];
}

// Scratch of the ray sort for n rays: keys and indices (twice), the batch
// costs, keys and indices (twice) and CUB's temporary storage of both
// sorts; 0 when the rays keep their order (few or too many).
struct SortLayout {
  size_t kb, ib, nbb, cub_rays, cub_batches, total;
};

static size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

static int sort_rays_layout(int64_t n, SortLayout& L) {
  L = SortLayout{};
  if (n < 64 || n > (int64_t)0x7fffffff) return VT_OK;
  const int64_t nb = (n + kBatch - 1) / kBatch;
  VT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, L.cub_rays, (unsigned long long*)nullptr,
                                          (unsigned long long*)nullptr, (int32_t*)nullptr,
                                          (int32_t*)nullptr, (int)n, 0, 63));
  VT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, L.cub_batches, (uint32_t*)nullptr,
                                          (uint32_t*)nullptr, (int32_t*)nullptr,
                                          (int32_t*)nullptr, (int)nb, 0, 32));
  L.kb = up256((size_t)n * 8);
  L.ib = up256((size_t)n * 4);
  L.nbb = up256((size_t)nb * 4);
  // keys x2 | idx x2 | cost | batch keys x2 | batch idx x2 | cub (max of both)
  L.total = 2 * L.kb + 2 * L.ib + L.ib + 4 * L.nbb + std::max(L.cub_rays, L.cub_batches);
  return VT_OK;
}

static int sort_rays_bytes(int64_t n, size_t& total, size_t& cub_bytes) {
  SortLayout L;
  const int rc = sort_rays_layout(n, L);
  total = L.total;
  cub_bytes = L.cub_rays;
  return rc;
}

// Enqueue the ray sort into `base` (sort_rays_bytes of scratch) and point
// io.order at the result; no host synchronisation.
static int sort_rays_into(const DevCloud& view, WalkIO& io, uint8_t* base, size_t total,
                          size_t cub_bytes, cudaStream_t st) {
  const int64_t n = io.nrays;
  io.order = nullptr;
  if (total == 0) return VT_OK;
  SortLayout L;
  int rc = sort_rays_layout(n, L);
  if (rc) return rc;
  if (L.total > total) return set_error(VT_ERR_RUNTIME, "ray sort scratch too small");
  const int64_t nb = (n + kBatch - 1) / kBatch;
  auto* k0 = reinterpret_cast<unsigned long long*>(base);
  auto* k1 = reinterpret_cast<unsigned long long*>(base + L.kb);
  auto* i0 = reinterpret_cast<int32_t*>(base + 2 * L.kb);
  auto* i1 = reinterpret_cast<int32_t*>(base + 2 * L.kb + L.ib);
  auto* cost = reinterpret_cast<uint32_t*>(base + 2 * L.kb + 2 * L.ib);
  uint8_t* bb = base + 2 * L.kb + 3 * L.ib;
  auto* bk0 = reinterpret_cast<uint32_t*>(bb);
  auto* bk1 = reinterpret_cast<uint32_t*>(bb + L.nbb);
  auto* bi0 = reinterpret_cast<int32_t*>(bb + 2 * L.nbb);
  auto* bi1 = reinterpret_cast<int32_t*>(bb + 3 * L.nbb);
  void* tmp = bb + 4 * L.nbb;
  const int B = 256;
  k_ray_keys<<<(unsigned)((n + B - 1) / B), B, 0, st>>>(io.starts, io.ends, n, view, k0, i0);
  VT_CUDA(cudaGetLastError());
  size_t cb = L.cub_rays;
  VT_CUDA(cub::DeviceRadixSort::SortPairs(tmp, cb, k0, k1, i0, i1, (int)n, 0, 63, st));
  int dev = 0, nsms = 0;
  VT_CUDA(cudaGetDevice(&dev));
  VT_CUDA(cudaDeviceGetAttribute(&nsms, cudaDevAttrMultiProcessorCount, dev));
  if (nb >= (int64_t)kLptMaxBatchesPerSm * nsms) {
    io.order = i1;
    return VT_OK;
  }
  // longest batches first: i1 (coherent order) -> i0 (batches by cost)
  k_ray_cost<<<(unsigned)((n + B - 1) / B), B, 0, st>>>(io.starts, io.ends, i1, n, view, cost);
  VT_CUDA(cudaGetLastError());
  k_batch_keys<<<(unsigned)((nb + B - 1) / B), B, 0, st>>>(cost, n, nb, bk0, bi0);
  VT_CUDA(cudaGetLastError());
  cb = L.cub_batches;
  VT_CUDA(cub::DeviceRadixSort::SortPairs(tmp, cb, bk0, bk1, bi0, bi1, (int)nb, 0, 32, st));
  k_permute_batches<<<(unsigned)((n + B - 1) / B), B, 0, st>>>(i1, bi1, n, i0);
  VT_CUDA(cudaGetLastError());
  io.order = i0;
  (void)cub_bytes;
  return VT_OK;
}

// Fill io.order (workspace) with the coherent ray order.
static int sort_rays(vt_cloud* cl, WalkIO& io, cudaStream_t st) {
  size_t total = 0, cub_bytes = 0;
  int rc = sort_rays_bytes(io.nrays, total, cub_bytes);
  if (rc) return rc;
  if (total && (rc = cl->ws_order.reserve(total))) return rc;
  return sort_rays_into(cl->view, io, cl->ws_order.p, total, cub_bytes, st);
}

// Walk launch with the handle's (grow-only) workspace as scratch.
int run_walk(vt_cloud* cl, WalkIO& io, int out_kind, int mode, int kernel, cudaStream_t st,
             vt_stats* stats) {
  if (kernel != VT_KERNEL_PLAIN_FP64 && !cl->periodic) {
    const int rc = sort_rays(cl, io, st);
    if (rc) return rc;
  } else {
    io.order = nullptr;  // the plain kernel keeps the caller's order
  }
  const int slow_threads = 1024;
  if (cl->ws_stats.reserve(1)) return VT_ERR_NOMEM;
  if (cl->ws_slow.reserve(io.nrays > 0 ? io.nrays : 1)) return VT_ERR_NOMEM;
  if (cl->ws_stack_id.reserve((size_t)slow_threads * cl->stack_cap)) return VT_ERR_NOMEM;
  if (cl->ws_stack_s.reserve((size_t)slow_threads * cl->stack_cap)) return VT_ERR_NOMEM;
  io.stats = cl->ws_stats.p;
  io.slow_q = cl->ws_slow.p;
  io.gstack_id = cl->ws_stack_id.p;
  io.gstack_s = cl->ws_stack_s.p;
  io.gstack_cap = cl->stack_cap;
  io.slow_threads = slow_threads;
  return run_walk_on(cl, io, out_kind, mode, kernel, st, stats, nullptr, true);
}

int compiled_blocks_per_sm(int kernel, int64_t nrays) {
  switch (kernel) {
    case VT_KERNEL_THREAD_FP32: {
      int dev = 0, nsms = 0;
      if (cudaGetDevice(&dev) != cudaSuccess ||
          cudaDeviceGetAttribute(&nsms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return VT_BATCHED_MINB_FEW;
      return batched_minb(true, nrays, nsms);
    }
    case VT_KERNEL_BATCHED_FP64:
      return VT_BATCHED_MINB64;
    case VT_KERNEL_BATCHED:
      return VT_WARP_MINB;
    default:
      return 0;
  }
}

}  // namespace vt

// ------------------------------------------------------ CUDA graph of a walk
// A forward projection of fixed device buffers captured once (counter
// resets, ray sort, walk kernel, global-stack kernel) and replayed with one
// cudaGraphLaunch.  The graph owns its scratch; it reads the rays and writes
// the image through the pointers given at creation, so a caller refills the
// same buffers between launches.
struct vt_graph {
  vt_cloud* cl = nullptr;
  int device = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  vt::DevBuf<vt::DevStats> stats;
  vt::DevBuf<unsigned long long> slow;
  vt::DevBuf<int> stack_id;
  vt::DevBuf<double> stack_s;
  vt::DevBuf<uint8_t> order;
  vt::WalkIO io{};
  int mode = 0;
  const double4* pts = nullptr;  // the cloud's buffers at capture time
  const double* fields = nullptr;
  ~vt_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

extern "C" {

int vt_graph_create(vt_cloud* cl, const double* d_starts, const double* d_ends, uint64_t nrays,
                    int mode, int kernel, double* d_out, vt_graph** out) {
  using namespace vt;
  try {
    if (!out) return set_error(VT_ERR_INVALID, "out must not be NULL");
    *out = nullptr;
    int rc = check_projectable(cl, mode);
    if (rc) return rc;
    if (nrays == 0 || !d_starts || !d_ends || !d_out)
      return set_error(VT_ERR_INVALID, "a graph needs rays and device buffers");
    std::lock_guard<std::mutex> lk(cl->mu);
    VT_CUDA(cudaSetDevice(cl->device));
    std::unique_ptr<vt_graph> g(new vt_graph());
    g->cl = cl;
    g->device = cl->device;
    const int slow_threads = 1024;
    if ((rc = g->stats.alloc(1)) || (rc = g->slow.alloc(nrays)) ||
        (rc = g->stack_id.alloc((size_t)slow_threads * cl->stack_cap)) ||
        (rc = g->stack_s.alloc((size_t)slow_threads * cl->stack_cap)))
      return rc;
    g->mode = mode;
    WalkIO& io = g->io;
    io.starts = d_starts;
    io.ends = d_ends;
    io.nrays = (int64_t)nrays;
    io.nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
    io.out = d_out;
    io.stats = g->stats.p;
    io.slow_q = g->slow.p;
    io.gstack_id = g->stack_id.p;
    io.gstack_s = g->stack_s.p;
    io.gstack_cap = cl->stack_cap;
    io.slow_threads = slow_threads;
    const int k = resolve_kernel(cl, kernel, nrays);
    size_t total = 0, cub_bytes = 0;
    if (k != VT_KERNEL_PLAIN_FP64 && !cl->periodic) {
      if ((rc = sort_rays_bytes(io.nrays, total, cub_bytes))) return rc;
      if (total && (rc = g->order.alloc(total))) return rc;
    }
    cudaStream_t cs = nullptr;
    VT_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
      cudaStreamDestroy(cs);
      VT_CUDA(e);
    }
    rc = sort_rays_into(cl->view, io, g->order.p, total, cub_bytes, cs);
    if (!rc) rc = enqueue_walk(cl, io, kOutImage, mode, k, cs);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    if (rc || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (rc) return rc;
      VT_CUDA(e);
    }
    g->graph = graph;
    VT_CUDA(cudaGraphInstantiate(&g->exec, graph, 0));
    g->pts = cl->view.pts;
    g->fields = cl->view.fields;
    *out = g.release();
    return VT_OK;
  } catch (const std::bad_alloc&) {
    return set_error(VT_ERR_NOMEM, "host allocation failed");
  }
}

int vt_graph_launch(vt_graph* g, void* stream) {
  using namespace vt;
  if (!g) return set_error(VT_ERR_INVALID, "null graph handle");
  if (g->cl->view.pts != g->pts || g->cl->view.fields != g->fields)
    return set_error(VT_ERR_RUNTIME,
                     "the cloud's tree or fields were reallocated after the graph was created");
  VT_CUDA(cudaSetDevice(g->device));
  VT_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  return VT_OK;
}

int vt_graph_finish(vt_graph* g, void* stream, vt_stats* stats) {
  using namespace vt;
  if (!g) return set_error(VT_ERR_INVALID, "null graph handle");
  if (stats) memset(stats, 0, sizeof(*stats));
  std::lock_guard<std::mutex> lk(g->cl->mu);
  VT_CUDA(cudaSetDevice(g->device));
  cudaStream_t st = (cudaStream_t)stream;
  DevStats hs;
  VT_CUDA(cudaMemcpyAsync(&hs, g->io.stats, sizeof(DevStats), cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  // rays deferred for the reference-order tree finish here, outside the graph
  const int rc = complete_deferred(g->cl, g->io, kOutImage, g->mode, st, true, hs);
  if (rc) return rc;
  return finish_walk(g->cl, g->io, hs, 0.f, st, stats, nullptr);
}

void vt_graph_destroy(vt_graph* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  delete g;
}

}  // extern "C"

namespace vt {

// Block size of the tape scatters (one shared-memory slot per thread).
constexpr int kScatterBlock = 256;

// Sum of the terms v[] of the lanes in `peers` (ascending lane order, from
// 0.0) through the warp's slots of shared memory: each lane stores its term,
// the group's leader adds its peers' (a warp of shuffles per field cost
// twice the time: 6.37 against 3.10 ms for clustered_2m's 1.99e8 entries).
__device__ __forceinline__ double group_sum(double* s_warp, int lane, unsigned peers, bool leader,
                                            double v) {
  s_warp[lane] = v;
  __syncwarp();
  double sum = 0.0;
  if (leader)
    for (unsigned m = peers; m; m &= m - 1) sum += s_warp[__ffs(m) - 1];
  __syncwarp();
  return sum;
}

// Adjoint of 'integrate' from a tape: grad[pid, f] += gout[ray, f] * ds for
// every entry.  The lanes of a warp holding the same cell add their terms
// first (neighbouring rays cross the same cells), then one atomic per cell.
template <int NF>
__global__ void __launch_bounds__(kScatterBlock)
    k_tape_scatter(const TapeEntry* __restrict__ t, uint64_t n, int nf_rt,
                   const double* __restrict__ gout, double* __restrict__ grad) {
  __shared__ double s_v[kScatterBlock];
  const int lane = threadIdx.x & 31;
  double* s_warp = s_v + (threadIdx.x & ~31);
  const int nf = NF > 0 ? NF : nf_rt;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
    const uint64_t i = base + threadIdx.x;
    int pid = -1, ray = 0;
    double ds = 0.0;
    if (i < n) {
      const TapeEntry e = t[i];
      pid = e.pid;
      ray = e.ray;
      ds = e.ds;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, pid);
    const bool leader = __ffs(peers) - 1 == lane;
    for (int f = 0; f < nf; ++f) {
      const double v = pid >= 0 ? gout[(int64_t)ray * nf + f] * ds : 0.0;
      const double sum = group_sum(s_warp, lane, peers, leader, v);
      if (leader && pid >= 0) atomicAdd(&grad[(int64_t)pid * nf + f], sum);
    }
  }
}

// Adjoint of 'volume' from a tape (the formulas of AdjSink): with
// e = exp(-alpha ds), o = 1 - e, T and P of the entry and C the ray's final
// colour, grad[rgb_k] += g_k T o and grad[alpha] += ds sum_k g_k (T rgb_k e -
// (C_k - P_k)); lanes holding the same cell add their terms first.
__global__ void __launch_bounds__(kScatterBlock)
    k_tape_scatter_vol(DevCloud c, const TapeEntryV* __restrict__ t, uint64_t n,
                       const double* __restrict__ gout, const double* __restrict__ fwd,
                       double* __restrict__ grad) {
  __shared__ double s_v[kScatterBlock];
  const int lane = threadIdx.x & 31;
  double* s_warp = s_v + (threadIdx.x & ~31);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
    const uint64_t i = base + threadIdx.x;
    int pid = -1;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (i < n) {
      const TapeEntryV e = t[i];
      pid = c.perm[e.cell];
      const double* F = c.fields + (int64_t)e.cell * 4;
      const double ex = exp(dmul(-F[3], e.ds));
      const double o = dsub(1.0, ex);
      double galpha = 0.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double g = gout[(int64_t)e.ray * 3 + k];
        const double S = fwd[(int64_t)e.ray * 3 + k] - e.P[k];
        galpha += g * (e.T * F[k] * ex - S);
        v[k] = g * e.T * o;
      }
      v[3] = e.ds * galpha;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, pid);
    const bool leader = __ffs(peers) - 1 == lane;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const double sum = group_sum(s_warp, lane, peers, leader, v[f]);
      if (leader && pid >= 0) atomicAdd(&grad[(int64_t)pid * 4 + f], sum);
    }
  }
}

int run_tape_scatter_vol(vt_cloud* cl, const void* tape, uint64_t n, const double* d_gout,
                         const double* d_fwd, double* d_grad, cudaStream_t st) {
  if (n == 0) return VT_OK;
  int dev = 0, nsms = 0;
  VT_CUDA(cudaGetDevice(&dev));
  VT_CUDA(cudaDeviceGetAttribute(&nsms, cudaDevAttrMultiProcessorCount, dev));
  const int B = kScatterBlock;
  uint64_t blocks = (n + B - 1) / B;
  if (blocks > (uint64_t)nsms * 16) blocks = (uint64_t)nsms * 16;
  k_tape_scatter_vol<<<(unsigned)blocks, B, 0, st>>>(
      cl->view, static_cast<const TapeEntryV*>(tape), n, d_gout, d_fwd, d_grad);
  VT_CUDA(cudaGetLastError());
  return VT_OK;
}

int run_tape_scatter(vt_cloud* cl, const void* tape, uint64_t n, const double* d_gout,
                     double* d_grad, cudaStream_t st) {
  if (n == 0) return VT_OK;
  int dev = 0, nsms = 0;
  VT_CUDA(cudaGetDevice(&dev));
  VT_CUDA(cudaDeviceGetAttribute(&nsms, cudaDevAttrMultiProcessorCount, dev));
  const int B = kScatterBlock;
  uint64_t blocks = (n + B - 1) / B;
  if (blocks > (uint64_t)nsms * 16) blocks = (uint64_t)nsms * 16;
  const TapeEntry* t = static_cast<const TapeEntry*>(tape);
  const int nf = (int)cl->nfields;
  if (nf == 1) k_tape_scatter<1><<<(unsigned)blocks, B, 0, st>>>(t, n, nf, d_gout, d_grad);
  else if (nf == 3) k_tape_scatter<3><<<(unsigned)blocks, B, 0, st>>>(t, n, nf, d_gout, d_grad);
  else k_tape_scatter<0><<<(unsigned)blocks, B, 0, st>>>(t, n, nf, d_gout, d_grad);
  VT_CUDA(cudaGetLastError());
  return VT_OK;
}

// ------------------------------------------------- slice / brute projection
// Slice::makeSlice (src/slice.cpp:6-60): pixel (i, j) samples the field of
// the nearest cell at (x0 + dx i, y0 + dy j, depth); out[(i ny + j) nf + f].
__global__ void k_slice(DevCloud c, uint64_t nx, uint64_t ny, double x0, double y0, double dx,
                        double dy, double depth, double* __restrict__ out,
                        unsigned long long* __restrict__ bad) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * ny) return;
  const uint64_t i = t / ny, j = t % ny;
  const double qx = dadd(x0, dmul(dx, (double)i));
  const double qy = dadd(y0, dmul(dy, (double)j));
  unsigned v = 0;
  const int cell = nn1_exact64<true, true>(c, qx, qy, depth, v);
  if (cell == kTieUnresolved) {
    atomicOr(&bad[1], 1ULL);
    return;
  }
  if (cell < 0) {
    atomicMin(bad, (unsigned long long)t);
    return;
  }
  for (int f = 0; f < c.nf; f++) out[t * c.nf + f] = c.fields[(int64_t)cell * c.nf + f];
}

// BruteProjection::makeProjection (src/brute_projection.cpp:10-96): pixel
// (i, j) reduces the fields of the nearest cells of the samples
// (x0 + dx i, y0 + dy j, z0 + dz k), k = 0 .. nz-1 in order; Sum is scaled
// by dz at the end.
template <int MODE>
__global__ void k_brute(DevCloud c, uint64_t nx, uint64_t ny, uint64_t nz, double x0, double y0,
                        double z0, double dx, double dy, double dz, double* __restrict__ out,
                        unsigned long long* __restrict__ bad) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * ny) return;
  const uint64_t i = t / ny, j = t % ny;
  const double qx = dadd(x0, dmul(dx, (double)i));
  const double qy = dadd(y0, dmul(dy, (double)j));
  const int nf = c.nf;
  double* row = out + t * nf;
  const double init = MODE == kSum ? 0.0 : (MODE == kMax ? -pinf() : pinf());
  for (int f = 0; f < nf; f++) row[f] = init;
  for (uint64_t k = 0; k < nz; k++) {
    const double qz = dadd(z0, dmul(dz, (double)k));
    unsigned v = 0;
    const int cell = nn1_exact64<true, true>(c, qx, qy, qz, v);
    if (cell == kTieUnresolved) {
      atomicOr(&bad[1], 1ULL);
      return;
    }
    if (cell < 0) {
      atomicMin(bad, (unsigned long long)t);
      return;
    }
    for (int f = 0; f < nf; f++) {
      const double val = c.fields[(int64_t)cell * nf + f];
      if (MODE == kSum) row[f] = dadd(row[f], val);
      else if (MODE == kMax) row[f] = val > row[f] ? val : row[f];
      else row[f] = val < row[f] ? val : row[f];
    }
  }
  if (MODE == kSum)
    for (int f = 0; f < nf; f++) row[f] = dmul(row[f], dz);
}

// Launch one of the two; `bad` (device, two slots) receives the first pixel
// whose query had no finite distance (UINT64_MAX when none) and, in bad[1],
// 1 when a sample met an exact tie while the reference-order tree was not
// built (the host then builds it and samples again).
int run_grid_sample(vt_cloud* cl, bool brute, int mode, const uint64_t* npix, const double* lo,
                    const double* step, double depth, double* d_out, unsigned long long* d_bad,
                    cudaStream_t st) {
  const uint64_t n = npix[0] * npix[1];
  if (n == 0) return VT_OK;
  const int B = 128;
  const unsigned blocks = (unsigned)((n + B - 1) / B);
  const DevCloud& c = cl->view;
  if (!brute) {
    k_slice<<<blocks, B, 0, st>>>(c, npix[0], npix[1], lo[0], lo[1], step[0], step[1], depth,
                                  d_out, d_bad);
  } else if (mode == kSum) {
    k_brute<kSum><<<blocks, B, 0, st>>>(c, npix[0], npix[1], npix[2], lo[0], lo[1], lo[2],
                                        step[0], step[1], step[2], d_out, d_bad);
  } else if (mode == kMax) {
    k_brute<kMax><<<blocks, B, 0, st>>>(c, npix[0], npix[1], npix[2], lo[0], lo[1], lo[2],
                                        step[0], step[1], step[2], d_out, d_bad);
  } else {
    k_brute<kMin><<<blocks, B, 0, st>>>(c, npix[0], npix[1], npix[2], lo[0], lo[1], lo[2],
                                        step[0], step[1], step[2], d_out, d_bad);
  }
  VT_CUDA(cudaGetLastError());
  return VT_OK;
}

// k-NN of nq device queries; exact ties in the reference's order (a second
// pass on the reference-order tree when the first saw one).  Synchronises.
int run_knn(vt_cloud* cl, const double* d_q, int64_t nq, int k, int64_t* d_ids, double* d_r2,
            cudaStream_t st) {
  const int B = 128;
  if (nq <= 0) return VT_OK;
  if (cl->ws_stats.reserve(1)) return VT_ERR_NOMEM;
  unsigned* d_tie = reinterpret_cast<unsigned*>(cl->ws_stats.p);
  VT_CUDA(cudaMemsetAsync(d_tie, 0, sizeof(unsigned), st));
  const unsigned blocks = (unsigned)((nq + B - 1) / B);
  k_knn<false><<<blocks, B, 0, st>>>(cl->view, d_q, nq, k, d_ids, d_r2, d_tie);
  VT_CUDA(cudaGetLastError());
  unsigned tie = 0;
  VT_CUDA(cudaMemcpyAsync(&tie, d_tie, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  if (!tie) return VT_OK;
  const int rc = build_tie_tree(cl, st);
  if (rc) return rc;
  k_knn<true><<<blocks, B, 0, st>>>(cl->view, d_q, nq, k, d_ids, d_r2, d_tie);
  VT_CUDA(cudaGetLastError());
  return VT_OK;
}

// exclusive prefix sum of counts[0..n) into offsets[0..n]
int scan_offsets(vt_cloud* cl, const int64_t* d_counts, int64_t* d_offsets, int64_t n,
                 cudaStream_t st) {
  size_t bytes = 0;
  VT_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, d_counts, d_offsets + 1, (int)n, st));
  if (cl->ws_tmp.reserve(bytes)) return VT_ERR_NOMEM;
  VT_CUDA(cudaMemsetAsync(d_offsets, 0, sizeof(int64_t), st));
  if (n > 0)
    VT_CUDA(cub::DeviceScan::InclusiveSum(cl->ws_tmp.p, bytes, d_counts, d_offsets + 1, (int)n, st));
  return VT_OK;
}

}  // namespace vt

namespace vt {

// ------------------------------------------- projection without allocation
// Some callers cannot allocate device memory while they run projections: a
// framework whose caching allocator owns the device pool (a cudaMalloc of
// ours would bypass its budget or fail), or a latency-critical loop where
// cudaMalloc/cudaFree and their implicit device synchronisation are not
// acceptable.  vt_project_device_noalloc serves them: the walk's scratch
// (counters and work-queue head, the first-error slot, the diagnosis record,
// the hand-over queue and the global-memory stacks of k_slow) lives in the
// file-scope array below, which every GPU that loads the library holds
// until the process exits.  The cloud and its tree are allocated earlier,
// by vt_cloud_create / vt_cloud_build_tree.
constexpr int64_t kNoAllocMaxRays = 1LL << 20;  // hand-over queue slots (1 per ray)
constexpr int kNoAllocSlowThreads = 128;       // threads of k_slow
constexpr int kNoAllocStackCap = 512;          // pending points per handed-over ray
constexpr size_t kNoAllocOffStats = 0;
constexpr size_t kNoAllocOffDiag = 256;
constexpr size_t kNoAllocOffQueue = 512;
constexpr size_t kNoAllocOffStackId = kNoAllocOffQueue + (size_t)kNoAllocMaxRays * 8;
constexpr size_t kNoAllocOffStackS =
    kNoAllocOffStackId + (size_t)kNoAllocSlowThreads * kNoAllocStackCap * 4;
constexpr size_t kNoAllocBytes =
    kNoAllocOffStackS + (size_t)kNoAllocSlowThreads * kNoAllocStackCap * 8;  // 8.9 MB
static_assert(sizeof(DevStats) <= 256 && sizeof(WalkDiag) <= 256, "scratch layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch, looked up once per device with that
// device current (the host-side symbol is not a device address).
static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_ptr[128] = {};

static int noalloc_scratch(int dev, unsigned char** out) {
  if (dev < 0 || dev >= 128) return set_error(VT_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return set_error(VT_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-allocation "
                                                "scratch failed: ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = (unsigned char*)p;
  }
  *out = g_noalloc_ptr[dev];
  return VT_OK;
}

}  // namespace vt

extern "C" int vt_project_device_noalloc(vt_cloud* cl, const double* d_starts,
                                         const double* d_ends, uint64_t nrays, int mode,
                                         double* d_out, void* stream) {
  using namespace vt;
  try {
    int rc = check_projectable(cl, mode);
    if (rc) return rc;
    if (nrays > (uint64_t)kNoAllocMaxRays)
      return set_error(VT_ERR_INVALID,
                       "vt_project_device_noalloc: " + std::to_string(nrays) +
                           " rays exceed the no-allocation limit of " +
                           std::to_string(kNoAllocMaxRays) + " rays per call");
    std::lock_guard<std::mutex> lk(cl->mu);
    VT_CUDA(cudaSetDevice(cl->device));
    if (nrays == 0) return VT_OK;
    unsigned char* base = nullptr;
    if ((rc = noalloc_scratch(cl->device, &base))) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : cl->stream;
    WalkIO io{};
    io.starts = d_starts;
    io.ends = d_ends;
    io.nrays = (int64_t)nrays;
    io.nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
    io.out = d_out;
    io.stats = reinterpret_cast<DevStats*>(base + kNoAllocOffStats);
    io.slow_q = reinterpret_cast<unsigned long long*>(base + kNoAllocOffQueue);
    io.gstack_id = reinterpret_cast<int*>(base + kNoAllocOffStackId);
    io.gstack_s = reinterpret_cast<double*>(base + kNoAllocOffStackS);
    io.gstack_cap = cl->stack_cap < kNoAllocStackCap ? cl->stack_cap : kNoAllocStackCap;
    io.slow_threads = kNoAllocSlowThreads;
    // counters and the first-error slot are cleared by run_walk_on; the
    // queue and stacks need no clearing (written before they are read)
    return run_walk_on(cl, io, kOutImage, mode, VT_KERNEL_BATCHED, st, nullptr,
                       reinterpret_cast<WalkDiag*>(base + kNoAllocOffDiag), false, false);
  } catch (const std::exception& e) {
    return set_error(VT_ERR_RUNTIME, e.what());
  }
}

