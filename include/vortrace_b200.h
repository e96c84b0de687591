/*
 * vortrace_b200.h -- C ABI of libvortrace_b200.so, the B200 (sm_100a)
 * implementation of vortrace's exact ray walk through Voronoi meshes.
 *
 * The library replaces the reference's pybind11 module ``Cvortrace``
 * (src/bindings.cpp:71-326) for the projection path.  Every entry point
 * below names the reference interface it stands in for.  Conventions:
 *   - plain pointers and sizes, no C++ or framework types;
 *   - inputs are float64, C-contiguous, and copied by the callee unless the
 *     entry point says "device" (then they are device pointers that stay
 *     owned by the caller);
 *   - every call returns a status code: VT_OK, VT_ERR_INVALID (the
 *     reference's std::invalid_argument, i.e. Python ValueError) or another
 *     code (the reference's std::runtime_error, i.e. Python RuntimeError);
 *     the message is available from vt_last_error() on the calling thread;
 *   - a vt_cloud handle owns its device memory and one CUDA stream, a
 *     blocking one: the work that a call given a NULL stream enqueues there
 *     is ordered with the legacy default stream (stream 0) both ways; calls
 *     on one handle are serialised by an internal mutex.
 */
#ifndef VORTRACE_B200_H
#define VORTRACE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VT_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
#define VT_OK 0
#define VT_ERR_INVALID 1   /* reference: std::invalid_argument -> ValueError */
#define VT_ERR_RUNTIME 2   /* reference: std::runtime_error -> RuntimeError  */
#define VT_ERR_CUDA 3      /* a CUDA call failed (no reference counterpart)  */
#define VT_ERR_NOMEM 4     /* host or device allocation failed               */
/* per-ray walk failures, one per throw site of the reference's Ray::walk   */
#define VT_ERR_MAX_ITER 10     /* src/ray.cpp:260-261 MAX_ITERATIONS           */
#define VT_ERR_SPLIT_BOUNDS 11 /* src/ray.cpp:282-289 split outside segment    */
#define VT_ERR_BINSEARCH 12    /* src/ray.cpp:125-126 bisection no convergence */
#define VT_ERR_PERTURB 13      /* src/ray.cpp:182-184 perturbation exhausted   */
#define VT_ERR_KNN_EXPAND 14   /* src/ray.cpp:331-336 100-NN classification   */
#define VT_ERR_STACK 15        /* pending-point stack above VT_PARAM_STACK_CAP
                                  (the reference's list is heap-grown)         */
#define VT_ERR_PERIODIC_BISECT 18 /* src/ray.cpp:243-246 periodic same-cell ray */
#define VT_ERR_TIE 19          /* an exact distance tie could not be resolved
                                  in the reference's order (no counterpart) */

/* ---- reduction modes: include/mytypes.hpp:14 (ReductionMode) ----------- */
#define VT_REDUCE_SUM 0
#define VT_REDUCE_MAX 1
#define VT_REDUCE_MIN 2
#define VT_REDUCE_VOLUME 3

/* ---- walk kernels ------------------------------------------------------ */
#define VT_KERNEL_AUTO 0        /* THREAD_FP32; BATCHED below 65,536 rays       */
#define VT_KERNEL_PLAIN_FP64 1  /* one ray per thread in the caller's order,    */
                                /* full-FP64 k-NN from the root                 */
#define VT_KERNEL_BATCHED 2     /* persistent queue, one warp per ray,          */
                                /* warp-cooperative guarded-FP32 k-NN           */
#define VT_KERNEL_BATCHED_FP64 3 /* persistent queue, one ray per thread, rays  */
                                 /* in a coherent (sorted) order, bounded FP64  */
                                 /* k-NN                                        */
#define VT_KERNEL_THREAD_FP32 4 /* as BATCHED_FP64 with the top-down bounded    */
                                /* guarded-FP32 k-NN (FP64 re-checks)           */

/* ---- tunable parameters (vt_cloud_set_param) --------------------------- */
#define VT_PARAM_MAX_ITERATIONS 1 /* src/ray.cpp:10, default 100000           */
#define VT_PARAM_STACK_CAP 2      /* pending ray points per ray, default 4096  */
#define VT_PARAM_BLOCK_SIZE 3     /* threads per block of the batched kernel   */
#define VT_PARAM_SMEM_LEVELS 4    /* tree levels staged in shared memory       */
#define VT_PARAM_BLOCKS_PER_SM 5  /* resident blocks per SM (0 = occupancy)    */
#define VT_PARAM_LEAF_SIZE 6      /* max points per tree leaf (before build)   */
#define VT_PARAM_LOCAL_STACK 7    /* pending points a ray may keep in the      */
                                  /* kernels' in-register stack before it is   */
                                  /* handed to the global-stack kernel         */
                                  /* (default and maximum: the compiled size)  */
#define VT_PARAM_CACHE 8          /* batched kernel: per-ray neighbourhood     */
                                  /* cache of the split-point queries (1, 0)   */
#define VT_PARAM_ADJOINT_KERNEL 9 /* walk kernel of the re-walk adjoint        */
                                  /* (VT_KERNEL_*; default AUTO)               */
#define VT_PARAM_DETAILED_KERNEL 10 /* walk kernel of vt_project_detailed      */
                                    /* (VT_KERNEL_*; default AUTO)             */
#define VT_PARAM_TUNE_LEAF_SIZE 11  /* 1: vt_cloud_autotune also times leaf    */
                                    /* sizes 6 and 12 (rebuilding the tree;    */
                                    /* default 0)                              */

typedef struct vt_cloud vt_cloud;
typedef struct vt_segments vt_segments;
typedef struct vt_tape vt_tape;
typedef struct vt_graph vt_graph;

typedef struct {
  uint64_t npart;      /* points after filtering (PointCloud::get_npart)   */
  uint64_t nfields;    /* fields per point (get_nfields)                    */
  double pad;          /* filtering pad (get_pad)                           */
  double subbox[6];    /* [xmin,xmax,ymin,ymax,zmin,zmax] (get_subbox)     */
  int32_t valid_rgba;  /* get_valid_rgba                                    */
  int32_t tree_built;  /* get_tree_built                                    */
  int32_t periodic;    /* get_periodic                                      */
  int32_t tree_depth;  /* internal levels of the implicit tree              */
  uint64_t tree_leaves;
  double tree_build_ms;
  uint64_t device_bytes; /* device memory held by the handle                */
  uint64_t tie_tree_nodes; /* reference-order tree: nodes (0: not built)    */
  int32_t tie_tree_depth;  /* ... its depth in nodes                        */
  int32_t reserved;
  double tie_tree_build_ms;
} vt_cloud_info;

typedef struct {
  uint64_t rays;          /* rays walked                                      */
  uint64_t crossings;     /* segments (cell crossings) produced               */
  uint64_t queries;       /* k-NN queries issued                              */
  uint64_t fp64_resolves; /* guarded-FP32 queries re-resolved fully in FP64  */
  uint64_t slow_rays;     /* rays finished by the degenerate-geometry kernel */
  uint64_t max_stack;     /* deepest pending-point stack seen                */
  double walk_ms;         /* device time of the walk launch(es)               */
  uint64_t search_steps;  /* nodes / node groups the searches expanded        */
  uint64_t fp64_checks;   /* FP64 re-checks of points passing the FP32 test  */
                          /* (these three: the library built with
                             VT_BATCHED_COUNTERS=1, or k_warp)               */
  uint64_t cache_refreshes; /* neighbourhood-cache refills (batched kernel)  */
  uint64_t cache_hits;    /* split queries answered from the cache           */
  uint64_t ties;          /* 1-NN queries whose nearest distance was exactly
                             shared, answered in the reference's order       */
  uint64_t fp32_queries;  /* guarded-FP32 split queries (counters build)     */
  uint64_t fp64_check_queries; /* ... with at least one FP64 re-check        */
  uint64_t trip_cycles[3];  /* counters build, one-ray-per-thread kernel:
                               warp cycles before / in / after the split
                               search of each loop trip                     */
  uint64_t search_warp_steps; /* ... search steps of the warps (longest lane) */
  uint64_t search_lane_steps; /* ... search steps of all lanes                */
} vt_stats;

/* ---- library ----------------------------------------------------------- */
int vt_abi_version(void);
/* Thread-local message of the last failing call on this thread. */
const char *vt_last_error(void);
/* vortrace::verbose (include/mytypes.hpp:17; src/bindings.cpp:91-95) */
void vt_set_verbose(int verbose);
int vt_get_verbose(void);
/* vortrace::warning_handler (include/mytypes.hpp:19-25; src/bindings.cpp:77-80).
 * NULL restores the default (stderr "vortrace warning: <msg>"). */
void vt_set_warning_callback(void (*cb)(const char *msg));
/* Select the CUDA device used by handles created afterwards. */
int vt_set_device(int device);

/* ---- point cloud ------------------------------------------------------- */
/* PointCloud() + PointCloud::loadPoints (src/pointcloud.cpp:12-191,
 * src/bindings.cpp:29-69).  pos: npart x 3; fields: npart_fields x nfields;
 * subbox: 6 values; vol: nvol values or NULL.  Filters to the padded box
 * (non-periodic), builds orig_ids, checks valid_rgba and raises the
 * reference's warnings through the warning callback. */
int vt_cloud_create(const double *pos, uint64_t npart, const double *fields,
                    uint64_t npart_fields, uint64_t nfields, const double *subbox,
                    const double *vol, uint64_t nvol, int periodic, vt_cloud **out);
/* PointCloud::buildTree (src/pointcloud.cpp:193-212): device build. */
int vt_cloud_build_tree(vt_cloud *cloud);
int vt_cloud_set_param(vt_cloud *cloud, int param, int64_t value);
/* Replace the per-point fields (npart x nfields, internal order, i.e. the
 * order of vt_cloud_orig_ids) without rebuilding the tree, and re-check
 * valid_rgba.  No reference counterpart (the reference reloads the points);
 * used by the differentiable path.  The _device form takes a device pointer
 * and a cudaStream_t (NULL: the handle's stream). */
int vt_cloud_set_fields(vt_cloud *cloud, const double *fields);
int vt_cloud_set_fields_device(vt_cloud *cloud, const double *d_fields, void *stream);
/* PointCloud getters (src/bindings.cpp:134-154). */
int vt_cloud_get_info(const vt_cloud *cloud, vt_cloud_info *info);
/* PointCloud::get_orig_ids: writes min(cap, npart) ids. */
int vt_cloud_orig_ids(const vt_cloud *cloud, int64_t *out, uint64_t cap);
void vt_cloud_destroy(vt_cloud *cloud);

/* PointCloud::queryTree(q, k) (src/bindings.cpp:155-174): exact k-NN of nq
 * query points (host buffers); ids are internal (filtered) indices, r2 the
 * squared distances in the reference's summation order.  Missing entries
 * (k > npart) get id -1 and r2 = DBL_MAX.  Exactly tied distances come in
 * the reference's order (the queries are repeated on the reference-order
 * tree when a tie is seen, see vt_cloud_build_tie_tree). */
int vt_knn(const vt_cloud *cloud, const double *q, uint64_t nq, int k, int64_t *ids,
           double *r2);

/* The reference-order tree: nanoflann's middle-split k-d tree (the
 * reference's PointCloud::buildTree, src/pointcloud.cpp:193-212, over
 * include/nanoflann.hpp:858-1003) built on the host and kept on the device
 * beside the device tree.  The device tree answers every query; when the
 * nearest distance of a 1-NN query (ray ends, bisection, perturbation,
 * Slice, BruteProjection) or the order of a k-NN list depends on exactly
 * tied generators (lattices, quantised positions, rays along faces), the
 * query is repeated on this tree so that the tie resolves as in the
 * reference.  Projections build it on first need (and finish the affected
 * rays after it); this call builds it ahead, e.g. before
 * vt_project_device_noalloc, which never allocates and fails with
 * VT_ERR_RUNTIME on a tie while the tree is missing.  Rebuilding or
 * reloading the device tree drops it. */
int vt_cloud_build_tie_tree(vt_cloud *cloud);

/* ---- projections ------------------------------------------------------- */
/* Projection(starts, ends) + makeProjection(cloud, mode) + returnProjection
 * (src/projection.cpp:10-73, src/bindings.cpp:178-201).  Host buffers:
 * starts/ends nrays x 3, out nrays x nout (nout = 3 for VOLUME, else
 * nfields).  stats may be NULL. */
int vt_project(vt_cloud *cloud, const double *starts, const double *ends, uint64_t nrays,
               int mode, int kernel, double *out, vt_stats *stats);
/* Same, on device buffers, enqueued on `stream` (a cudaStream_t, NULL for
 * the handle's stream); returns after the launch has completed. */
int vt_project_device(vt_cloud *cloud, const double *d_starts, const double *d_ends,
                      uint64_t nrays, int mode, int kernel, double *d_out, void *stream,
                      vt_stats *stats);

/* No counterpart in the reference.  vt_project_device without any device
 * allocation, for callers that cannot allocate device memory while they
 * project: a framework whose caching allocator owns the device pool, or a
 * latency-critical loop that cannot afford cudaMalloc/cudaFree and their
 * implicit synchronisation.  Inputs and outputs are the caller's device
 * buffers (starts/ends nrays x 3, out nrays x nout).  The walk kernel is
 * fixed: one warp per ray (VT_KERNEL_BATCHED) in the caller's ray order,
 * because the coherent ray sort of the other batched kernel needs scratch
 * that grows with the batch.  The walk's scratch is a fixed 8.9 MB static
 * device array, placed on a device when the library's device code is first
 * loaded there (with lazy module loading: by the first projection call on
 * that device) and held until exit.  Limits: at most 1,048,576 rays per
 * call (larger requests fail with VT_ERR_INVALID) and 512 pending ray
 * points for rays handed to the global-stack kernel (VT_ERR_STACK beyond).
 * An exact distance tie needs the reference-order tree, which this call
 * never builds: it fails with VT_ERR_RUNTIME until vt_cloud_build_tie_tree
 * has been called on the handle.  The first call on a device looks up the
 * scratch's device address; make that first call before any stream
 * capture.  All calls share the one scratch array: calls that overlap on
 * the GPU (other streams, other threads, other handles on the same device)
 * race and must be serialised by the caller.  The call synchronises
 * `stream` and returns after the launch has completed. */
int vt_project_device_noalloc(vt_cloud *cloud, const double *d_starts, const double *d_ends,
                              uint64_t nrays, int mode, double *d_out, void *stream);

/* The rays of an unrotated projection grid, generated on the device
 * (replaces generate_projection_grid with center=None, vortrace/grid.py:35-44
 * and :100-192, on the host).  extent = {x0, x1, y0, y1}; nx x ny pixels;
 * ray i*ny + j runs from (x_i, y_j, bounds[0]) to (x_i, y_j, bounds[1]), x_i
 * and y_j the pixel centres numpy.linspace gives the reference's generator,
 * bit for bit.  d_starts / d_ends hold nx*ny*3 doubles; enqueued on `stream`
 * (a cudaStream_t) without synchronising. */
int vt_grid_rays_device(const double extent[4], uint64_t nx, uint64_t ny,
                        const double bounds[2], double *d_starts, double *d_ends, void *stream);
/* grid_projection with center=None (vortrace/vortrace.py:141-195): the grid's
 * rays generated on the device (vt_grid_rays_device) and projected as by
 * vt_project; out holds nx*ny*nout values, ray i*ny + j.  No ray crosses the
 * host-device link. */
int vt_project_grid(vt_cloud *cloud, const double extent[4], uint64_t nx, uint64_t ny,
                    const double bounds[2], int mode, int kernel, double *out,
                    vt_stats *stats);

/* One unrotated projection grid of a batch: the rays vt_grid_rays_device
 * makes for extent = {x0, x1, y0, y1}, nx x ny pixels, z from bounds[0] to
 * bounds[1]. */
typedef struct {
  double extent[4];
  uint64_t nx, ny;
  double bounds[2];
} vt_grid_desc;
/* Many projections in one walk launch.  Replaces the reference's one
 * Projection / makeProjection per view (src/projection.cpp:26-73, driven by
 * ProjectionCloud.grid_projection, vortrace/vortrace.py:141-195, once per
 * grid): the rays of ngrids unrotated grids are generated on the device (as
 * vt_grid_rays_device), followed by nrays arbitrary rays from host buffers
 * (starts/ends nrays x 3; nrays may be 0 and the pointers NULL, e.g. rotated
 * views generated on the host), all walked by one launch of `kernel`.  out
 * holds (nx_0*ny_0 + ... + nrays) x nout values, grid by grid (ray i*ny + j
 * of each), then the arbitrary rays in their order.  Errors as
 * vt_project. */
int vt_project_batch(vt_cloud *cloud, const vt_grid_desc *grids, uint64_t ngrids,
                     const double *starts, const double *ends, uint64_t nrays, int mode,
                     int kernel, double *out, vt_stats *stats);

/* makeDetailedProjection + returnSegments (src/projection.cpp:75-144,
 * src/bindings.cpp:206-238).  Writes out (as vt_project) and the CSR
 * offsets (nrays + 1 entries), and returns a library-owned segment list
 * whose arrays are copied out with vt_segments_copy. */
int vt_project_detailed(vt_cloud *cloud, const double *starts, const double *ends,
                        uint64_t nrays, int mode, double *out, int64_t *offsets,
                        vt_segments **segs);
uint64_t vt_segments_count(const vt_segments *segs);
/* cell_ids are internal (filtered) indices, as returnSegments gives them. */
int vt_segments_copy(const vt_segments *segs, int64_t *cell_ids, double *s_enter,
                     double *s_exit);
void vt_segments_free(vt_segments *segs);

/* Adjoint of vt_project with respect to the per-cell fields (no reference
 * counterpart; the reference has no gradients).  grad_out: nrays x nout
 * upstream gradient; out: the forward result (needed by VOLUME); grad_fields
 * (npart x nfields, internal order) is accumulated into, not overwritten.
 * SUM: grad[c,f] += grad_out[r,f] * ds over every segment of ray r in c.
 * VOLUME: reverse-mode front-to-back compositing, transmittance recomputed
 * by re-walking the ray. */
int vt_project_adjoint(vt_cloud *cloud, const double *starts, const double *ends,
                       uint64_t nrays, int mode, const double *out, const double *grad_out,
                       double *grad_fields);
int vt_project_adjoint_device(vt_cloud *cloud, const double *d_starts, const double *d_ends,
                              uint64_t nrays, int mode, const double *d_out,
                              const double *d_grad_out, double *d_grad_fields, void *stream);

/* Saved trees: PointCloud::saveTreeToBytes / loadTreeFromBytes
 * (src/pointcloud.cpp:214-281, used by vortrace/io.py:137-241).  The blob is
 * this library's own (versioned; the permutation and node splits of the
 * device tree, about 4 bytes per point plus 24 per internal node, and a hash
 * of the filtered points); loading it onto a cloud with the same points
 * restores the tree without building it.  vt_cloud_tree_save with buf ==
 * NULL only stores the blob size in *size.  A blob that is not this
 * library's (e.g. a nanoflann index) is refused with VT_ERR_INVALID. */
int vt_cloud_tree_save(vt_cloud *cloud, void *buf, uint64_t cap, uint64_t *size);
int vt_cloud_tree_load(vt_cloud *cloud, const void *buf, uint64_t size);

/* CUDA graph of a forward projection (no reference counterpart): the
 * counter resets, the ray sort, the walk kernel and the global-stack kernel
 * for fixed device buffers (d_starts, d_ends: nrays x 3; d_out: nrays x nout)
 * captured once; vt_graph_launch replays them on `stream` with one
 * cudaGraphLaunch, reading the rays the buffers hold at that time.
 * vt_graph_finish waits for `stream`, returns the counters and reports a
 * failed ray like vt_project_device.  The graph owns its scratch; rebuilding
 * the cloud's tree or reallocating its fields invalidates it (launch then
 * fails).  Launches of one graph must not overlap. */
int vt_graph_create(vt_cloud *cloud, const double *d_starts, const double *d_ends,
                    uint64_t nrays, int mode, int kernel, double *d_out, vt_graph **out);
int vt_graph_launch(vt_graph *graph, void *stream);
int vt_graph_finish(vt_graph *graph, void *stream, vt_stats *stats);
void vt_graph_destroy(vt_graph *graph);

/* Autotuner (no reference counterpart).  On a sample of the given rays
 * (host arrays, nrays x 3) -- up to max_sample (0: 1,048,576) rays in four
 * contiguous blocks, each configuration run twice, the second run timed --
 * it times, one dimension after the other:
 *   1. the walk kernel (rays per warp: one ray per thread with the
 *      guarded-FP32 or the FP64 search, or one ray per warp) x the tree
 *      levels staged in shared memory (0-9);
 *   2. for the chosen pair, the resident blocks per SM of the persistent
 *      kernel (its occupancy: all that its register cap lets fit, 3/4 or
 *      1/2 of them; a value above the cap of a later launch's kernel is
 *      clamped to that cap);
 *   3. with VT_PARAM_TUNE_LEAF_SIZE = 1, the tree's leaf size (the cloud's,
 *      6 and 12; each candidate rebuilds the tree, ~30 ms per 2M points,
 *      and the best one is kept, which invalidates graphs and tapes
 *      recorded before);
 * and makes the fastest the cloud's VT_KERNEL_AUTO choice for batches at
 * least as large as the sample (VT_PARAM_SMEM_LEVELS, VT_PARAM_BLOCKS_PER_SM
 * and VT_PARAM_LEAF_SIZE are set to its values).  The pending-point stack
 * depth needs no tuning: rays whose stack outgrows the in-register one are
 * finished by the global-stack kernel.  Results of every configuration are
 * the same bits; only the speed changes. */
typedef struct {
  int32_t kernel;           /* chosen VT_KERNEL_*                            */
  int32_t smem_levels;      /* chosen tree levels in shared memory           */
  int32_t tried;            /* configurations timed                          */
  int32_t blocks_per_sm;    /* chosen resident blocks per SM (0: all fit)    */
  uint64_t sample_rays;     /* rays in the sample                            */
  double mcrossings_per_s;  /* the chosen configuration on the sample        */
  int32_t leaf_size;        /* the tree's leaf size after tuning             */
  int32_t pad;
} vt_tune_result;
int vt_cloud_autotune(vt_cloud *cloud, const double *starts, const double *ends,
                      uint64_t nrays, int mode, uint64_t max_sample,
                      vt_tune_result *result);

/* Slice::makeSlice (src/slice.cpp:6-60, src/bindings.cpp:259-273): out[(i *
 * npix[1] + j) * nfields + f] = field f of the cell nearest to (extent[0] +
 * i dx, extent[2] + j dy, depth), dx = (extent[1] - extent[0]) / (npix[0] -
 * 1); extent = {xmin, xmax, ymin, ymax} must lie in the cloud's subbox. */
int vt_slice(vt_cloud *cloud, const uint64_t npix[2], const double extent[4], double depth,
             double *out);
/* BruteProjection::makeProjection (src/brute_projection.cpp:10-96,
 * src/bindings.cpp:240-257): per pixel (i, j), SUM (times dz), MAX or MIN
 * of the nearest cells' fields at the npix[2] depth samples; extent = {xmin,
 * xmax, ymin, ymax, zmin, zmax}.  out: npix[0] * npix[1] * nfields. */
int vt_brute_projection(vt_cloud *cloud, const uint64_t npix[3], const double extent[6],
                        int mode, double *out);

/* Segment tape (no reference counterpart; the reference has no gradients).
 * vt_project_device_tape is vt_project_device for SUM or VOLUME that also
 * records, in device memory owned by the tape, one entry per segment: (cell,
 * ray, ds), 16 bytes per crossing (3.2 GB for 2e8 crossings), for SUM; also
 * the transmittance in front of the segment and the colour composited up to
 * it, 48 bytes per crossing, for VOLUME.  vt_tape_adjoint_device then
 * computes the adjoint as a scatter of those entries instead of a second
 * walk.  The tape grows to the entries the last forward on it
 * needed; a forward whose segments did not fit leaves the tape invalid, and
 * the adjoint of an invalid or mismatched tape (other cloud, ray count or
 * mode) re-walks the rays like vt_project_adjoint_device, so the result is
 * the same either way.  One tape per forward whose adjoint is pending. */
int vt_tape_create(vt_cloud *cloud, vt_tape **out);
void vt_tape_destroy(vt_tape *tape);
/* Entries recorded by the last forward on the tape; 0 if they did not fit. */
uint64_t vt_tape_size(const vt_tape *tape);
int vt_project_device_tape(vt_cloud *cloud, vt_tape *tape, const double *d_starts,
                           const double *d_ends, uint64_t nrays, int mode, int kernel,
                           double *d_out, void *stream, vt_stats *stats);
int vt_tape_adjoint_device(vt_cloud *cloud, vt_tape *tape, const double *d_starts,
                           const double *d_ends, uint64_t nrays, int mode,
                           const double *d_out, const double *d_grad_out,
                           double *d_grad_fields, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* VORTRACE_B200_H */
