// api.cu -- the C ABI of libvortrace_b200 (include/vortrace_b200.h).
//
// Host side of the boundary the reference implements in src/bindings.cpp
// (pybind11 module Cvortrace), src/pointcloud.cpp (loadPoints filtering,
// padding, warnings, valid_rgba) and src/projection.cpp (driver).  Error and
// warning texts are the reference's.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <limits>
#include <memory>
#include <new>

#include "internal.h"

#include "walkio.h"

namespace vt {
int run_knn(vt_cloud* cl, const double* d_q, int64_t nq, int k, int64_t* d_ids, double* d_r2,
            cudaStream_t st);
int scan_offsets(vt_cloud* cl, const int64_t* d_counts, int64_t* d_offsets, int64_t n,
                 cudaStream_t st);
int run_tape_scatter(vt_cloud* cl, const void* tape, uint64_t n, const double* d_gout,
                     double* d_grad, cudaStream_t st);
int run_tape_scatter_vol(vt_cloud* cl, const void* tape, uint64_t n, const double* d_gout,
                         const double* d_fwd, double* d_grad, cudaStream_t st);
int run_grid_sample(vt_cloud* cl, bool brute, int mode, const uint64_t* npix, const double* lo,
                    const double* step, double depth, double* d_out, unsigned long long* d_bad,
                    cudaStream_t st);
}  // namespace vt

namespace {
thread_local std::string g_last_error;
std::atomic<bool> g_verbose{false};
std::mutex g_warn_mu;
void (*g_warn_cb)(const char*) = nullptr;
std::atomic<int> g_device{0};
constexpr double kPi = 3.14159265358979323846;
}  // namespace

namespace vt {
int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
void warn(const std::string& msg) {
  std::lock_guard<std::mutex> lk(g_warn_mu);
  if (g_warn_cb) g_warn_cb(msg.c_str());
  else std::cerr << "vortrace warning: " << msg << std::endl;
}
bool verbose() { return g_verbose.load(); }
}  // namespace vt

using vt::check_projectable;
using vt::resolve_kernel;
using vt::set_error;

#define VT_GUARD_BEGIN try {
#define VT_GUARD_END                                                       \
  }                                                                        \
  catch (const std::bad_alloc&) {                                          \
    return set_error(VT_ERR_NOMEM, "host allocation failed");             \
  }                                                                        \
  catch (const std::exception& e) {                                        \
    return set_error(VT_ERR_RUNTIME, e.what());                           \
  }

int vt::check_projectable(const vt_cloud* cl, int mode) {
  if (!cl) return set_error(VT_ERR_INVALID, "null cloud handle");
  if (!cl->tree_built)
    return set_error(VT_ERR_RUNTIME, "There is currently no valid tree for this point cloud");
  if (mode < 0 || mode > 3) return set_error(VT_ERR_INVALID, "Unrecognized reduction mode");
  if (mode == VT_REDUCE_VOLUME) {
    if (cl->nfields != 4)
      return set_error(VT_ERR_INVALID,
                       "VolumeRender requires exactly 4 fields (R, G, B, alpha), got " +
                           std::to_string(cl->nfields));
    if (!cl->valid_rgba)
      return set_error(VT_ERR_INVALID,
                       "Volume rendering requires R, G, B values in [0, 1] and alpha >= 0");
  }
  return VT_OK;
}

// VT_KERNEL_AUTO: one ray per thread needs about 20 resident warps on each
// of the device's SMs to hide its memory latency; batches smaller than
// kThreadKernelMinRays cannot fill the device that way and run one ray per
// warp instead (measured on B200, contiguous blocks of the clustered_2m
// image, Mcrossings/s one ray per warp / per thread: 1,024 rays 30 / 5,
// 16,384 rays 126 / 97, 65,536 rays 142 / 324; short rays cross over
// earlier: 16,384 rays of uniform_100k 174 / 188).
// vt_cloud_autotune replaces the rule by its measured choice for batches of
// at least its sample's size.
constexpr uint64_t kThreadKernelMinRays = 65536;
int vt::resolve_kernel(const vt_cloud* cl, int kernel, uint64_t nrays) {
  if (kernel != VT_KERNEL_AUTO) return kernel;
  if (cl->tuned_kernel != VT_KERNEL_AUTO && nrays >= cl->tuned_min_rays) return cl->tuned_kernel;
  return nrays < kThreadKernelMinRays ? VT_KERNEL_BATCHED : VT_KERNEL_THREAD_FP32;
}

static cudaStream_t pick_stream(vt_cloud* cl, void* s) {
  return s ? (cudaStream_t)s : cl->stream;
}

extern "C" {

int vt_abi_version(void) { return VT_ABI_VERSION; }
const char* vt_last_error(void) { return g_last_error.c_str(); }
void vt_set_verbose(int v) { g_verbose.store(v != 0); }
int vt_get_verbose(void) { return g_verbose.load() ? 1 : 0; }
void vt_set_warning_callback(void (*cb)(const char*)) {
  std::lock_guard<std::mutex> lk(g_warn_mu);
  g_warn_cb = cb;
}
int vt_set_device(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return set_error(VT_ERR_CUDA, "no CUDA device available");
  if (device < 0 || device >= n) return set_error(VT_ERR_INVALID, "invalid CUDA device index");
  g_device.store(device);
  return VT_OK;
}

int vt_cloud_create(const double* pos, uint64_t npart, const double* fields,
                    uint64_t npart_fields, uint64_t nfields, const double* subbox,
                    const double* vol, uint64_t nvol, int periodic, vt_cloud** out) {
  VT_GUARD_BEGIN
  if (!out) return set_error(VT_ERR_INVALID, "out must not be NULL");
  *out = nullptr;
  // src/bindings.cpp:53-56, src/pointcloud.cpp:18-22
  if (npart != npart_fields)
    return set_error(VT_ERR_INVALID, "Input sizes must match: pos has " + std::to_string(npart) +
                                         " rows but fields has " + std::to_string(npart_fields));
  if (!subbox) return set_error(VT_ERR_INVALID, "subbox must have 6 values");
  if (npart > 0 && (!pos || !fields)) return set_error(VT_ERR_INVALID, "pos/fields must not be NULL");
  if (nfields == 0) return set_error(VT_ERR_INVALID, "fields must have at least one column");
  if (npart > (uint64_t)std::numeric_limits<int32_t>::max())
    return set_error(VT_ERR_INVALID, "at most 2^31-1 points are supported");
  if (nvol > 0 && !vol) return set_error(VT_ERR_INVALID, "vol must not be NULL when nvol > 0");

  std::unique_ptr<vt_cloud> cl(new vt_cloud());
  cl->device = g_device.load();
  cl->nfields = nfields;
  for (int i = 0; i < 6; ++i) cl->subbox[i] = subbox[i];
  cl->periodic = periodic != 0;
  const bool verbose = vt::verbose();

  // src/pointcloud.cpp:38-53: small-cell warning
  if (nvol > 0) {
    double min_vol = std::numeric_limits<double>::max();
    for (uint64_t i = 0; i < nvol; i++)
      if (vol[i] > 0 && vol[i] < min_vol) min_vol = vol[i];
    if (min_vol < std::numeric_limits<double>::max()) {
      double min_radius = std::cbrt(3.0 * min_vol / (4.0 * kPi));
      if (min_radius < 1e-6)
        vt::warn(
            "Some cells have radii smaller than 1e-6, which approaches the internal "
            "ray-tracing tolerance (1e-9). Results may be unreliable for very small cells. "
            "Consider rescaling your coordinate system.");
    }
  }
  cl->pts.reserve(3 * npart);
  cl->fields.reserve(nfields * npart);
  if (!cl->periodic) {
    // src/pointcloud.cpp:55-108: padding and filtering
    const double dx = subbox[1] - subbox[0], dy = subbox[3] - subbox[2],
                 dz = subbox[5] - subbox[4];
    if (nvol > 0) {
      double max_vol = 0.0;
      for (uint64_t i = 0; i < nvol; i++)
        if (vol[i] > max_vol) max_vol = vol[i];
      cl->pad = 10.0 * std::cbrt(3.0 * max_vol / (4.0 * kPi));
    } else {
      cl->pad = 0.15 * std::max(dx, std::max(dy, dz));
      vt::warn(
          "No cell volumes provided; using 15% of longest box side as padding. Pass vol= for "
          "adaptive padding.");
    }
    const double xmin = subbox[0] - cl->pad, xmax = subbox[1] + cl->pad;
    const double ymin = subbox[2] - cl->pad, ymax = subbox[3] + cl->pad;
    const double zmin = subbox[4] - cl->pad, zmax = subbox[5] + cl->pad;
    if (verbose) std::cout << "Filtering and loading points...\n";
    for (uint64_t i = 0; i < npart; i++) {
      const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
      if (px >= xmin && px <= xmax && py >= ymin && py <= ymax && pz >= zmin && pz <= zmax) {
        cl->pts.push_back(px);
        cl->pts.push_back(py);
        cl->pts.push_back(pz);
        for (uint64_t f = 0; f < nfields; f++) cl->fields.push_back(fields[i * nfields + f]);
        cl->orig_ids.push_back((int64_t)i);
      }
    }
  } else {
    // src/pointcloud.cpp:109-163: periodic, no filtering
    cl->pad = 0.0;
    if (verbose) std::cout << "Loading all points (periodic)...\n";
    double pmin[3], pmax[3];
    for (int d = 0; d < 3; ++d) {
      pmin[d] = std::numeric_limits<double>::max();
      pmax[d] = std::numeric_limits<double>::lowest();
    }
    for (uint64_t i = 0; i < npart; i++) {
      for (int d = 0; d < 3; ++d) {
        const double v = pos[3 * i + d];
        cl->pts.push_back(v);
        if (v < pmin[d]) pmin[d] = v;
        if (v > pmax[d]) pmax[d] = v;
      }
      for (uint64_t f = 0; f < nfields; f++) cl->fields.push_back(fields[i * nfields + f]);
      cl->orig_ids.push_back((int64_t)i);
    }
    if (pmin[0] < subbox[0] || pmax[0] > subbox[1] || pmin[1] < subbox[2] ||
        pmax[1] > subbox[3] || pmin[2] < subbox[4] || pmax[2] > subbox[5])
      return set_error(VT_ERR_INVALID,
                       "Periodic mode: some particles lie outside the bounding box. All "
                       "particles must be within the periodic domain.");
    const double box[3] = {subbox[1] - subbox[0], subbox[3] - subbox[2], subbox[5] - subbox[4]};
    for (int d = 0; d < 3; d++) {
      if (pmax[d] - pmin[d] < 0.6 * box[d]) {
        vt::warn(
            "Periodic mode: particle extent is less than 60% of the bounding box in at least "
            "one dimension. The bounding box may be too large for the particle distribution.");
        break;
      }
    }
  }
  cl->npart = cl->orig_ids.size();
  // src/pointcloud.cpp:167-179
  cl->valid_rgba = false;
  if (nfields == 4 && cl->npart > 0) {
    cl->valid_rgba = true;
    for (uint64_t i = 0; i < cl->npart && cl->valid_rgba; i++) {
      for (int k = 0; k < 3; k++) {
        const double v = cl->fields[i * 4 + k];
        if (v < 0.0 || v > 1.0) {
          cl->valid_rgba = false;
          break;
        }
      }
      if (cl->valid_rgba && cl->fields[i * 4 + 3] < 0.0) cl->valid_rgba = false;
    }
  }
  if (verbose) {
    if (!cl->periodic)
      std::cout << "Filtered " << npart << " -> " << cl->npart << " particles\n";
    else
      std::cout << "Loaded " << cl->npart << " particles (periodic, no filtering)\n";
    std::cout << "Padding: " << cl->pad << "\n";
    std::cout << "Snapshot loaded." << std::endl;
  }
  if (cudaSetDevice(cl->device) != cudaSuccess)
    return set_error(VT_ERR_CUDA, "cannot select CUDA device " + std::to_string(cl->device));
  // a blocking stream: a caller that passes NULL (for instance from the
  // legacy default stream, PyTorch's default) gets its work ordered with that
  // stream's, before and after, as if it had been enqueued there.  A
  // non-blocking stream let an adjoint's atomics race the caller's zero fill
  // of the gradient buffer and the caller's read of the result.
  VT_CUDA(cudaStreamCreateWithFlags(&cl->stream, cudaStreamDefault));
  *out = cl.release();
  return VT_OK;
  VT_GUARD_END
}

void vt_cloud_destroy(vt_cloud* cl) {
  if (!cl) return;
  cudaSetDevice(cl->device);
  if (cl->stream) {
    cudaStreamSynchronize(cl->stream);
    cudaStreamDestroy(cl->stream);
  }
  delete cl;
}

int vt_cloud_build_tree(vt_cloud* cl) {
  VT_GUARD_BEGIN
  if (!cl) return set_error(VT_ERR_INVALID, "null cloud handle");
  std::lock_guard<std::mutex> lk(cl->mu);
  if (cl->npart == 0)
    return set_error(VT_ERR_RUNTIME, "There are no points in the cloud; cannot build tree");
  VT_CUDA(cudaSetDevice(cl->device));
  if (vt::verbose()) std::cout << "Building tree...\n";
  auto t0 = std::chrono::high_resolution_clock::now();
  cl->tree_built = false;
  vt::drop_tie_tree(cl);
  int rc = vt::build_tree_device(cl);
  if (rc) return rc;
  auto t1 = std::chrono::high_resolution_clock::now();
  cl->build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  cl->tree_built = true;
  ++cl->tree_gen;
  if (vt::verbose())
    std::cout << "Tree build took " << (long long)cl->build_ms << " milliseconds." << std::endl;
  return VT_OK;
  VT_GUARD_END
}

int vt_cloud_tree_save(vt_cloud* cl, void* buf, uint64_t cap, uint64_t* size) {
  VT_GUARD_BEGIN
  if (!cl || !size) return set_error(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(cl->mu);
  if (!cl->tree_built)
    return set_error(VT_ERR_RUNTIME, "There is currently no valid tree for this point cloud");
  *size = vt::tree_blob_size(cl);
  if (!buf) return VT_OK;
  if (cap < *size) return set_error(VT_ERR_INVALID, "buffer too small for the tree blob");
  VT_CUDA(cudaSetDevice(cl->device));
  return vt::save_tree_blob(cl, buf);
  VT_GUARD_END
}

int vt_cloud_tree_load(vt_cloud* cl, const void* buf, uint64_t size) {
  VT_GUARD_BEGIN
  if (!cl || !buf) return set_error(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(cl->mu);
  if (cl->npart == 0)
    return set_error(VT_ERR_RUNTIME, "There are no points in the cloud; cannot build tree");
  VT_CUDA(cudaSetDevice(cl->device));
  auto t0 = std::chrono::high_resolution_clock::now();
  cl->tree_built = false;
  vt::drop_tie_tree(cl);
  int rc = vt::load_tree_blob(cl, buf, size);
  if (rc) return rc;
  auto t1 = std::chrono::high_resolution_clock::now();
  cl->build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  cl->tree_built = true;
  ++cl->tree_gen;
  return VT_OK;
  VT_GUARD_END
}

int vt_cloud_set_param(vt_cloud* cl, int param, int64_t value) {
  if (!cl) return set_error(VT_ERR_INVALID, "null cloud handle");
  std::lock_guard<std::mutex> lk(cl->mu);
  switch (param) {
    case VT_PARAM_MAX_ITERATIONS:
      if (value < 1) return set_error(VT_ERR_INVALID, "max iterations must be >= 1");
      cl->max_iter = value;
      return VT_OK;
    case VT_PARAM_STACK_CAP:
      if (value < 2 || value > (1 << 22)) return set_error(VT_ERR_INVALID, "stack capacity out of range");
      cl->stack_cap = (int)value;
      return VT_OK;
    case VT_PARAM_BLOCK_SIZE:
      if (value != 128) return set_error(VT_ERR_INVALID, "block size must be 128");
      cl->block_size = (int)value;
      return VT_OK;
    case VT_PARAM_SMEM_LEVELS:
      if (value < 0 || value > 13) return set_error(VT_ERR_INVALID, "smem levels out of range [0, 13]");
      cl->smem_levels = (int)value;
      return VT_OK;
    case VT_PARAM_BLOCKS_PER_SM:
      if (value < 0 || value > 64) return set_error(VT_ERR_INVALID, "blocks per SM out of range");
      cl->blocks_per_sm = (int)value;
      return VT_OK;
    case VT_PARAM_LOCAL_STACK:
      if (value < 1) return set_error(VT_ERR_INVALID, "local stack size must be >= 1");
      cl->local_stack = value > (1 << 30) ? (1 << 30) : (int)value;
      return VT_OK;
    case VT_PARAM_CACHE:
      if (value < 0 || value > 1) return set_error(VT_ERR_INVALID, "cache mode must be 0 or 1");
      cl->cache_mode = (int)value;
      return VT_OK;
    case VT_PARAM_ADJOINT_KERNEL:
      if (value < VT_KERNEL_AUTO || value > VT_KERNEL_THREAD_FP32)
        return set_error(VT_ERR_INVALID, "unknown kernel");
      cl->adjoint_kernel = (int)value;
      return VT_OK;
    case VT_PARAM_DETAILED_KERNEL:
      if (value < VT_KERNEL_AUTO || value > VT_KERNEL_THREAD_FP32)
        return set_error(VT_ERR_INVALID, "unknown kernel");
      cl->detailed_kernel = (int)value;
      return VT_OK;
    case VT_PARAM_LEAF_SIZE:
      if (value < 2 || value > 64) return set_error(VT_ERR_INVALID, "leaf size out of range [2, 64]");
      cl->leaf_size = (int)value;
      return VT_OK;
    case VT_PARAM_TUNE_LEAF_SIZE:
      if (value < 0 || value > 1) return set_error(VT_ERR_INVALID, "tune leaf size must be 0 or 1");
      cl->tune_leaf = (int)value;
      return VT_OK;
    default:
      return set_error(VT_ERR_INVALID, "unknown parameter " + std::to_string(param));
  }
}

int vt_cloud_set_fields(vt_cloud* cl, const double* fields) {
  VT_GUARD_BEGIN
  if (!cl || !fields) return set_error(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(cl->mu);
  if (!cl->tree_built)
    return set_error(VT_ERR_RUNTIME, "There is currently no valid tree for this point cloud");
  VT_CUDA(cudaSetDevice(cl->device));
  memcpy(cl->fields.data(), fields, cl->npart * cl->nfields * sizeof(double));
  return vt::upload_fields(cl, fields, false, cl->stream);
  VT_GUARD_END
}

int vt_cloud_set_fields_device(vt_cloud* cl, const double* d_fields, void* stream) {
  VT_GUARD_BEGIN
  if (!cl || !d_fields) return set_error(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(cl->mu);
  if (!cl->tree_built)
    return set_error(VT_ERR_RUNTIME, "There is currently no valid tree for this point cloud");
  VT_CUDA(cudaSetDevice(cl->device));
  return vt::upload_fields(cl, d_fields, true, pick_stream(cl, stream));
  VT_GUARD_END
}

int vt_cloud_get_info(const vt_cloud* cl, vt_cloud_info* info) {
  if (!cl || !info) return set_error(VT_ERR_INVALID, "null argument");
  info->npart = cl->npart;
  info->nfields = cl->nfields;
  info->pad = cl->pad;
  for (int i = 0; i < 6; ++i) info->subbox[i] = cl->subbox[i];
  info->valid_rgba = cl->valid_rgba;
  info->tree_built = cl->tree_built;
  info->periodic = cl->periodic;
  info->tree_depth = cl->tree_built ? cl->view.depth : 0;
  info->tree_leaves = cl->tree_built ? (uint64_t)cl->view.nleaves : 0;
  info->tree_build_ms = cl->build_ms;
  info->device_bytes = cl->pts_d.bytes() + cl->pts32_d.bytes() + cl->nodes_d.bytes() +
                       cl->nodes32_d.bytes() + cl->perm_d.bytes() + cl->fields_d.bytes() +
                       cl->boxlo_d.bytes() + cl->boxhi_d.bytes() + cl->leaf32_d.bytes() + cl->tt_nodes_d.bytes() +
                       cl->tt_pts_d.bytes() + cl->tt_tid_d.bytes();
  info->tie_tree_nodes = cl->view.tt_nodes ? cl->tt_nodes_d.n : 0;
  info->tie_tree_depth = cl->view.tt_nodes ? cl->tt_depth : 0;
  info->reserved = 0;
  info->tie_tree_build_ms = cl->tt_ms;
  return VT_OK;
}

int vt_cloud_orig_ids(const vt_cloud* cl, int64_t* out, uint64_t cap) {
  if (!cl) return set_error(VT_ERR_INVALID, "null cloud handle");
  const uint64_t n = cl->orig_ids.size() < cap ? cl->orig_ids.size() : cap;
  if (n && !out) return set_error(VT_ERR_INVALID, "out must not be NULL");
  if (n) memcpy(out, cl->orig_ids.data(), n * sizeof(int64_t));
  return VT_OK;
}

int vt_knn(const vt_cloud* ccl, const double* q, uint64_t nq, int k, int64_t* ids, double* r2) {
  VT_GUARD_BEGIN
  vt_cloud* cl = const_cast<vt_cloud*>(ccl);
  if (!cl) return set_error(VT_ERR_INVALID, "null cloud handle");
  std::lock_guard<std::mutex> lk(cl->mu);
  if (!cl->tree_built)
    return set_error(VT_ERR_RUNTIME, "There is currently no valid tree for this point cloud");
  if (k < 1 || k > 128) return set_error(VT_ERR_INVALID, "k must be in [1, 128]");
  if (nq == 0) return VT_OK;
  VT_CUDA(cudaSetDevice(cl->device));
  vt::DevBuf<double> dq, dr;
  vt::DevBuf<int64_t> di;
  int rc;
  if ((rc = dq.alloc(3 * nq)) || (rc = dr.alloc(nq * k)) || (rc = di.alloc(nq * k))) return rc;
  cudaStream_t st = cl->stream;
  VT_CUDA(cudaMemcpyAsync(dq.p, q, 3 * nq * sizeof(double), cudaMemcpyHostToDevice, st));
  if ((rc = vt::run_knn(cl, dq.p, (int64_t)nq, k, di.p, dr.p, st))) return rc;
  VT_CUDA(cudaMemcpyAsync(ids, di.p, nq * k * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaMemcpyAsync(r2, dr.p, nq * k * sizeof(double), cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  return VT_OK;
  VT_GUARD_END
}

static int project_device_locked(vt_cloud* cl, const double* d_starts, const double* d_ends,
                                 uint64_t nrays, int mode, int kernel, double* d_out,
                                 cudaStream_t st, vt_stats* stats, int out_kind,
                                 int64_t* d_counts) {
  vt::WalkIO io{};
  io.starts = d_starts;
  io.ends = d_ends;
  io.nrays = (int64_t)nrays;
  io.nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
  io.out = d_out;
  io.counts = d_counts;
  return vt::run_walk(cl, io, out_kind, mode, resolve_kernel(cl, kernel, io.nrays), st, stats);
}

int vt_project_device(vt_cloud* cl, const double* d_starts, const double* d_ends,
                      uint64_t nrays, int mode, int kernel, double* d_out, void* stream,
                      vt_stats* stats) {
  VT_GUARD_BEGIN
  int rc = check_projectable(cl, mode);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(cl->mu);
  VT_CUDA(cudaSetDevice(cl->device));
  if (stats) memset(stats, 0, sizeof(*stats));
  if (nrays == 0) return VT_OK;
  return project_device_locked(cl, d_starts, d_ends, nrays, mode, kernel, d_out,
                               pick_stream(cl, stream), stats, vt::kOutImage, nullptr);
  VT_GUARD_END
}

int vt_project(vt_cloud* cl, const double* starts, const double* ends, uint64_t nrays, int mode,
               int kernel, double* out, vt_stats* stats) {
  VT_GUARD_BEGIN
  int rc = check_projectable(cl, mode);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(cl->mu);
  VT_CUDA(cudaSetDevice(cl->device));
  if (stats) memset(stats, 0, sizeof(*stats));
  if (nrays == 0) return VT_OK;
  const int nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
  if ((rc = cl->ws_starts.reserve(3 * nrays)) || (rc = cl->ws_ends.reserve(3 * nrays)) ||
      (rc = cl->ws_out.reserve(nrays * nout)))
    return rc;
  cudaStream_t st = cl->stream;
  if (vt::verbose()) std::cout << "Making projection...\n";
  auto t0 = std::chrono::high_resolution_clock::now();
  VT_CUDA(cudaMemcpyAsync(cl->ws_starts.p, starts, 3 * nrays * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  VT_CUDA(cudaMemcpyAsync(cl->ws_ends.p, ends, 3 * nrays * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  rc = project_device_locked(cl, cl->ws_starts.p, cl->ws_ends.p, nrays, mode, kernel,
                             cl->ws_out.p, st, stats, vt::kOutImage, nullptr);
  if (rc) return rc;
  VT_CUDA(cudaMemcpyAsync(out, cl->ws_out.p, nrays * nout * sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  if (vt::verbose()) {
    auto t1 = std::chrono::high_resolution_clock::now();
    std::cout << "Projection generation took "
              << (long long)std::chrono::duration<double, std::milli>(t1 - t0).count()
              << " milliseconds." << std::endl;
  }
  return VT_OK;
  VT_GUARD_END
}

static int check_grid_args(const double* extent, uint64_t nx, uint64_t ny,
                           const double* bounds) {
  if (!extent || !bounds) return set_error(VT_ERR_INVALID, "null argument");
  if (nx == 0 || ny == 0) return set_error(VT_ERR_INVALID, "grid resolution must be positive");
  if (nx > (uint64_t)1 << 31 || ny > (uint64_t)1 << 31 || nx * ny > (uint64_t)1 << 40)
    return set_error(VT_ERR_INVALID, "grid resolution too large");
  for (int i = 0; i < 4; ++i)
    if (!std::isfinite(extent[i])) return set_error(VT_ERR_INVALID, "extent must be finite");
  if (!std::isfinite(bounds[0]) || !std::isfinite(bounds[1]))
    return set_error(VT_ERR_INVALID, "bounds must be finite");
  return VT_OK;
}

int vt_grid_rays_device(const double extent[4], uint64_t nx, uint64_t ny,
                        const double bounds[2], double* d_starts, double* d_ends, void* stream) {
  VT_GUARD_BEGIN
  int rc = check_grid_args(extent, nx, ny, bounds);
  if (rc) return rc;
  if (!d_starts || !d_ends) return set_error(VT_ERR_INVALID, "null argument");
  return vt::launch_grid_rays(extent, nx, ny, bounds, d_starts, d_ends,
                              (cudaStream_t)stream);
  VT_GUARD_END
}

int vt_project_grid(vt_cloud* cl, const double extent[4], uint64_t nx, uint64_t ny,
                    const double bounds[2], int mode, int kernel, double* out,
                    vt_stats* stats) {
  VT_GUARD_BEGIN
  int rc = check_projectable(cl, mode);
  if (rc) return rc;
  if ((rc = check_grid_args(extent, nx, ny, bounds))) return rc;
  if (!out) return set_error(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(cl->mu);
  VT_CUDA(cudaSetDevice(cl->device));
  if (stats) memset(stats, 0, sizeof(*stats));
  const uint64_t nrays = nx * ny;
  const int nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
  if ((rc = cl->ws_starts.reserve(3 * nrays)) || (rc = cl->ws_ends.reserve(3 * nrays)) ||
      (rc = cl->ws_out.reserve(nrays * nout)))
    return rc;
  cudaStream_t st = cl->stream;
  if ((rc = vt::launch_grid_rays(extent, nx, ny, bounds, cl->ws_starts.p, cl->ws_ends.p, st)))
    return rc;
  rc = project_device_locked(cl, cl->ws_starts.p, cl->ws_ends.p, nrays, mode, kernel,
                             cl->ws_out.p, st, stats, vt::kOutImage, nullptr);
  if (rc) return rc;
  VT_CUDA(cudaMemcpyAsync(out, cl->ws_out.p, nrays * nout * sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  return VT_OK;
  VT_GUARD_END
}

int vt_project_batch(vt_cloud* cl, const vt_grid_desc* grids, uint64_t ngrids,
                     const double* starts, const double* ends, uint64_t nrays, int mode,
                     int kernel, double* out, vt_stats* stats) {
  VT_GUARD_BEGIN
  int rc = check_projectable(cl, mode);
  if (rc) return rc;
  if (ngrids > 0 && !grids) return set_error(VT_ERR_INVALID, "null argument");
  if (nrays > 0 && (!starts || !ends)) return set_error(VT_ERR_INVALID, "null argument");
  uint64_t total = nrays;
  for (uint64_t g = 0; g < ngrids; ++g) {
    if ((rc = check_grid_args(grids[g].extent, grids[g].nx, grids[g].ny, grids[g].bounds)))
      return rc;
    total += grids[g].nx * grids[g].ny;
    if (total > (uint64_t)1 << 40) return set_error(VT_ERR_INVALID, "batch too large");
  }
  if (total > 0 && !out) return set_error(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(cl->mu);
  VT_CUDA(cudaSetDevice(cl->device));
  if (stats) memset(stats, 0, sizeof(*stats));
  if (total == 0) return VT_OK;
  const int nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
  if ((rc = cl->ws_starts.reserve(3 * total)) || (rc = cl->ws_ends.reserve(3 * total)) ||
      (rc = cl->ws_out.reserve(total * nout)))
    return rc;
  cudaStream_t st = cl->stream;
  // the grids' rays made on the device, one block of rays after another,
  // then the arbitrary rays copied in behind them: one walk launch for all
  uint64_t at = 0;
  for (uint64_t g = 0; g < ngrids; ++g) {
    if ((rc = vt::launch_grid_rays(grids[g].extent, grids[g].nx, grids[g].ny, grids[g].bounds,
                                   cl->ws_starts.p + 3 * at, cl->ws_ends.p + 3 * at, st)))
      return rc;
    at += grids[g].nx * grids[g].ny;
  }
  if (nrays > 0) {
    VT_CUDA(cudaMemcpyAsync(cl->ws_starts.p + 3 * at, starts, 3 * nrays * sizeof(double),
                            cudaMemcpyHostToDevice, st));
    VT_CUDA(cudaMemcpyAsync(cl->ws_ends.p + 3 * at, ends, 3 * nrays * sizeof(double),
                            cudaMemcpyHostToDevice, st));
  }
  rc = project_device_locked(cl, cl->ws_starts.p, cl->ws_ends.p, total, mode, kernel,
                             cl->ws_out.p, st, stats, vt::kOutImage, nullptr);
  if (rc) return rc;
  VT_CUDA(cudaMemcpyAsync(out, cl->ws_out.p, total * nout * sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  return VT_OK;
  VT_GUARD_END
}

int vt_project_detailed(vt_cloud* cl, const double* starts, const double* ends, uint64_t nrays,
                        int mode, double* out, int64_t* offsets, vt_segments** segs) {
  VT_GUARD_BEGIN
  if (!segs || !offsets) return set_error(VT_ERR_INVALID, "segs/offsets must not be NULL");
  *segs = nullptr;
  int rc = check_projectable(cl, mode);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(cl->mu);
  VT_CUDA(cudaSetDevice(cl->device));
  std::unique_ptr<vt_segments> sg(new vt_segments());
  sg->device = cl->device;
  offsets[0] = 0;
  if (nrays == 0) {
    *segs = sg.release();
    return VT_OK;
  }
  const int nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
  if ((rc = cl->ws_starts.reserve(3 * nrays)) || (rc = cl->ws_ends.reserve(3 * nrays)) ||
      (rc = cl->ws_out.reserve(nrays * nout)) || (rc = cl->ws_counts.reserve(2 * nrays + 1)))
    return rc;
  cudaStream_t st = cl->stream;
  if (vt::verbose()) std::cout << "Making detailed projection...\n";
  auto t0 = std::chrono::high_resolution_clock::now();
  VT_CUDA(cudaMemcpyAsync(cl->ws_starts.p, starts, 3 * nrays * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  VT_CUDA(cudaMemcpyAsync(cl->ws_ends.p, ends, 3 * nrays * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  int64_t* d_counts = cl->ws_counts.p;
  int64_t* d_off = cl->ws_counts.p + nrays;
  // pass 1: reduction + segment counts; both passes run the same kernel
  const int kernel = resolve_kernel(cl, cl->detailed_kernel, nrays);
  rc = project_device_locked(cl, cl->ws_starts.p, cl->ws_ends.p, nrays, mode, kernel,
                             cl->ws_out.p, st, nullptr, vt::kOutCount, d_counts);
  if (rc) return rc;
  if ((rc = vt::scan_offsets(cl, d_counts, d_off, (int64_t)nrays, st))) return rc;
  VT_CUDA(cudaMemcpyAsync(offsets, d_off, (nrays + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                          st));
  VT_CUDA(cudaMemcpyAsync(out, cl->ws_out.p, nrays * nout * sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  const uint64_t total = (uint64_t)offsets[nrays];
  if ((rc = sg->cell.alloc(total)) || (rc = sg->s_enter.alloc(total)) ||
      (rc = sg->s_exit.alloc(total)))
    return rc;
  sg->count = total;
  // pass 2: segments
  vt::WalkIO io{};
  io.starts = cl->ws_starts.p;
  io.ends = cl->ws_ends.p;
  io.nrays = (int64_t)nrays;
  io.nout = nout;
  io.offsets = d_off;
  io.seg_cell = sg->cell.p;
  io.seg_enter = sg->s_enter.p;
  io.seg_exit = sg->s_exit.p;
  rc = vt::run_walk(cl, io, vt::kOutFill, mode, kernel, st, nullptr);
  if (rc) return rc;
  VT_CUDA(cudaStreamSynchronize(st));
  if (vt::verbose()) {
    auto t1 = std::chrono::high_resolution_clock::now();
    std::cout << "Detailed projection generation took "
              << (long long)std::chrono::duration<double, std::milli>(t1 - t0).count()
              << " milliseconds." << std::endl;
  }
  *segs = sg.release();
  return VT_OK;
  VT_GUARD_END
}

uint64_t vt_segments_count(const vt_segments* s) { return s ? s->count : 0; }

int vt_segments_copy(const vt_segments* s, int64_t* cell_ids, double* s_enter, double* s_exit) {
  if (!s) return set_error(VT_ERR_INVALID, "null segments handle");
  if (s->count == 0) return VT_OK;
  VT_CUDA(cudaSetDevice(s->device));
  if (cell_ids)
    VT_CUDA(cudaMemcpy(cell_ids, s->cell.p, s->count * sizeof(int64_t), cudaMemcpyDeviceToHost));
  if (s_enter)
    VT_CUDA(cudaMemcpy(s_enter, s->s_enter.p, s->count * sizeof(double), cudaMemcpyDeviceToHost));
  if (s_exit)
    VT_CUDA(cudaMemcpy(s_exit, s->s_exit.p, s->count * sizeof(double), cudaMemcpyDeviceToHost));
  return VT_OK;
}

void vt_segments_free(vt_segments* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  delete s;
}

static int adjoint_locked(vt_cloud* cl, const double* d_starts, const double* d_ends,
                          uint64_t nrays, int mode, const double* d_out,
                          const double* d_gout, double* d_grad, cudaStream_t st) {
  vt::WalkIO io{};
  io.starts = d_starts;
  io.ends = d_ends;
  io.nrays = (int64_t)nrays;
  io.nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
  io.gout = d_gout;
  io.fwd = d_out;
  io.grad = d_grad;
  return vt::run_walk(cl, io, vt::kOutAdj, mode, resolve_kernel(cl, cl->adjoint_kernel, nrays), st,
                      nullptr);
}

int vt_project_adjoint_device(vt_cloud* cl, const double* d_starts, const double* d_ends,
                              uint64_t nrays, int mode, const double* d_out,
                              const double* d_grad_out, double* d_grad_fields, void* stream) {
  VT_GUARD_BEGIN
  int rc = check_projectable(cl, mode);
  if (rc) return rc;
  if (mode != VT_REDUCE_SUM && mode != VT_REDUCE_VOLUME)
    return set_error(VT_ERR_INVALID, "adjoint is defined for 'integrate' and 'volume' only");
  if (mode == VT_REDUCE_VOLUME && !d_out)
    return set_error(VT_ERR_INVALID, "the volume adjoint needs the forward output");
  std::lock_guard<std::mutex> lk(cl->mu);
  VT_CUDA(cudaSetDevice(cl->device));
  if (nrays == 0) return VT_OK;
  return adjoint_locked(cl, d_starts, d_ends, nrays, mode, d_out, d_grad_out, d_grad_fields,
                        pick_stream(cl, stream));
  VT_GUARD_END
}

// Slice / BruteProjection: grid of nearest-cell samples, host buffers.
static int grid_sample(vt_cloud* cl, bool brute, int mode, const uint64_t* npix,
                       const double* lo, const double* step, double depth, double* out) {
  const uint64_t n = npix[0] * npix[1];
  const uint64_t nf = cl->nfields;
  int rc;
  if ((rc = cl->ws_out.reserve(n * nf))) return rc;
  if ((rc = cl->ws_slow.reserve(2))) return rc;
  cudaStream_t st = cl->stream;
  unsigned long long flags[2] = {~0ULL, 0ULL};
  for (int pass = 0; pass < 2; ++pass) {
    // a sample that met an exact tie without the reference-order tree sets
    // flags[1]: build the tree and sample again
    VT_CUDA(cudaMemcpyAsync(cl->ws_slow.p, flags, sizeof(flags), cudaMemcpyHostToDevice, st));
    if ((rc = vt::run_grid_sample(cl, brute, mode, npix, lo, step, depth, cl->ws_out.p,
                                  cl->ws_slow.p, st)))
      return rc;
    unsigned long long got[2];
    VT_CUDA(cudaMemcpyAsync(got, cl->ws_slow.p, sizeof(got), cudaMemcpyDeviceToHost, st));
    VT_CUDA(cudaStreamSynchronize(st));
    if (!got[1] || pass == 1) break;
    if ((rc = vt::build_tie_tree(cl, st))) return rc;
  }
  unsigned long long bad = 0;
  VT_CUDA(cudaMemcpyAsync(&bad, cl->ws_slow.p, sizeof(bad), cudaMemcpyDeviceToHost, st));
  if (n * nf > 0)
    VT_CUDA(cudaMemcpyAsync(out, cl->ws_out.p, n * nf * sizeof(double), cudaMemcpyDeviceToHost,
                            st));
  VT_CUDA(cudaStreamSynchronize(st));
  if (bad != ~0ULL)
    return set_error(VT_ERR_INVALID, "pixel " + std::to_string(bad) +
                                         " has no finite distance to any cell (non-finite "
                                         "sample position)");
  return VT_OK;
}

int vt_slice(vt_cloud* cl, const uint64_t npix[2], const double extent[4], double depth,
             double* out) {
  VT_GUARD_BEGIN
  if (!cl || !npix || !extent || !out) return set_error(VT_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(cl->mu);
  // src/slice.cpp:9-21
  if (!cl->tree_built)
    return set_error(VT_ERR_RUNTIME, "There is currently no valid tree for this point cloud");
  const double* sb = cl->subbox;
  if ((extent[0] < sb[0]) || (extent[1] > sb[1]) || (extent[2] < sb[2]) || (extent[3] > sb[3]) ||
      (depth < sb[4]) || (depth > sb[5]))
    return set_error(VT_ERR_RUNTIME, "Slice extent out of bounds of current cloud subbox");
  VT_CUDA(cudaSetDevice(cl->device));
  const double lo[2] = {extent[0], extent[2]};
  const double step[2] = {(extent[1] - extent[0]) / (double)(npix[0] - 1),
                          (extent[3] - extent[2]) / (double)(npix[1] - 1)};
  return grid_sample(cl, false, VT_REDUCE_SUM, npix, lo, step, depth, out);
  VT_GUARD_END
}

int vt_brute_projection(vt_cloud* cl, const uint64_t npix[3], const double extent[6], int mode,
                        double* out) {
  VT_GUARD_BEGIN
  if (!cl || !npix || !extent || !out) return set_error(VT_ERR_INVALID, "null argument");
  // src/brute_projection.cpp:12-32
  if (mode == VT_REDUCE_VOLUME)
    return set_error(VT_ERR_INVALID,
                     "VolumeRender is not supported by BruteProjection: "
                     "it requires ordered ray segments");
  if (mode < 0 || mode > 2) return set_error(VT_ERR_INVALID, "Unrecognized reduction mode");
  std::lock_guard<std::mutex> lk(cl->mu);
  if (!cl->tree_built)
    return set_error(VT_ERR_RUNTIME, "There is currently no valid tree for this point cloud");
  const double* sb = cl->subbox;
  if ((extent[0] < sb[0]) || (extent[1] > sb[1]) || (extent[2] < sb[2]) || (extent[3] > sb[3]) ||
      (extent[4] < sb[4]) || (extent[5] > sb[5]))
    return set_error(VT_ERR_INVALID, "Projection extent out of bounds of current cloud subbox");
  VT_CUDA(cudaSetDevice(cl->device));
  const double lo[3] = {extent[0], extent[2], extent[4]};
  const double step[3] = {(extent[1] - extent[0]) / (double)(npix[0] - 1),
                          (extent[3] - extent[2]) / (double)(npix[1] - 1),
                          (extent[5] - extent[4]) / (double)(npix[2] - 1)};
  return grid_sample(cl, true, mode, npix, lo, step, 0.0, out);
  VT_GUARD_END
}

int vt_cloud_autotune(vt_cloud* cl, const double* starts, const double* ends, uint64_t nrays,
                      int mode, uint64_t max_sample, vt_tune_result* result) {
  VT_GUARD_BEGIN
  int rc = check_projectable(cl, mode);
  if (rc) return rc;
  if (!result) return set_error(VT_ERR_INVALID, "result must not be NULL");
  memset(result, 0, sizeof(*result));
  std::lock_guard<std::mutex> lk(cl->mu);
  VT_CUDA(cudaSetDevice(cl->device));
  if (nrays == 0) return set_error(VT_ERR_INVALID, "autotune needs at least one ray");
  // the sample must fill the device several times over (148 SMs x 9 blocks
  // x 128 threads ~ 170K rays resident), or it favours configurations that
  // cope with low occupancy; with 2^20 rays it also runs the guarded-FP32
  // kernel at the register cap of large launches
  if (max_sample == 0) max_sample = 1048576;
  const uint64_t m = nrays < max_sample ? nrays : max_sample;
  if (!starts || !ends) return set_error(VT_ERR_INVALID, "starts/ends must not be NULL");
  cudaStream_t st = cl->stream;
  // sample: four contiguous blocks (neighbouring rays stay neighbours)
  vt::DevBuf<double> ss, se, so;
  const int nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
  if ((rc = ss.alloc(3 * m)) || (rc = se.alloc(3 * m)) || (rc = so.alloc(m * nout))) return rc;
  uint64_t done = 0;
  for (int b = 0; b < 4; ++b) {
    const uint64_t len = (m * (b + 1)) / 4 - done;
    const uint64_t at = (nrays * (2 * b + 1)) / 8 > len / 2 ? (nrays * (2 * b + 1)) / 8 - len / 2 : 0;
    const uint64_t from = at + len <= nrays ? at : nrays - len;
    VT_CUDA(cudaMemcpyAsync(ss.p + 3 * done, starts + 3 * from, 3 * len * sizeof(double),
                            cudaMemcpyHostToDevice, st));
    VT_CUDA(cudaMemcpyAsync(se.p + 3 * done, ends + 3 * from, 3 * len * sizeof(double),
                            cudaMemcpyHostToDevice, st));
    done += len;
  }
  struct Cand {
    int kernel, smem;
  };
  const Cand cands[] = {{VT_KERNEL_THREAD_FP32, 0}, {VT_KERNEL_THREAD_FP32, 3},
                        {VT_KERNEL_THREAD_FP32, 5}, {VT_KERNEL_THREAD_FP32, 7},
                        {VT_KERNEL_THREAD_FP32, 9}, {VT_KERNEL_BATCHED_FP64, 0},
                        {VT_KERNEL_BATCHED_FP64, 5}, {VT_KERNEL_BATCHED, 5}};
  const int saved_smem = cl->smem_levels, saved_blocks = cl->blocks_per_sm;
  uint64_t crossings = 0;
  // time one configuration (second of two runs); <0 on failure (rc set)
  auto time_cfg = [&](int kernel, int smem, int blocks, double& ms_out) -> int {
    cl->smem_levels = smem;
    cl->blocks_per_sm = blocks;
    for (int rep = 0; rep < 2; ++rep) {  // the first run warms the caches
      vt::WalkIO io{};
      io.starts = ss.p;
      io.ends = se.p;
      io.nrays = (int64_t)m;
      io.nout = nout;
      io.out = so.p;
      vt_stats sts;
      const int r = vt::run_walk(cl, io, vt::kOutImage, mode, kernel, st, &sts);
      if (r) return r;
      ms_out = sts.walk_ms;
      crossings = sts.crossings;
    }
    ++result->tried;
    return VT_OK;
  };
  struct Best {
    int kernel, smem, blocks;
    double ms;
  } best{cands[0].kernel, cands[0].smem, 0, -1.0};
  // 1. kernel (rays per warp) x shared-memory tree depth, all blocks that fit
  auto tune_kernel = [&]() -> int {
    best.ms = -1.0;
    for (const Cand& cd : cands) {
      if (cl->periodic && cd.kernel != VT_KERNEL_THREAD_FP32) continue;  // one kernel serves them
      double ms = 0.0;
      const int r = time_cfg(cd.kernel, cd.smem, 0, ms);
      if (r) return r;
      if (best.ms < 0.0 || ms < best.ms) best = Best{cd.kernel, cd.smem, 0, ms};
    }
    // 2. occupancy of the persistent kernel: fewer resident blocks than its
    // launch bounds allow (3/4 and 1/2 of them) leave each more L1
    const int full = vt::compiled_blocks_per_sm(best.kernel, (int64_t)m);
    for (int blocks : {(3 * full) / 4, full / 2}) {
      if (blocks < 1) blocks = 1;
      double ms = 0.0;
      const int r = time_cfg(best.kernel, best.smem, blocks, ms);
      if (r) return r;
      if (ms < best.ms) best = Best{best.kernel, best.smem, blocks, ms};
    }
    return VT_OK;
  };
  auto restore = [&]() {
    cl->smem_levels = saved_smem;
    cl->blocks_per_sm = saved_blocks;
  };
  if ((rc = tune_kernel())) {
    restore();
    return rc;
  }
  // 3. leaf size (rebuilds the tree for each candidate; the results do not
  // depend on it)
  int best_leaf = cl->leaf_size;
  if (cl->tune_leaf && !cl->periodic) {
    const int leaf0 = cl->leaf_size;
    const Best at0 = best;
    auto rebuild = [&](int leaf) -> int {
      cl->leaf_size = leaf;
      cl->tree_built = false;
      vt::drop_tie_tree(cl);
      const int r = vt::build_tree_device(cl);
      if (r) return r;
      cl->tree_built = true;
      ++cl->tree_gen;
      return VT_OK;
    };
    Best overall = at0;
    for (int leaf : {6, 12}) {
      if (leaf == leaf0) continue;
      if ((rc = rebuild(leaf)) || (rc = tune_kernel())) {
        // leave the cloud as it was: its own leaf size and tree
        restore();
        rebuild(leaf0);
        return rc;
      }
      if (best.ms < overall.ms) {
        overall = best;
        best_leaf = leaf;
      }
    }
    best = overall;
    if (cl->leaf_size != best_leaf && (rc = rebuild(best_leaf))) {
      restore();
      return rc;
    }
  }
  cl->smem_levels = best.smem;
  cl->blocks_per_sm = best.blocks;
  cl->tuned_kernel = best.kernel;
  cl->tuned_min_rays = m;
  result->kernel = best.kernel;
  result->smem_levels = best.smem;
  result->blocks_per_sm = best.blocks;
  result->leaf_size = best_leaf;
  result->sample_rays = m;
  result->mcrossings_per_s = best.ms > 0.0 ? (double)crossings / (best.ms * 1e3) : 0.0;
  return VT_OK;
  VT_GUARD_END
}

int vt_tape_create(vt_cloud* cl, vt_tape** out) {
  VT_GUARD_BEGIN
  if (!out) return set_error(VT_ERR_INVALID, "out must not be NULL");
  *out = nullptr;
  if (!cl) return set_error(VT_ERR_INVALID, "null cloud handle");
  vt_tape* t = new vt_tape();
  t->device = cl->device;
  *out = t;
  return VT_OK;
  VT_GUARD_END
}

void vt_tape_destroy(vt_tape* t) {
  if (!t) return;
  cudaSetDevice(t->device);
  delete t;
}

uint64_t vt_tape_size(const vt_tape* t) { return (t && t->valid) ? t->n : 0; }

int vt_project_device_tape(vt_cloud* cl, vt_tape* tape, const double* d_starts,
                           const double* d_ends, uint64_t nrays, int mode, int kernel,
                           double* d_out, void* stream, vt_stats* stats) {
  VT_GUARD_BEGIN
  int rc = check_projectable(cl, mode);
  if (rc) return rc;
  if (!tape) return set_error(VT_ERR_INVALID, "null tape handle");
  if (mode != VT_REDUCE_SUM && mode != VT_REDUCE_VOLUME)
    return set_error(VT_ERR_INVALID, "a tape is recorded for 'integrate' and 'volume' only");
  if (nrays > (uint64_t)std::numeric_limits<int32_t>::max())
    return set_error(VT_ERR_INVALID, "a taped projection takes at most 2^31-1 rays");
  std::lock_guard<std::mutex> lk(cl->mu);
  VT_CUDA(cudaSetDevice(cl->device));
  if (stats) memset(stats, 0, sizeof(*stats));
  tape->valid = false;
  tape->n = 0;
  tape->nrays = nrays;
  tape->nfields = cl->nfields;
  tape->mode = mode;
  tape->cloud = cl;
  tape->tree_gen = cl->tree_gen;
  const size_t esize = mode == VT_REDUCE_VOLUME ? sizeof(vt::TapeEntryV) : sizeof(vt::TapeEntry);
  if (nrays == 0) {
    tape->valid = true;
    return VT_OK;
  }
  // size: the entries the last taped forward needed, else an estimate from
  // the cloud's last walk (25% margin); a tape that overflows is invalid and
  // its adjoint re-walks the rays
  uint64_t need = tape->want;
  if (cl->cross_per_ray > 0.0)
    need = std::max<uint64_t>(need, (uint64_t)(1.25 * cl->cross_per_ray * (double)nrays) + 1024);
  if (need * esize > tape->buf.bytes()) {
    if ((rc = tape->buf.reserve(need * esize))) return rc;
  }
  tape->cap = tape->buf.bytes() / esize;
  if ((rc = tape->count.reserve(1))) return rc;
  cudaStream_t st = pick_stream(cl, stream);
  VT_CUDA(cudaMemsetAsync(tape->count.p, 0, sizeof(unsigned long long), st));
  vt::WalkIO io{};
  io.starts = d_starts;
  io.ends = d_ends;
  io.nrays = (int64_t)nrays;
  io.nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
  io.out = d_out;
  io.tape = tape->buf.p;
  io.tape_count = tape->count.p;
  io.tape_cap = tape->cap;
  const int k = resolve_kernel(cl, kernel, nrays);
  if ((rc = vt::run_walk(cl, io, vt::kOutTape, mode, k, st, stats))) return rc;
  unsigned long long used = 0;
  VT_CUDA(cudaMemcpyAsync(&used, tape->count.p, sizeof(used), cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  tape->want = used;
  tape->n = used <= tape->cap ? used : 0;
  tape->valid = used <= tape->cap;
  return VT_OK;
  VT_GUARD_END
}

int vt_tape_adjoint_device(vt_cloud* cl, vt_tape* tape, const double* d_starts,
                           const double* d_ends, uint64_t nrays, int mode, const double* d_out,
                           const double* d_grad_out, double* d_grad_fields, void* stream) {
  VT_GUARD_BEGIN
  int rc = check_projectable(cl, mode);
  if (rc) return rc;
  if (!tape) return set_error(VT_ERR_INVALID, "null tape handle");
  if (mode != VT_REDUCE_SUM && mode != VT_REDUCE_VOLUME)
    return set_error(VT_ERR_INVALID, "adjoint is defined for 'integrate' and 'volume' only");
  if (mode == VT_REDUCE_VOLUME && !d_out)
    return set_error(VT_ERR_INVALID, "the volume adjoint needs the forward output");
  std::lock_guard<std::mutex> lk(cl->mu);
  VT_CUDA(cudaSetDevice(cl->device));
  if (nrays == 0) return VT_OK;
  cudaStream_t st = pick_stream(cl, stream);
  if (tape->valid && tape->mode == mode && tape->cloud == cl && tape->nrays == nrays &&
      tape->nfields == cl->nfields && tape->tree_gen == cl->tree_gen) {
    if (mode == VT_REDUCE_VOLUME)
      return vt::run_tape_scatter_vol(cl, tape->buf.p, tape->n, d_grad_out, d_out,
                                      d_grad_fields, st);
    return vt::run_tape_scatter(cl, tape->buf.p, tape->n, d_grad_out, d_grad_fields, st);
  }
  return adjoint_locked(cl, d_starts, d_ends, nrays, mode, d_out, d_grad_out, d_grad_fields, st);
  VT_GUARD_END
}

int vt_project_adjoint(vt_cloud* cl, const double* starts, const double* ends, uint64_t nrays,
                       int mode, const double* out, const double* grad_out,
                       double* grad_fields) {
  VT_GUARD_BEGIN
  int rc = check_projectable(cl, mode);
  if (rc) return rc;
  if (mode != VT_REDUCE_SUM && mode != VT_REDUCE_VOLUME)
    return set_error(VT_ERR_INVALID, "adjoint is defined for 'integrate' and 'volume' only");
  if (mode == VT_REDUCE_VOLUME && !out)
    return set_error(VT_ERR_INVALID, "the volume adjoint needs the forward output");
  std::lock_guard<std::mutex> lk(cl->mu);
  VT_CUDA(cudaSetDevice(cl->device));
  if (nrays == 0) return VT_OK;
  const int nout = mode == VT_REDUCE_VOLUME ? 3 : (int)cl->nfields;
  const uint64_t ng = cl->npart * cl->nfields;
  if ((rc = cl->ws_starts.reserve(3 * nrays)) || (rc = cl->ws_ends.reserve(3 * nrays)) ||
      (rc = cl->ws_out.reserve(nrays * nout)) || (rc = cl->ws_gout.reserve(nrays * nout)) ||
      (rc = cl->ws_grad.reserve(ng)))
    return rc;
  cudaStream_t st = cl->stream;
  VT_CUDA(cudaMemcpyAsync(cl->ws_starts.p, starts, 3 * nrays * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  VT_CUDA(cudaMemcpyAsync(cl->ws_ends.p, ends, 3 * nrays * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  if (out)
    VT_CUDA(cudaMemcpyAsync(cl->ws_out.p, out, nrays * nout * sizeof(double),
                            cudaMemcpyHostToDevice, st));
  VT_CUDA(cudaMemcpyAsync(cl->ws_gout.p, grad_out, nrays * nout * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  VT_CUDA(cudaMemcpyAsync(cl->ws_grad.p, grad_fields, ng * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  rc = adjoint_locked(cl, cl->ws_starts.p, cl->ws_ends.p, nrays, mode, cl->ws_out.p,
                      cl->ws_gout.p, cl->ws_grad.p, st);
  if (rc) return rc;
  VT_CUDA(cudaMemcpyAsync(grad_fields, cl->ws_grad.p, ng * sizeof(double),
                          cudaMemcpyDeviceToHost, st));
  VT_CUDA(cudaStreamSynchronize(st));
  return VT_OK;
  VT_GUARD_END
}

}  // extern "C"
