// internal.h -- host-side internals of libvortrace_b200 (not installed).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/vortrace_b200.h"
#include "common.cuh"

namespace vt {

// Record the message of a failing call for vt_last_error() on this thread;
// returns `code` so call sites can `return set_error(...)`.
int set_error(int code, const std::string& msg);
void warn(const std::string& msg);
bool verbose();

#define VT_CUDA(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return ::vt::set_error(VT_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e_) + \
                                              " at " + __FILE__ + ":" + std::to_string(__LINE__)); \
  } while (0)

// Owning device buffer of T (cudaMalloc/cudaFree).
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      reset();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  int alloc(size_t count) {
    reset();
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return set_error(VT_ERR_NOMEM, std::string("device allocation of ") +
                                         std::to_string(count * sizeof(T)) +
                                         " bytes failed: " + cudaGetErrorString(e));
    }
    n = count;
    return VT_OK;
  }
  // grow-only (contents not preserved)
  int reserve(size_t count) { return count <= n ? VT_OK : alloc(count); }
  size_t bytes() const { return n * sizeof(T); }
};

}  // namespace vt

struct vt_segments {
  vt::DevBuf<int64_t> cell;
  vt::DevBuf<double> s_enter, s_exit;
  uint64_t count = 0;
  int device = 0;
};

struct vt_cloud {
  std::mutex mu;
  int device = 0;
  cudaStream_t stream = nullptr;
  // loadPoints state (src/pointcloud.cpp:12-191)
  uint64_t npart = 0, nfields = 1;
  double pad = 0.0;
  double subbox[6] = {0, 0, 0, 0, 0, 0};
  bool periodic = false, valid_rgba = false, tree_built = false;
  std::vector<double> pts;     // filtered, internal order, n x 3
  std::vector<double> fields;  // filtered, n x nfields
  std::vector<int64_t> orig_ids;
  // parameters
  int64_t max_iter = 100000;
  int stack_cap = 4096;
  int leaf_size = 8;
  int block_size = 128;
  int smem_levels = 5;
  int blocks_per_sm = 0;
  int local_stack = 1 << 30;  // capped to the compiled size in the kernels
  int cache_mode = 0;
  int adjoint_kernel = VT_KERNEL_AUTO;  // kernel of the re-walk adjoint
  int detailed_kernel = VT_KERNEL_AUTO;  // kernel of the detailed projection
  int tuned_kernel = VT_KERNEL_AUTO;    // vt_cloud_autotune's choice for AUTO
  uint64_t tuned_min_rays = 0;          // ... for batches at least this large
  int tune_leaf = 0;                    // vt_cloud_autotune also tries leaf sizes
  uint64_t tree_gen = 0;                // bumped by every tree build or load
  // device tree (tree order)
  vt::DevBuf<double4> pts_d;
  vt::DevBuf<float4> pts32_d;
  vt::DevBuf<double2> nodes_d;
  vt::DevBuf<float2> nodes32_d;
  vt::DevBuf<int32_t> perm_d;
  vt::DevBuf<double> fields_d;
  vt::DevBuf<float4> boxlo_d, boxhi_d;
  vt::DevBuf<float4> leaf32_d;  // SoA leaf blocks (common.cuh)
  // reference-order tree (tietree.cu), built when an exact tie needs it
  vt::DevBuf<vt::TieNode> tt_nodes_d;
  vt::DevBuf<double4> tt_pts_d;
  vt::DevBuf<int32_t> tt_tid_d;
  int tt_depth = 0;
  double tt_ms = 0.0;
  vt::DevCloud view{};
  double build_ms = 0.0;
  double cross_per_ray = 0.0;  // crossings per ray of the last walk (tape sizing)
  // per-call workspace (grow-only)
  vt::DevBuf<double> ws_starts, ws_ends, ws_out, ws_gout, ws_grad;
  vt::DevBuf<int64_t> ws_counts;
  vt::DevBuf<unsigned long long> ws_slow;
  vt::DevBuf<int> ws_stack_id;
  vt::DevBuf<double> ws_stack_s;
  vt::DevBuf<vt::DevStats> ws_stats;
  vt::DevBuf<uint8_t> ws_tmp;
  vt::DevBuf<uint8_t> ws_order;  // ray sort keys, order and CUB scratch
};

// Segment tape of one 'integrate' or 'volume' forward
// (vt_project_device_tape): one entry per segment (TapeEntry / TapeEntryV),
// in no particular order, so that the adjoint is a scatter instead of a
// second walk.
struct vt_tape {
  int device = 0;
  vt::DevBuf<uint8_t> buf;                 // cap entries
  vt::DevBuf<unsigned long long> count;    // entries appended by the last forward
  uint64_t cap = 0;     // entries buf holds
  uint64_t n = 0;       // entries recorded by the last forward
  uint64_t want = 0;    // entries the last forward needed
  uint64_t nrays = 0;   // rays of the last forward
  uint64_t nfields = 0;
  int mode = 0;         // reduction of the last forward (SUM or VOLUME)
  const vt_cloud* cloud = nullptr;
  uint64_t tree_gen = 0;  // the cloud's tree the entries refer to
  bool valid = false;   // the last forward recorded every segment
};

namespace vt {
int build_tree_device(vt_cloud* cl);
// reference-order tree for exact ties (tietree.cu): build (no-op when built)
// and free (the device tree was rebuilt or reloaded)
int build_tie_tree(vt_cloud* cl, cudaStream_t st);
void drop_tie_tree(vt_cloud* cl);
// saved trees (tree_build.cu)
uint64_t tree_blob_size(const vt_cloud* cl);
int save_tree_blob(vt_cloud* cl, void* buf);
int load_tree_blob(vt_cloud* cl, const void* buf, uint64_t size);
int upload_fields(vt_cloud* cl, const double* src, bool src_device, cudaStream_t st);
// tree built, mode valid, volume needs valid RGBA (src/reduction.cpp:59-66)
int check_projectable(const vt_cloud* cl, int mode);
// the kernel VT_KERNEL_AUTO stands for with this cloud and batch size
int resolve_kernel(const vt_cloud* cl, int kernel, uint64_t nrays);
// resident blocks per SM the launch bounds of the walk kernel that runs a
// launch of nrays rays are compiled for (VT_KERNEL_THREAD_FP32,
// _BATCHED_FP64, _BATCHED on the current device; 0 for the others)
int compiled_blocks_per_sm(int kernel, int64_t nrays);
// pixel-centre z-grid rays on the device (grid.cu), ray i*ny + j
int launch_grid_rays(const double extent[4], uint64_t nx, uint64_t ny, const double bounds[2],
                     double* d_starts, double* d_ends, cudaStream_t st);
}
