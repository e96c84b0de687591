"""ctypes binding of libvortrace_b200.so (declared in include/vortrace_b200.h).

The library is loaded on first use.  When it is missing or cannot be loaded
the call fails with an ImportError: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
import warnings

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("VORTRACE_B200_LIB", os.path.join(HERE, "libvortrace_b200.so"))

VT_OK = 0
VT_ERR_INVALID = 1
VT_ERR_RUNTIME = 2
VT_ERR_CUDA = 3
VT_ERR_NOMEM = 4

REDUCE_SUM, REDUCE_MAX, REDUCE_MIN, REDUCE_VOLUME = 0, 1, 2, 3
KERNEL_AUTO, KERNEL_PLAIN_FP64, KERNEL_BATCHED, KERNEL_BATCHED_FP64 = 0, 1, 2, 3
KERNEL_THREAD_FP32 = 4
KERNELS = {"auto": KERNEL_AUTO, "plain": KERNEL_PLAIN_FP64, "batched": KERNEL_BATCHED,
           "batched_fp64": KERNEL_BATCHED_FP64, "thread_fp32": KERNEL_THREAD_FP32}

PARAM_MAX_ITERATIONS = 1
PARAM_STACK_CAP = 2
PARAM_BLOCK_SIZE = 3
PARAM_SMEM_LEVELS = 4
PARAM_BLOCKS_PER_SM = 5
PARAM_LEAF_SIZE = 6
PARAM_LOCAL_STACK = 7
PARAM_CACHE = 8
PARAM_ADJOINT_KERNEL = 9
PARAM_DETAILED_KERNEL = 10
PARAM_TUNE_LEAF_SIZE = 11

# every symbol the header declares (checked by the tests)
EXPORTS = (
    "vt_abi_version", "vt_last_error", "vt_set_verbose", "vt_get_verbose",
    "vt_set_warning_callback", "vt_set_device", "vt_cloud_create", "vt_cloud_build_tree",
    "vt_cloud_set_param", "vt_cloud_set_fields", "vt_cloud_set_fields_device",
    "vt_cloud_get_info", "vt_cloud_orig_ids", "vt_cloud_destroy", "vt_knn",
    "vt_project", "vt_project_device", "vt_project_device_noalloc", "vt_project_detailed",
    "vt_segments_count",
    "vt_segments_copy", "vt_segments_free", "vt_project_adjoint", "vt_project_adjoint_device",
    "vt_tape_create", "vt_tape_destroy", "vt_tape_size", "vt_project_device_tape",
    "vt_tape_adjoint_device", "vt_slice", "vt_brute_projection", "vt_cloud_autotune",
    "vt_graph_create", "vt_graph_launch", "vt_graph_finish", "vt_graph_destroy",
    "vt_cloud_tree_save", "vt_cloud_tree_load", "vt_grid_rays_device", "vt_project_grid",
    "vt_cloud_build_tie_tree", "vt_project_batch",
)


class GridDesc(C.Structure):
    """vt_grid_desc: one unrotated grid of a vt_project_batch call."""
    _fields_ = [("extent", C.c_double * 4), ("nx", C.c_uint64), ("ny", C.c_uint64),
                ("bounds", C.c_double * 2)]


class CloudInfo(C.Structure):
    _fields_ = [("npart", C.c_uint64), ("nfields", C.c_uint64), ("pad", C.c_double),
                ("subbox", C.c_double * 6), ("valid_rgba", C.c_int32),
                ("tree_built", C.c_int32), ("periodic", C.c_int32), ("tree_depth", C.c_int32),
                ("tree_leaves", C.c_uint64), ("tree_build_ms", C.c_double),
                ("device_bytes", C.c_uint64), ("tie_tree_nodes", C.c_uint64),
                ("tie_tree_depth", C.c_int32), ("reserved", C.c_int32),
                ("tie_tree_build_ms", C.c_double)]


class TuneResult(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("smem_levels", C.c_int32), ("tried", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("sample_rays", C.c_uint64),
                ("mcrossings_per_s", C.c_double), ("leaf_size", C.c_int32),
                ("pad", C.c_int32)]

    def as_dict(self):
        names = {v: k for k, v in KERNELS.items()}
        return {"kernel": names.get(self.kernel, self.kernel), "smem_levels": self.smem_levels,
                "blocks_per_sm": self.blocks_per_sm, "leaf_size": self.leaf_size,
                "tried": self.tried, "sample_rays": self.sample_rays,
                "mcrossings_per_s": self.mcrossings_per_s}


class Stats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("crossings", C.c_uint64), ("queries", C.c_uint64),
                ("fp64_resolves", C.c_uint64), ("slow_rays", C.c_uint64),
                ("max_stack", C.c_uint64), ("walk_ms", C.c_double),
                ("search_steps", C.c_uint64), ("fp64_checks", C.c_uint64),
                ("cache_refreshes", C.c_uint64), ("cache_hits", C.c_uint64),
                ("ties", C.c_uint64), ("fp32_queries", C.c_uint64),
                ("fp64_check_queries", C.c_uint64), ("trip_cycles", C.c_uint64 * 3),
                ("search_warp_steps", C.c_uint64), ("search_lane_steps", C.c_uint64)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["trip_cycles"] = list(self.trip_cycles)
        return d


_lib = None
_lock = threading.Lock()
_WARN_CB_T = C.CFUNCTYPE(None, C.c_char_p)


def _on_warning(msg):
    warnings.warn(msg.decode(errors="replace"), UserWarning, stacklevel=3)


_warn_cb = _WARN_CB_T(_on_warning)


def load(path: str | None = None):
    """Load (once) and return the ctypes library handle."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        _lib = _open(path or LIB_PATH)
        return _lib


def load_variant(path: str):
    """A separately loaded build of the library (e.g. the one with the search
    counters compiled in, libvortrace_b200_counters.so): its own handles,
    streams and device memory; not the default library of the package."""
    return _open(path)


def _open(p: str):
    if not os.path.exists(p):
        raise ImportError(
            f"{os.path.basename(p)} not found at {p}; build it with "
            "`python -m vortrace_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(p)
    dp = C.POINTER(C.c_double)
    i64p = C.POINTER(C.c_int64)
    vp = C.c_void_p
    u64 = C.c_uint64
    L.vt_abi_version.restype = C.c_int
    L.vt_last_error.restype = C.c_char_p
    L.vt_set_verbose.argtypes = [C.c_int]
    L.vt_get_verbose.restype = C.c_int
    L.vt_set_warning_callback.argtypes = [_WARN_CB_T]
    L.vt_set_device.argtypes = [C.c_int]
    L.vt_cloud_create.argtypes = [dp, u64, dp, u64, u64, dp, dp, u64, C.c_int,
                                  C.POINTER(vp)]
    L.vt_cloud_build_tree.argtypes = [vp]
    L.vt_cloud_build_tie_tree.argtypes = [vp]
    L.vt_cloud_set_param.argtypes = [vp, C.c_int, C.c_int64]
    L.vt_cloud_set_fields.argtypes = [vp, dp]
    L.vt_cloud_set_fields_device.argtypes = [vp, vp, vp]
    L.vt_cloud_get_info.argtypes = [vp, C.POINTER(CloudInfo)]
    L.vt_cloud_orig_ids.argtypes = [vp, i64p, u64]
    L.vt_cloud_destroy.argtypes = [vp]
    L.vt_cloud_destroy.restype = None
    L.vt_knn.argtypes = [vp, dp, u64, C.c_int, i64p, dp]
    L.vt_project.argtypes = [vp, dp, dp, u64, C.c_int, C.c_int, dp, C.POINTER(Stats)]
    L.vt_project_device.argtypes = [vp, vp, vp, u64, C.c_int, C.c_int, vp, vp,
                                    C.POINTER(Stats)]
    L.vt_project_device_noalloc.argtypes = [vp, vp, vp, u64, C.c_int, vp, vp]
    L.vt_project_detailed.argtypes = [vp, dp, dp, u64, C.c_int, dp, i64p, C.POINTER(vp)]
    L.vt_segments_count.argtypes = [vp]
    L.vt_segments_count.restype = u64
    L.vt_segments_copy.argtypes = [vp, i64p, dp, dp]
    L.vt_segments_free.argtypes = [vp]
    L.vt_segments_free.restype = None
    L.vt_project_adjoint.argtypes = [vp, dp, dp, u64, C.c_int, dp, dp, dp]
    L.vt_project_adjoint_device.argtypes = [vp, vp, vp, u64, C.c_int, vp, vp, vp, vp]
    L.vt_tape_create.argtypes = [vp, C.POINTER(vp)]
    L.vt_tape_destroy.argtypes = [vp]
    L.vt_tape_destroy.restype = None
    L.vt_slice.argtypes = [vp, C.POINTER(u64), dp, C.c_double, dp]
    L.vt_cloud_autotune.argtypes = [vp, dp, dp, u64, C.c_int, u64, C.POINTER(TuneResult)]
    L.vt_graph_create.argtypes = [vp, vp, vp, u64, C.c_int, C.c_int, vp, C.POINTER(vp)]
    L.vt_graph_launch.argtypes = [vp, vp]
    L.vt_cloud_tree_save.argtypes = [vp, vp, u64, C.POINTER(u64)]
    L.vt_cloud_tree_load.argtypes = [vp, vp, u64]
    L.vt_graph_finish.argtypes = [vp, vp, C.POINTER(Stats)]
    L.vt_graph_destroy.argtypes = [vp]
    L.vt_graph_destroy.restype = None
    L.vt_brute_projection.argtypes = [vp, C.POINTER(u64), dp, C.c_int, dp]
    L.vt_grid_rays_device.argtypes = [dp, u64, u64, dp, vp, vp, vp]
    L.vt_project_grid.argtypes = [vp, dp, u64, u64, dp, C.c_int, C.c_int, dp,
                                  C.POINTER(Stats)]
    L.vt_project_batch.argtypes = [vp, vp, u64, dp, dp, u64, C.c_int, C.c_int, dp,
                                   C.POINTER(Stats)]
    L.vt_tape_size.argtypes = [vp]
    L.vt_tape_size.restype = u64
    L.vt_project_device_tape.argtypes = [vp, vp, vp, vp, u64, C.c_int, C.c_int, vp, vp,
                                         C.POINTER(Stats)]
    L.vt_tape_adjoint_device.argtypes = [vp, vp, vp, vp, u64, C.c_int, vp, vp, vp, vp]
    for name in ("vt_cloud_create", "vt_cloud_build_tree", "vt_cloud_build_tie_tree",
                 "vt_cloud_set_param",
                 "vt_cloud_set_fields", "vt_cloud_set_fields_device",
                 "vt_cloud_get_info", "vt_cloud_orig_ids", "vt_knn", "vt_project",
                 "vt_project_device", "vt_project_device_noalloc", "vt_project_detailed",
                 "vt_segments_copy",
                 "vt_project_adjoint", "vt_project_adjoint_device", "vt_set_device",
                 "vt_tape_create", "vt_project_device_tape", "vt_tape_adjoint_device",
                 "vt_slice", "vt_brute_projection", "vt_cloud_autotune",
                 "vt_graph_create", "vt_graph_launch", "vt_graph_finish",
                 "vt_cloud_tree_save", "vt_cloud_tree_load", "vt_grid_rays_device",
                 "vt_project_grid", "vt_project_batch"):
        getattr(L, name).restype = C.c_int
    L.vt_set_warning_callback(_warn_cb)
    return L


class VortraceError(RuntimeError):
    """A per-ray walk failure; ``code`` is the VT_ERR_* status."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def check(rc: int, lib=None):
    """Raise the Python exception the reference raises for this status
    (``lib``: the library that returned it, default the package's)."""
    if rc == VT_OK:
        return
    msg = ((lib or _lib).vt_last_error() or b"").decode(errors="replace")
    if rc == VT_ERR_INVALID:
        raise ValueError(msg)
    if rc == VT_ERR_NOMEM:
        raise MemoryError(msg)
    raise VortraceError(rc, msg)


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def i64ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64)) if a is not None else None


class Tape:
    """Owner of a vt_tape handle (segment tape of a taped 'integrate'
    forward); destroyed with the object."""

    def __init__(self, lib, cloud_handle):
        self._lib = lib
        h = C.c_void_p()
        check(lib.vt_tape_create(cloud_handle, C.byref(h)))
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            self._lib.vt_tape_destroy(h)
            self.h = None
