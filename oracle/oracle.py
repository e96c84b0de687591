"""ctypes front end of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py``
use this module, and only as the checker or the timed CPU baseline.  The
product package ``vortrace_b200`` never imports it.

Contents
--------
* :func:`load_points` -- numpy restatement of ``PointCloud::loadPoints``
  (src/pointcloud.cpp:12-191, non-periodic branch and the periodic
  bounds/extent checks) returning the filtered points, fields, ``orig_ids``,
  ``pad`` and ``valid_rgba`` plus the warnings the reference would emit.
* :class:`OracleTree` -- the C restatement in ``vt_oracle.c`` (nanoflann
  v1.3.2 middle-split tree + exact k-NN + ``Ray::walk`` + reductions).
* :func:`load_reference_module` -- the reference's own ``Cvortrace`` module as
  compiled from its sources by ``oracle/build_ref.sh`` (``None`` when absent).
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import math
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libvt_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

SUM, MAX, MIN, VOLUME = 0, 1, 2, 3
MODES = {"integrate": SUM, "sum": SUM, "max": MAX, "min": MIN, "volume": VOLUME}

_lib = None


def build(force: bool = False) -> str:
    """Compile vt_oracle.c (make) if needed and return the library path."""
    src = os.path.join(HERE, "vt_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        i64p = C.POINTER(C.c_int64)
        szp = C.POINTER(C.c_size_t)
        L.vto_tree_build.restype = C.c_void_p
        L.vto_tree_build.argtypes = [dp, C.c_size_t, C.c_size_t]
        L.vto_tree_free.argtypes = [C.c_void_p]
        L.vto_tree_nnodes.restype = C.c_size_t
        L.vto_tree_nnodes.argtypes = [C.c_void_p]
        L.vto_knn.restype = C.c_size_t
        L.vto_knn.argtypes = [C.c_void_p, dp, C.c_size_t, szp, dp]
        L.vto_knn_batch.argtypes = [C.c_void_p, dp, C.c_size_t, C.c_size_t, i64p, dp]
        L.vto_last_counters.argtypes = [C.POINTER(C.c_ulonglong)]
        L.vto_split_point_distance.restype = C.c_double
        L.vto_split_point_distance.argtypes = [dp, dp, dp, dp]
        L.vto_project.restype = C.c_int
        L.vto_project.argtypes = [C.c_void_p, dp, C.c_size_t, C.c_int, dp, dp, C.c_size_t,
                                  C.c_int, dp, i64p, i64p, i64p, dp, dp, C.c_int, i64p,
                                  C.c_char_p, C.c_size_t]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _i64p(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64)) if a is not None else None


# --------------------------------------------------------------- loadPoints

def load_points(pos, fields, subbox, vol=None, periodic=False):
    """Restatement of ``PointCloud::loadPoints`` (src/pointcloud.cpp:12-191).

    Returns a dict with ``pts`` (n,3), ``fields`` (n,nf), ``orig_ids``,
    ``pad``, ``valid_rgba``, ``nfields`` and ``warnings`` (list of str).
    Raises ValueError where the reference throws ``std::invalid_argument``.
    """
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    fields = np.ascontiguousarray(fields, dtype=np.float64)
    if pos.ndim != 2:
        raise ValueError("pos array must be two-dimensional")
    if fields.ndim == 1:
        nf = 1
        f2 = fields.reshape(-1, 1)
    elif fields.ndim == 2:
        nf = fields.shape[1]
        f2 = fields
    else:
        raise ValueError("fields array must be one-dimensional or two-dimensional")
    if pos.shape[0] != f2.shape[0]:
        raise ValueError(f"Input sizes must match: pos has {pos.shape[0]} rows but fields has "
                         f"{f2.shape[0]}")
    sb = [float(x) for x in subbox]
    warnings = []
    nvol = 0 if vol is None else np.asarray(vol).size
    if nvol > 0:
        v = np.asarray(vol, dtype=np.float64).ravel()
        pos_v = v[v > 0]
        if pos_v.size:
            min_vol = pos_v.min()
            min_radius = math.cbrt(3.0 * min_vol / (4.0 * math.pi))
            if min_radius < 1e-6:
                warnings.append(
                    "Some cells have radii smaller than 1e-6, which approaches the internal "
                    "ray-tracing tolerance (1e-9). Results may be unreliable for very small "
                    "cells. Consider rescaling your coordinate system.")
    if not periodic:
        dx, dy, dz = sb[1] - sb[0], sb[3] - sb[2], sb[5] - sb[4]
        if nvol > 0:
            max_vol = max(0.0, float(np.max(v)))
            pad = 10.0 * math.cbrt(3.0 * max_vol / (4.0 * math.pi))
        else:
            pad = 0.15 * max(dx, dy, dz)
            warnings.append("No cell volumes provided; using 15% of longest box side as "
                            "padding. Pass vol= for adaptive padding.")
        lo = np.array([sb[0] - pad, sb[2] - pad, sb[4] - pad])
        hi = np.array([sb[1] + pad, sb[3] + pad, sb[5] + pad])
        mask = np.all((pos >= lo) & (pos <= hi), axis=1)
        orig_ids = np.nonzero(mask)[0].astype(np.int64)
    else:
        pad = 0.0
        orig_ids = np.arange(pos.shape[0], dtype=np.int64)
        if pos.shape[0]:
            pmin, pmax = pos.min(axis=0), pos.max(axis=0)
            if (pmin[0] < sb[0] or pmax[0] > sb[1] or pmin[1] < sb[2] or pmax[1] > sb[3]
                    or pmin[2] < sb[4] or pmax[2] > sb[5]):
                raise ValueError("Periodic mode: some particles lie outside the bounding box. "
                                 "All particles must be within the periodic domain.")
            box = np.array([sb[1] - sb[0], sb[3] - sb[2], sb[5] - sb[4]])
            if np.any(pmax - pmin < 0.6 * box):
                warnings.append("Periodic mode: particle extent is less than 60% of the "
                                "bounding box in at least one dimension. The bounding box may "
                                "be too large for the particle distribution.")
    pts = np.ascontiguousarray(pos[orig_ids])
    fl = np.ascontiguousarray(f2[orig_ids])
    valid_rgba = False
    if nf == 4 and pts.shape[0] > 0:
        rgb = fl[:, :3]
        valid_rgba = bool(np.all((rgb >= 0.0) & (rgb <= 1.0)) and np.all(fl[:, 3] >= 0.0))
    return {"pts": pts, "fields": fl, "orig_ids": orig_ids, "pad": pad,
            "valid_rgba": valid_rgba, "nfields": nf, "warnings": warnings}


# ---------------------------------------------------------------- the tree

class OracleError(RuntimeError):
    def __init__(self, code, ray, msg):
        super().__init__(msg)
        self.code = code
        self.ray = ray


class OracleTree:
    """nanoflann-identical tree over ``pts`` (n,3) plus walk/projection."""

    def __init__(self, pts, fields=None, valid_rgba=False, leaf_max=10):
        self.pts = np.ascontiguousarray(pts, dtype=np.float64)
        if self.pts.shape[0] == 0:
            raise ValueError("There are no points in the cloud; cannot build tree")
        f = np.ones(self.pts.shape[0]) if fields is None else np.asarray(fields, np.float64)
        self.fields = np.ascontiguousarray(f.reshape(self.pts.shape[0], -1))
        self.nf = self.fields.shape[1]
        self.valid_rgba = bool(valid_rgba)
        L = lib()
        self._h = L.vto_tree_build(_dp(self.pts), self.pts.shape[0], leaf_max)
        if not self._h:
            raise MemoryError("oracle tree build failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().vto_tree_free(h)
            self._h = None

    @property
    def nnodes(self):
        return lib().vto_tree_nnodes(self._h)

    def knn(self, q, k):
        """Batch k-NN: q (m,3) -> ids (m,k) int64 (-1 missing), r2 (m,k)."""
        q = np.ascontiguousarray(np.atleast_2d(q), dtype=np.float64)
        ids = np.empty((q.shape[0], k), np.int64)
        r2 = np.empty((q.shape[0], k), np.float64)
        lib().vto_knn_batch(self._h, _dp(q), q.shape[0], k, _i64p(ids), _dp(r2))
        return ids, r2

    def project(self, starts, ends, mode=SUM, segments=False, nthreads=0):
        """Walk every ray; returns ``out`` (nrays, nout) and, when
        ``segments`` is true, CSR ``(cell_ids, s_enter, s_exit, offsets)``."""
        if isinstance(mode, str):
            mode = MODES[mode]
        s = np.ascontiguousarray(starts, dtype=np.float64).reshape(-1, 3)
        e = np.ascontiguousarray(ends, dtype=np.float64).reshape(-1, 3)
        n = s.shape[0]
        nout = 3 if mode == VOLUME else self.nf
        out = np.zeros((n, nout), np.float64)
        counts = np.zeros(n, np.int64)
        err_ray = np.zeros(1, np.int64)
        msg = C.create_string_buffer(512)
        rc = lib().vto_project(self._h, _dp(self.fields), self.nf, int(self.valid_rgba), _dp(s),
                               _dp(e), n, mode, _dp(out), _i64p(counts), None, None, None,
                               None, nthreads, _i64p(err_ray), msg, 512)
        self._check(rc, err_ray, msg)
        if not segments:
            return out
        offsets = np.zeros(n + 1, np.int64)
        np.cumsum(counts, out=offsets[1:])
        tot = int(offsets[-1])
        cid = np.empty(tot, np.int64)
        se = np.empty(tot, np.float64)
        sx = np.empty(tot, np.float64)
        out2 = np.zeros_like(out)
        rc = lib().vto_project(self._h, _dp(self.fields), self.nf, int(self.valid_rgba), _dp(s),
                               _dp(e), n, mode, _dp(out2), None, _i64p(offsets), _i64p(cid),
                               _dp(se), _dp(sx), nthreads, _i64p(err_ray), msg, 512)
        self._check(rc, err_ray, msg)
        return out, (cid, se, sx, offsets)

    @staticmethod
    def last_counters():
        """k-NN work of the last project() call: queries, nodes visited,
        leaves visited, point distance evaluations."""
        a = (C.c_ulonglong * 4)()
        lib().vto_last_counters(a)
        return {"queries": a[0], "nodes": a[1], "leaves": a[2], "points": a[3]}

    @staticmethod
    def _check(rc, err_ray, msg):
        if rc == 0:
            return
        text = msg.value.decode(errors="replace")
        if rc == 1:
            raise ValueError(text)
        raise OracleError(rc, int(err_ray[0]), text)


def split_point_distance(start, end, p1, p2):
    """``Ray(start,end).findSplitPointDistance(p1, p2)`` (src/ray.cpp:14-60)."""
    start = np.asarray(start, np.float64)
    end = np.asarray(end, np.float64)
    d = end - start
    s = math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
    dirv = np.ascontiguousarray(d / s)
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (start, p1, p2)]
    return lib().vto_split_point_distance(_dp(a[0]), _dp(dirv), _dp(a[1]), _dp(a[2]))


# ------------------------------------------------------- reference module

def load_reference_module():
    """Import the reference's ``Cvortrace`` built into oracle/_ref, or None."""
    if not os.path.isdir(REF_DIR):
        return None
    for fn in os.listdir(REF_DIR):
        if fn.startswith("Cvortrace") and fn.endswith(".so"):
            path = os.path.join(REF_DIR, fn)
            spec = importlib.util.spec_from_file_location("Cvortrace", path)
            mod = importlib.util.module_from_spec(spec)
            try:
                spec.loader.exec_module(mod)
            except ImportError:
                return None
            sys.modules.setdefault("Cvortrace", mod)
            return mod
    return None


def reference_cloud(mod, pos, fields, subbox, vol=None, periodic=False):
    """The reference's PointCloud after loadPoints + buildTree."""
    import warnings as _w
    pc = mod.PointCloud()
    with _w.catch_warnings():
        _w.simplefilter("ignore")
        if vol is not None:
            pc.loadPoints(np.ascontiguousarray(pos, np.float64),
                          np.ascontiguousarray(fields, np.float64), list(subbox),
                          np.ascontiguousarray(vol, np.float64), bool(periodic))
        else:
            pc.loadPoints(np.ascontiguousarray(pos, np.float64),
                          np.ascontiguousarray(fields, np.float64), list(subbox),
                          periodic=bool(periodic))
    pc.buildTree()
    return pc


def reference_project(mod, pos, fields, subbox, starts, ends, mode="integrate", vol=None,
                      detailed=False, periodic=False):
    """Run the reference's own native path: PointCloud.loadPoints/buildTree,
    Projection.makeProjection (or makeDetailedProjection + returnSegments)."""
    pc = reference_cloud(mod, pos, fields, subbox, vol, periodic)
    m = {"integrate": mod.ReductionMode.Sum, "sum": mod.ReductionMode.Sum,
         "max": mod.ReductionMode.Max, "min": mod.ReductionMode.Min,
         "volume": mod.ReductionMode.VolumeRender}[mode]
    proj = mod.Projection(np.ascontiguousarray(starts, np.float64).reshape(-1, 3),
                          np.ascontiguousarray(ends, np.float64).reshape(-1, 3))
    if detailed:
        proj.makeDetailedProjection(pc, m)
        return proj.returnProjection(), proj.returnSegments(), np.asarray(pc.get_orig_ids())
    proj.makeProjection(pc, m)
    return proj.returnProjection(), None, np.asarray(pc.get_orig_ids())
