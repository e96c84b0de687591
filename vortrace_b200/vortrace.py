"""High-level interface: :class:`ProjectionCloud`, a drop-in for the
reference's ``vortrace.ProjectionCloud`` (vortrace/vortrace.py:24-419).

Same constructor, methods, argument handling, output shapes and exceptions
as the reference; the work runs in libvortrace_b200.so (C ABI, ctypes) on a
B200.  Extras that do not change the reference's calls:
  * ``kernel`` attribute: ``'auto'`` (the batched guarded-FP32 kernel, one ray
    per thread; one ray per warp below 65,536 rays; or the autotuner's
    choice), ``'thread_fp32'``, ``'batched_fp64'``, ``'batched'`` (one ray per
    warp), ``'plain'`` (one ray per thread in the caller's order, FP64);
  * ``last_stats``: counters of the last projection (rays, crossings,
    queries, FP64 re-resolves, handed-over rays, walk time);
  * :meth:`batch_projection`: many grids and arbitrary rays in one launch;
  * :meth:`autotune`: kernel and shared-memory tree depth from timings;
  * :meth:`slice`, :class:`Slice`, :class:`BruteProjection`, :meth:`save` /
    :meth:`load` as in the reference (nearest-cell sampling, persistence).
"""
from __future__ import annotations

import ctypes as C
import logging
import warnings

import numpy as np

from . import _lib as L
from . import grid as gr

_log = logging.getLogger("vortrace")

_REDUCTIONS = {
    "integrate": L.REDUCE_SUM,
    "sum": L.REDUCE_SUM,
    "max": L.REDUCE_MAX,
    "min": L.REDUCE_MIN,
    "volume": L.REDUCE_VOLUME,
}


class _Cloud:
    """Owning wrapper of a ``vt_cloud`` handle (the reference's PointCloud)."""

    def __init__(self):
        self._lib = L.load()
        self._h = C.c_void_p()

    def loadPoints(self, pos, fields, subbox, vol=None, periodic=False):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        fields = np.ascontiguousarray(fields, dtype=np.float64)
        if pos.ndim != 2:
            raise ValueError("pos array must be two-dimensional")
        if fields.ndim == 1:
            nf, nfp = 1, fields.shape[0]
        elif fields.ndim == 2:
            nf, nfp = fields.shape[1], fields.shape[0]
        else:
            raise ValueError("fields array must be one-dimensional or two-dimensional")
        if pos.shape[0] != nfp:
            raise ValueError(f"Input sizes must match: pos has {pos.shape[0]} rows but fields "
                             f"has {nfp}")
        sb = np.ascontiguousarray(np.asarray(subbox, dtype=np.float64).ravel())
        if sb.size != 6:
            raise ValueError("subbox must have 6 values")
        v = None if vol is None else np.ascontiguousarray(vol, dtype=np.float64).ravel()
        self.destroy()
        L.check(self._lib.vt_cloud_create(L.dptr(pos), pos.shape[0], L.dptr(fields), nfp, nf,
                                          L.dptr(sb), L.dptr(v), 0 if v is None else v.size,
                                          int(bool(periodic)), C.byref(self._h)))

    def buildTree(self):
        L.check(self._lib.vt_cloud_build_tree(self._h))

    def info(self) -> L.CloudInfo:
        inf = L.CloudInfo()
        L.check(self._lib.vt_cloud_get_info(self._h, C.byref(inf)))
        return inf

    def get_npart(self):
        return self.info().npart

    def get_nfields(self):
        return self.info().nfields

    def get_pad(self):
        return self.info().pad

    def get_valid_rgba(self):
        return bool(self.info().valid_rgba)

    def get_tree_built(self):
        return bool(self.info().tree_built)

    def get_periodic(self):
        return bool(self.info().periodic)

    def get_orig_ids(self):
        n = self.get_npart()
        out = np.empty(n, np.int64)
        L.check(self._lib.vt_cloud_orig_ids(self._h, L.i64ptr(out), n))
        return out

    def set_param(self, param, value):
        L.check(self._lib.vt_cloud_set_param(self._h, param, int(value)))

    # tree persistence (src/bindings.cpp:119-133)
    def saveTreeToBytes(self) -> bytes:
        size = C.c_uint64()
        L.check(self._lib.vt_cloud_tree_save(self._h, None, 0, C.byref(size)))
        buf = C.create_string_buffer(size.value)
        L.check(self._lib.vt_cloud_tree_save(self._h, buf, size.value, C.byref(size)))
        return buf.raw[:size.value]

    def loadTreeFromBytes(self, data: bytes):
        data = bytes(data)
        L.check(self._lib.vt_cloud_tree_load(self._h, data, len(data)))

    def saveTree(self, filename):
        with open(filename, "wb") as f:
            f.write(self.saveTreeToBytes())

    def loadTree(self, filename):
        with open(filename, "rb") as f:
            self.loadTreeFromBytes(f.read())

    def queryTree(self, q, k=None):
        """PointCloud.queryTree (src/bindings.cpp:155-174): nearest id, or
        (ids, r2) arrays for k neighbours; ids are internal indices."""
        qa = np.ascontiguousarray(np.asarray(q, np.float64).reshape(-1, 3))
        kk = 1 if k is None else int(k)
        ids = np.empty((qa.shape[0], kk), np.int64)
        r2 = np.empty((qa.shape[0], kk), np.float64)
        L.check(self._lib.vt_knn(self._h, L.dptr(qa), qa.shape[0], kk, L.i64ptr(ids),
                                 L.dptr(r2)))
        if k is None:
            return int(ids[0, 0])
        return ids[0], r2[0]

    def knn(self, q, k):
        qa = np.ascontiguousarray(np.asarray(q, np.float64).reshape(-1, 3))
        ids = np.empty((qa.shape[0], k), np.int64)
        r2 = np.empty((qa.shape[0], k), np.float64)
        L.check(self._lib.vt_knn(self._h, L.dptr(qa), qa.shape[0], k, L.i64ptr(ids),
                                 L.dptr(r2)))
        return ids, r2

    def destroy(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.vt_cloud_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def _project(cloud: _Cloud, starts, ends, mode, kernel, nout):
    """Projection(starts, ends).makeProjection(cloud, mode) + returnProjection."""
    n = starts.shape[0]
    out = np.empty((n, nout), np.float64)
    st = L.Stats()
    L.check(cloud._lib.vt_project(cloud._h, L.dptr(starts), L.dptr(ends), n, mode,
                                  L.KERNELS[kernel], L.dptr(out), C.byref(st)))
    return out, st


def _project_detailed(cloud: _Cloud, starts, ends, mode, nout, kernel="auto"):
    n = starts.shape[0]
    cloud.set_param(L.PARAM_DETAILED_KERNEL, L.KERNELS[kernel])
    out = np.empty((n, nout), np.float64)
    offsets = np.empty(n + 1, np.int64)
    seg = C.c_void_p()
    lib = cloud._lib
    L.check(lib.vt_project_detailed(cloud._h, L.dptr(starts), L.dptr(ends), n, mode,
                                    L.dptr(out), L.i64ptr(offsets), C.byref(seg)))
    try:
        tot = lib.vt_segments_count(seg)
        cid = np.empty(tot, np.int64)
        se = np.empty(tot, np.float64)
        sx = np.empty(tot, np.float64)
        L.check(lib.vt_segments_copy(seg, L.i64ptr(cid), L.dptr(se), L.dptr(sx)))
    finally:
        lib.vt_segments_free(seg)
    return out, cid, se, sx, offsets


def _as_values(out, nout):
    """returnProjection shape: (n,) for one value per ray, else (n, nout)."""
    return out[:, 0].copy() if nout == 1 else out


def device_grid_args(extent, nres, bounds, proj=None):
    """Arguments of vt_project_grid / vt_grid_rays_device for an unrotated
    grid: ``(extent4, nx, ny, bounds2)`` with the bounds flip of
    generate_projection_grid applied (vortrace/grid.py:163-172), or None
    where the host generator must run instead: an extent whose dtype makes
    numpy compute the pixel centres in another precision (float32), or
    arguments the host generator rejects with the reference's errors."""
    ext = np.asarray(extent)
    if not (ext.dtype == np.float64 or ext.dtype.kind in "iu"):
        return None
    try:
        ext = gr._as_extent(ext).astype(np.float64)
        nx, ny = gr._as_nres(nres)
        b = np.asarray(bounds, dtype=np.float64).ravel()
    except (ValueError, TypeError):
        return None
    if nx <= 0 or ny <= 0 or b.size != 2 or ext.shape != (2, 2):
        return None
    hand = gr.projection_angles(proj)[3] if proj is not None else np.sign(b[1] - b[0])
    if hand != np.sign(b[1] - b[0]):
        b = b[::-1].copy()
    e4 = np.ascontiguousarray([ext[0][0], ext[0][1], ext[1][0], ext[1][1]], np.float64)
    return e4, nx, ny, np.ascontiguousarray(b)


class ProjectionCloud:
    """Projections through an unstructured Voronoi mesh on a B200.

    Same interface as the reference's ``vortrace.ProjectionCloud``.
    """

    _REDUCTION_MAP = dict(_REDUCTIONS)

    def __init__(self, pos, fields, boundbox=None, vol=None, *, periodic: bool = False,
                 _skip_build_tree: bool = False) -> None:
        self.pos_orig = np.ascontiguousarray(pos, dtype=np.float64)
        self.fields_orig = np.ascontiguousarray(fields, dtype=np.float64)
        self.vol_orig = (np.ascontiguousarray(vol, dtype=np.float64)
                         if vol is not None else None)
        self.periodic = periodic
        fa = self.fields_orig
        if fa.ndim == 1:
            self._nfields = 1
        elif fa.ndim == 2:
            self._nfields = fa.shape[1]
        else:
            raise ValueError("fields must be 1D (npart,) or 2D (npart, nfields)")
        if boundbox is None:
            boundbox = [pos[:, 0].min(), pos[:, 0].max(), pos[:, 1].min(), pos[:, 1].max(),
                        pos[:, 2].min(), pos[:, 2].max()]
        self.boundbox = boundbox
        self.kernel = "auto"
        self.last_stats = None
        self._cloud = _Cloud()
        self._cloud.loadPoints(self.pos_orig, self.fields_orig, boundbox, self.vol_orig,
                               periodic)
        if not _skip_build_tree:
            self._cloud.buildTree()
        self.orig_ids = np.array(self._cloud.get_orig_ids())
        _log.info("Applied bounding box filter: %d -> %d particles", len(self.pos_orig),
                  len(self.orig_ids))

    # -------------------------------------------------------------- helpers
    def _validate_reduction(self, reduction: str) -> int:
        mode = self._REDUCTION_MAP.get(reduction)
        if mode is None:
            raise ValueError(f"Unknown reduction {reduction!r}. "
                             f"Use one of {list(self._REDUCTION_MAP)}")
        if mode == L.REDUCE_VOLUME:
            if self._nfields != 4:
                raise ValueError("Volume rendering requires exactly 4 fields "
                                 f"(R, G, B, alpha), got {self._nfields}")
            if not self._cloud.get_valid_rgba():
                raise ValueError("Volume rendering requires R, G, B values in [0, 1] "
                                 "and alpha >= 0")
        return mode

    def _prepare_array_for_backend(self, arr) -> np.ndarray:
        a = np.asarray(arr)
        if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
            a = np.ascontiguousarray(a, dtype=np.float64)
        return a

    def _nout(self, mode):
        return 3 if mode == L.REDUCE_VOLUME else self._nfields

    def _run(self, starts, ends, mode):
        if starts.shape[0] == 0:
            # the reference's returnProjection on an empty result
            raise RuntimeError("Projection has not yet been made")
        out, st = _project(self._cloud, starts, ends, mode, self.kernel, self._nout(mode))
        self.last_stats = st.as_dict()
        return out

    # ----------------------------------------------------------- projections
    def grid_projection(self, extent, nres, bounds, center, *, proj=None, yaw=0.0, pitch=0.0,
                        roll=0.0, reduction="integrate") -> np.ndarray:
        """Grid projection; see the reference (vortrace/vortrace.py:141-195)."""
        mode = self._validate_reduction(reduction)
        if center is None:
            dev = self._device_grid_projection(extent, nres, bounds, proj, mode)
            if dev is not None:
                return dev
        ps, pe = gr.generate_projection_grid(extent, nres, bounds, center, proj=proj, yaw=yaw,
                                             pitch=pitch, roll=roll)
        shape = ps.shape
        ps = np.ascontiguousarray(ps.reshape(-1, shape[-1]))
        pe = np.ascontiguousarray(pe.reshape(-1, pe.shape[-1]))
        dat = self._run(ps, pe, mode)
        nout = self._nout(mode)
        if nout == 1:
            return np.reshape(dat, shape[:-1])
        return np.reshape(dat, (*shape[:-1], nout))

    def _device_grid_projection(self, extent, nres, bounds, proj, mode):
        """An unrotated grid's projection with its rays generated on the device
        (vt_project_grid); None where the host generator must run instead."""
        args = device_grid_args(extent, nres, bounds, proj)
        if args is None:
            return None
        e4, nx, ny, b = args
        nout = self._nout(mode)
        out = np.empty((nx * ny, nout), np.float64)
        st = L.Stats()
        cl = self._cloud
        L.check(cl._lib.vt_project_grid(cl._h, L.dptr(e4), nx, ny, L.dptr(b), mode,
                                        L.KERNELS[self.kernel], L.dptr(out), C.byref(st)))
        self.last_stats = st.as_dict()
        if nout == 1:
            return out.reshape(nx, ny)
        return out.reshape(nx, ny, nout)

    def projection(self, pos_start, pos_end, *, reduction="integrate") -> np.ndarray:
        """Projection of arbitrary rays (vortrace/vortrace.py:197-227)."""
        mode = self._validate_reduction(reduction)
        pos_start = self._prepare_array_for_backend(pos_start)
        pos_end = self._prepare_array_for_backend(pos_end)
        if (pos_start.ndim != 2 or pos_end.ndim != 2 or pos_start.shape != pos_end.shape
                or pos_start.shape[1] != 3):
            raise ValueError("pos_start / pos_end must be 2D arrays of identical shape (N,3)")
        out = self._run(pos_start, pos_end, mode)
        return _as_values(out, self._nout(mode))

    def traced_projection(self, pos_start, pos_end, return_midpoint: bool = True, *,
                          reduction: str = "integrate", flatten: bool = False) -> tuple:
        """Projection with per-segment detail (vortrace/vortrace.py:229-338)."""
        ps = np.asarray(pos_start)
        pe = np.asarray(pos_end)
        single = False
        if ps.ndim == 1 and pe.ndim == 1:
            if ps.shape != (3,) or pe.shape != (3,):
                raise ValueError("If 1D, pos_start and pos_end must both have shape (3,)")
            ps = ps[np.newaxis, :]
            pe = pe[np.newaxis, :]
            single = True
        elif ps.ndim == 2 and pe.ndim == 2:
            if ps.shape != pe.shape or ps.shape[1] != 3:
                raise ValueError("pos_start and pos_end must be 2D arrays of identical shape "
                                 "(N, 3)")
            if ps.shape[0] == 1:
                single = True
        else:
            raise ValueError("pos_start and pos_end must both be 1D shape (3,) or both 2D "
                             "shape (N, 3)")
        ps = self._prepare_array_for_backend(ps)
        pe = self._prepare_array_for_backend(pe)
        mode = self._validate_reduction(reduction)
        nout = self._nout(mode)
        if ps.shape[0] == 0:
            raise RuntimeError("Projection has not yet been made")
        out, cid, se, sx, offsets = _project_detailed(self._cloud, ps, pe, mode, nout,
                                                      self.kernel)
        values = _as_values(out, nout)
        cell_ids = self.orig_ids[cid]
        ds_vals = sx - se
        s_vals = (se + sx) / 2.0 if return_midpoint else se
        if single:
            if mode == L.REDUCE_VOLUME or self._nfields > 1:
                val_out = values[0]
            else:
                val_out = values[0] if values.ndim == 1 else values[0, 0]
            return val_out, cell_ids, s_vals, ds_vals
        if flatten:
            return values, cell_ids, s_vals, ds_vals, offsets
        nr = len(offsets) - 1
        return (values, [cell_ids[offsets[i]:offsets[i + 1]] for i in range(nr)],
                [s_vals[offsets[i]:offsets[i + 1]] for i in range(nr)],
                [ds_vals[offsets[i]:offsets[i + 1]] for i in range(nr)])

    def single_projection(self, *args, **kwargs):
        """Removed.  Use :meth:`traced_projection` instead."""
        raise AttributeError("'single_projection' has been removed. "
                             "Use 'traced_projection' instead.")

    def batch_projection(self, grids=(), rays=None, *, reduction="integrate"):
        """Many projections in one launch (extension; not in the reference).

        ``grids``: sequence of dicts with the keyword arguments of
        :meth:`grid_projection` (``extent``, ``nres``, ``bounds``, ``center``
        and optionally ``proj/yaw/pitch/roll``); ``rays``: optional
        ``(pos_start, pos_end)`` arrays of arbitrary rays.  Returns a list of
        images (one per grid) and, when ``rays`` is given, the ray values.
        """
        mode = self._validate_reduction(reduction)
        # unrotated grids: rays made on the device (vt_project_batch); the
        # others (rotations, float32 extents) on the host, walked in the same
        # launch behind them, then the arbitrary rays
        descs, dev_idx, starts, ends, host_idx, shapes = [], [], [], [], [], []
        for i, g in enumerate(grids):
            args = None
            if g.get("center") is None:
                args = device_grid_args(g["extent"], g["nres"], g["bounds"], g.get("proj"))
            if args is not None:
                e4, nx, ny, b = args
                d = L.GridDesc()
                d.extent[:] = list(e4)
                d.nx, d.ny = nx, ny
                d.bounds[:] = list(b)
                descs.append(d)
                dev_idx.append(i)
                shapes.append((nx, ny))
                continue
            ps, pe = gr.generate_projection_grid(
                g["extent"], g["nres"], g["bounds"], g.get("center"), proj=g.get("proj"),
                yaw=g.get("yaw", 0.0), pitch=g.get("pitch", 0.0), roll=g.get("roll", 0.0))
            shapes.append(ps.shape[:-1])
            starts.append(ps.reshape(-1, 3))
            ends.append(pe.reshape(-1, 3))
            host_idx.append(i)
        nextra = 0
        if rays is not None:
            rs = self._prepare_array_for_backend(rays[0]).reshape(-1, 3)
            re_ = self._prepare_array_for_backend(rays[1]).reshape(-1, 3)
            if rs.shape != re_.shape:
                raise ValueError("pos_start / pos_end must have identical shapes")
            starts.append(rs)
            ends.append(re_)
            nextra = rs.shape[0]
        S = np.ascontiguousarray(np.concatenate(starts)) if starts else np.empty((0, 3))
        E = np.ascontiguousarray(np.concatenate(ends)) if ends else np.empty((0, 3))
        ndev = sum(int(d.nx * d.ny) for d in descs)
        nout = self._nout(mode)
        if ndev + S.shape[0] == 0:
            raise RuntimeError("Projection has not yet been made")
        out = np.empty((ndev + S.shape[0], nout), np.float64)
        st = L.Stats()
        cl = self._cloud
        arr = (L.GridDesc * max(1, len(descs)))(*descs)
        L.check(cl._lib.vt_project_batch(cl._h, C.cast(arr, C.c_void_p), len(descs),
                                         L.dptr(S) if S.shape[0] else None,
                                         L.dptr(E) if E.shape[0] else None, S.shape[0], mode,
                                         L.KERNELS[self.kernel], L.dptr(out), C.byref(st)))
        self.last_stats = st.as_dict()
        imgs = [None] * len(grids)
        o = 0
        for i in dev_idx + host_idx:  # the order of the rays in `out`
            sh = shapes[i]
            k = int(np.prod(sh))
            blk = out[o:o + k]
            imgs[i] = blk.reshape(sh) if nout == 1 else blk.reshape(*sh, nout)
            o += k
        if rays is not None:
            return imgs, _as_values(out[o:], nout)
        return imgs

    # ------------------------------------------------------------- cloud
    def query(self, q, k=1):
        """Exact k nearest generators of query points (original ids, r^2)."""
        ids, r2 = self._cloud.knn(q, k)
        return np.where(ids >= 0, self.orig_ids[np.maximum(ids, 0)], -1), r2

    def autotune(self, pos_start, pos_end, *, reduction="integrate",
                 max_sample: int = 1048576, leaf_size: bool = False) -> dict:
        """Time the walk kernels (rays per warp), shared-memory tree depths and
        resident blocks per SM on a sample of these rays (extension; not in
        the reference) and make the fastest the ``'auto'`` configuration
        for batches at least as large as the sample; with ``leaf_size`` the
        tree is also rebuilt with leaf sizes 6 and 12 and the fastest kept.
        Results do not change, only the speed.  Returns the choice."""
        mode = self._validate_reduction(reduction)
        S = self._prepare_array_for_backend(pos_start).reshape(-1, 3)
        E = self._prepare_array_for_backend(pos_end).reshape(-1, 3)
        if S.shape != E.shape:
            raise ValueError("pos_start / pos_end must have identical shapes")
        res = L.TuneResult()
        self._cloud.set_param(L.PARAM_TUNE_LEAF_SIZE, 1 if leaf_size else 0)
        L.check(self._cloud._lib.vt_cloud_autotune(self._cloud._h, L.dptr(S), L.dptr(E),
                                                   S.shape[0], mode, int(max_sample),
                                                   C.byref(res)))
        return res.as_dict()

    # ------------------------------------------------ tree serialization
    TREE_MAGIC = b"VTB2TREE"

    def save_tree_bytes(self) -> bytes | None:
        """The device tree as bytes (this library's blob), or None if not
        built (vortrace/vortrace.py:389-393)."""
        if self._cloud.get_tree_built():
            return self._cloud.saveTreeToBytes()
        return None

    def load_tree_bytes(self, data: bytes) -> None:
        """Restore the tree from :meth:`save_tree_bytes` output.  A blob of
        another library (e.g. the reference's nanoflann index) cannot be used
        by the device walk: the tree is then built on the device instead."""
        data = bytes(data)
        if data[:8] != self.TREE_MAGIC:
            warnings.warn("tree blob is not a vortrace_b200 device tree (e.g. a nanoflann "
                          "index); rebuilding the tree on the device", UserWarning,
                          stacklevel=2)
            self._cloud.buildTree()
            return
        self._cloud.loadTreeFromBytes(data)

    def save(self, filename, *, fmt: str = "npz", save_tree: bool = True) -> None:
        """Save this cloud (see :func:`vortrace_b200.io.save_cloud`)."""
        from .io import save_cloud
        save_cloud(filename, self, fmt=fmt, save_tree=save_tree)

    @classmethod
    def load(cls, filename) -> "ProjectionCloud":
        """Load a cloud (see :func:`vortrace_b200.io.load_cloud`)."""
        from .io import load_cloud
        return load_cloud(filename)

    def slice(self, extent, nres, depth: float) -> np.ndarray:
        """2D slice at constant depth: the nearest cell's field values at
        each pixel (vortrace/vortrace.py:347-383; src/slice.cpp:6-60).

        ``extent`` = [xmin, xmax, ymin, ymax]; ``nres``: int or (nx, ny);
        pixel (i, j) sits at (xmin + i dx, ymin + j dy, depth) with
        dx = (xmax - xmin) / (nx - 1).  Returns (nx, ny) for one field,
        else (nx, ny, nfields).
        """
        npix = (nres, nres) if isinstance(nres, int) else tuple(nres)
        extent_arr = np.asarray(extent, dtype=np.float64).ravel()
        if extent_arr.size != 4:
            raise ValueError("extent must have 4 elements [xmin, xmax, ymin, ymax]")
        dat = Slice(list(npix), list(extent_arr), float(depth))
        dat.makeSlice(self._cloud)
        out = dat.returnSlice()
        if self._nfields == 1:
            return out.reshape(npix[0], npix[1])
        return out.reshape(npix[0], npix[1], self._nfields)


class Slice:
    """The reference's ``Cvortrace.Slice`` (src/bindings.cpp:259-273)."""

    def __init__(self, npix, extent, depth):
        self.npix = (int(npix[0]), int(npix[1]))
        self.extent = np.ascontiguousarray(extent, np.float64).reshape(4)
        self.depth = float(depth)
        self._data = None

    def makeSlice(self, cloud: _Cloud):
        n = self.npix[0] * self.npix[1]
        nf = int(cloud.info().nfields)
        out = np.empty((n, nf), np.float64)
        npx = (C.c_uint64 * 2)(*self.npix)
        L.check(cloud._lib.vt_slice(cloud._h, npx, L.dptr(self.extent), self.depth,
                                    L.dptr(out)))
        self._data = out

    def returnSlice(self):
        if self._data is None:
            raise RuntimeError("Slice has not yet been made")
        return self._data[:, 0].copy() if self._data.shape[1] == 1 else self._data


class BruteProjection:
    """The reference's ``Cvortrace.BruteProjection`` (src/bindings.cpp:240-257):
    per pixel, the nearest cell's fields summed (times dz), maximised or
    minimised over a regular grid of depth samples."""

    def __init__(self, npix, extent):
        self.npix = (int(npix[0]), int(npix[1]), int(npix[2]))
        self.extent = np.ascontiguousarray(extent, np.float64).reshape(6)
        self._data = None

    def makeProjection(self, cloud: _Cloud, reduction=L.REDUCE_SUM):
        mode = _REDUCTIONS[reduction] if isinstance(reduction, str) else int(reduction)
        n = self.npix[0] * self.npix[1]
        nf = int(cloud.info().nfields)
        out = np.empty((n, nf), np.float64)
        npx = (C.c_uint64 * 3)(*self.npix)
        L.check(cloud._lib.vt_brute_projection(cloud._h, npx, L.dptr(self.extent), mode,
                                               L.dptr(out)))
        self._data = out

    def returnProjection(self):
        if self._data is None:
            raise RuntimeError("Projection has not yet been made")
        return self._data[:, 0].copy() if self._data.shape[1] == 1 else self._data
