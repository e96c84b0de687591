"""Saving and loading projection grids and clouds (vortrace/io.py:1-241 in
the reference): the same functions, file layouts and key names, so files move
between the two libraries.

* ``save_grid`` / ``load_grid``: ``data``, optional ``extent`` and a JSON
  ``_metadata`` string (npz), or a ``data`` dataset, an ``extent`` dataset and
  a ``metadata`` attribute (hdf5).
* ``save_cloud`` / ``load_cloud``: ``pos``, ``fields``, ``boundbox``,
  ``periodic``, optional ``vol`` and the tree blob in ``_kdtree``.  The blob
  written here is this library's device tree; a file holding a blob of
  another kind (the reference's nanoflann index) loads with a device rebuild.

The format follows the file extension on load (.hdf5 / .h5: hdf5, else npz);
hdf5 needs h5py.
"""
from __future__ import annotations

import json

import numpy as np


def _h5py():
    try:
        import h5py
    except ImportError as exc:
        raise ImportError("h5py is required for HDF5 I/O. "
                          "Install it with:  pip install h5py") from exc
    return h5py


def _fmt_of(filename) -> str:
    return "hdf5" if str(filename).endswith((".hdf5", ".h5")) else "npz"


def _check_fmt(fmt):
    if fmt not in ("npz", "hdf5"):
        raise ValueError(f"Unknown format: {fmt!r}. Use 'npz' or 'hdf5'.")


def save_grid(filename, data, *, extent=None, metadata=None, fmt: str = "npz") -> None:
    """Save a 2D projection array with an optional extent and metadata."""
    _check_fmt(fmt)
    data = np.asarray(data)
    if fmt == "npz":
        items = {"data": data}
        if extent is not None:
            items["extent"] = np.asarray(extent)
        if metadata is not None:
            items["_metadata"] = np.array(json.dumps(metadata))
        np.savez(filename, **items)
        return
    with _h5py().File(filename, "w") as f:
        f.create_dataset("data", data=data)
        if extent is not None:
            f.create_dataset("extent", data=np.asarray(extent))
        if metadata is not None:
            f.attrs["metadata"] = json.dumps(metadata)


def load_grid(filename):
    """(data, metadata) of a file written by :func:`save_grid`; the extent,
    when stored, is metadata['extent']."""
    if _fmt_of(filename) == "npz":
        with np.load(filename, allow_pickle=False) as z:
            data = z["data"]
            meta = json.loads(str(z["_metadata"])) if "_metadata" in z else {}
            if "extent" in z:
                meta["extent"] = z["extent"]
        return data, meta
    with _h5py().File(filename, "r") as f:
        data = f["data"][:]
        meta = json.loads(f.attrs["metadata"]) if "metadata" in f.attrs else {}
        if "extent" in f:
            meta["extent"] = f["extent"][:]
    return data, meta


def save_cloud(filename, cloud, *, fmt: str = "npz", save_tree: bool = True) -> None:
    """Save a ProjectionCloud: its input arrays and, by default, its tree."""
    _check_fmt(fmt)
    pos = np.asarray(cloud.pos_orig)
    fields = np.asarray(cloud.fields_orig)
    boundbox = np.asarray(cloud.boundbox)
    periodic = bool(getattr(cloud, "periodic", False))
    blob = cloud.save_tree_bytes() if save_tree else None
    if fmt == "npz":
        items = {"pos": pos, "fields": fields, "boundbox": boundbox,
                 "periodic": np.bool_(periodic)}
        if cloud.vol_orig is not None:
            items["vol"] = np.asarray(cloud.vol_orig)
        if blob is not None:
            items["_kdtree"] = np.void(blob)
        np.savez(filename, **items)
        return
    with _h5py().File(filename, "w") as f:
        f.create_dataset("pos", data=pos)
        f.create_dataset("fields", data=fields)
        f.attrs["boundbox"] = boundbox
        f.attrs["periodic"] = periodic
        if cloud.vol_orig is not None:
            f.create_dataset("vol", data=np.asarray(cloud.vol_orig))
        if blob is not None:
            f.create_dataset("_kdtree", data=np.void(blob))


def load_cloud(filename):
    """A ready ProjectionCloud from a file written by :func:`save_cloud` (of
    either library); the saved tree is restored when it is this library's."""
    from .vortrace import ProjectionCloud
    blob = None
    if _fmt_of(filename) == "npz":
        with np.load(filename, allow_pickle=True) as z:
            pos, fields, boundbox = z["pos"], z["fields"], z["boundbox"]
            vol = z["vol"] if "vol" in z else None
            periodic = bool(z["periodic"]) if "periodic" in z else False
            if "_kdtree" in z:
                blob = bytes(z["_kdtree"])
    else:
        with _h5py().File(filename, "r") as f:
            pos, fields = f["pos"][:], f["fields"][:]
            boundbox = f.attrs["boundbox"]
            vol = f["vol"][:] if "vol" in f else None
            periodic = bool(f.attrs.get("periodic", False))
            if "_kdtree" in f:
                blob = bytes(f["_kdtree"][()])
    if blob is None:
        return ProjectionCloud(pos, fields, boundbox=list(boundbox), vol=vol, periodic=periodic)
    pc = ProjectionCloud(pos, fields, boundbox=list(boundbox), vol=vol, periodic=periodic,
                         _skip_build_tree=True)
    pc.load_tree_bytes(blob)
    return pc
