"""Ray-grid generation for :meth:`ProjectionCloud.grid_projection`.

Same behaviour as the reference's ``vortrace/grid.py`` (pixel-centre grid,
``bounds`` along the pre-rotation z axis, optional Tait-Bryan rotation about
``center``, named Cartesian projections).  The arithmetic steps are kept the
same as the reference's (``linspace`` over pixel centres, ``meshgrid`` with
``indexing='ij'``, ``grid @ R.T``) because the rays must be bit-identical for
the projections to be.

Reference: vortrace/grid.py:13-23 (named projections), :35-44 (base grid),
:86-97 (rotation matrix), :100-192 (projection grid).
"""
from __future__ import annotations

import numpy as np

# (yaw, pitch, roll, handedness) per named projection; vortrace/grid.py:13-23
PROJECTIONS = {
    "xy": (0.0, 0.0, 0.0, 1),
    "yz": (np.pi / 2.0, 0.0, np.pi / 2.0, 1),
    "zx": (3.0 * np.pi / 2.0, 3.0 * np.pi / 2.0, 0.0, 1),
    "yx": (np.pi / 2.0, 0.0, np.pi, -1),
    "xz": (0.0, 0.0, np.pi / 2.0, -1),
    "zy": (0.0, 3.0 * np.pi / 2.0, 0.0, -1),
}


def projection_angles(proj: str):
    """Return ``(yaw, pitch, roll, hand)`` for a named projection."""
    try:
        return PROJECTIONS[proj]
    except KeyError:
        raise ValueError(f"Unknown projection {proj!r}. Valid options: {list(PROJECTIONS)}")


def _as_extent(extent):
    ext = np.array(extent)
    n = ext.ravel().size
    if n == 2:
        return np.array([ext, ext])
    if n == 4:
        return ext
    raise ValueError("extent must be either (2,2) or (2,) array")


def _as_nres(nres):
    if isinstance(nres, (int, np.integer)):
        return (int(nres), int(nres))
    return tuple(int(v) for v in nres)


def generate_base_grid(extent, nres) -> np.ndarray:
    """(nx, ny, 3) grid of pixel centres in the x-y plane (z = 0)."""
    ext = _as_extent(extent)
    nx, ny = _as_nres(nres)
    dx = (ext[0][1] - ext[0][0]) / nx
    dy = (ext[1][1] - ext[1][0]) / ny
    xs = np.linspace(ext[0][0] + 0.5 * dx, ext[0][1] - 0.5 * dx, nx)
    ys = np.linspace(ext[1][0] + 0.5 * dy, ext[1][1] - 0.5 * dy, ny)
    gx, gy = np.meshgrid(xs, ys, indexing="ij")
    grid = np.zeros((nx, ny, 3))
    grid[..., 0] = gx
    grid[..., 1] = gy
    return grid


def rotation_matrix(yaw: float, pitch: float, roll: float) -> np.ndarray:
    """Tait-Bryan rotation matrix R = Rz(yaw) Ry(pitch) Rx(roll)."""
    ca, sa = np.cos(yaw), np.sin(yaw)
    cb, sb = np.cos(pitch), np.sin(pitch)
    cg, sg = np.cos(roll), np.sin(roll)
    return np.array([
        [ca * cb, ca * sb * sg - sa * cg, ca * sb * cg + sa * sg],
        [sa * cb, sa * sb * sg + ca * cg, sa * sb * cg - ca * sg],
        [-sb, cb * sg, cb * cg],
    ])


def generate_projection_grid(extent, nres, bounds, center, *, proj=None, yaw=0.0, pitch=0.0,
                             roll=0.0):
    """Start and end points, each (nx, ny, 3), of a (rotated) projection grid.

    The base grid spans ``extent`` in x-y; starts sit at z=bounds[0] and ends
    at z=bounds[1].  With ``center`` given, both are rotated about it by
    ``rotation_matrix(yaw, pitch, roll)`` (or the angles of ``proj``).  A
    named projection whose handedness disagrees with the sign of
    ``bounds[1]-bounds[0]`` gets its bounds flipped.
    """
    grid_start = generate_base_grid(extent, nres)
    grid_end = np.copy(grid_start)
    if proj is not None:
        yaw, pitch, roll, hand = projection_angles(proj)
    else:
        hand = np.sign(bounds[1] - bounds[0])
    if hand != np.sign(bounds[1] - bounds[0]):
        bounds = np.flip(bounds)
    grid_start[..., 2] = bounds[0]
    grid_end[..., 2] = bounds[1]
    if center is not None:
        grid_start -= center
        grid_end -= center
        rot = rotation_matrix(yaw, pitch, roll)
        grid_start = np.dot(grid_start, rot.T)
        grid_end = np.dot(grid_end, rot.T)
        grid_start += center
        grid_end += center
    return grid_start, grid_end
