"""Regenerate the golden fixtures in tests/golden/ (run in a container that
has the reference checkout and oracle/_ref built; not needed at test time).

1. ``galaxy_interaction.npz``: the reference's own golden case
   (tests/test_vortrace.py:12-32 in the reference): the snapshot
   tests/test_data/galaxy_interaction.hdf5 (PartType0 Coordinates/Density as
   float32, Parameters.BoxSize) and the expected 128x128 projection
   tests/test_data/galaxy_interaction-proj.npy.  h5py is not installed, so
   the uncompressed, contiguous datasets are read at their byte offsets; the
   HDF5 signature, the sizes and the value ranges are checked, and the
   projection produced from them by the reference module must match the
   stored one at decimal=14 before anything is written.
2. ``small_walks.npz``: segment lists (cell ids, s_enter, s_exit, offsets) and
   integrate/max/min/volume outputs produced by the reference module
   (oracle/_ref) on small seeded clouds: uniform, Plummer-clustered, a cubic
   lattice with degenerate rays, and float32-quantised positions.
3. ``periodic_walks.npz``: the same for periodic clouds (loadPoints with
   periodic=True): a uniform cloud with rays across the domain faces, rays
   leaving the domain and rays whose two ends lie in one cell (the
   same-cell bisection), the reference's periodic k-NN (queryTree(q, k))
   for queries inside, near and outside the domain, and a cubic lattice
   (tests/test_periodic.py in the reference).
4. ``slice_brute.npz``: Slice.makeSlice and BruteProjection.makeProjection
   (sum, max, min) of the reference module on a seeded uniform cloud with two
   fields, and a slice of its periodic counterpart.
5. ``tie_walks.npz``: exact-tie geometry, where the answer depends on the
   order in which the reference's tree meets equidistant generators:
   segment lists of lattice clouds (the degenerate rays of the reference's
   tests/test_degenerate.py, axis rays at face/edge offsets, rays between
   half- and quarter-grid points, face diagonals, a float32-quantised
   lattice), queryTree(q, k) on the half and quarter grids, and Slice /
   BruteProjection samples on lattice faces and vertices.

Usage:  python tests/golden/make_golden.py [/path/to/reference [galaxy|small|periodic|slice|ties ...]]
"""
from __future__ import annotations

import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

SNAP_COORD_OFF, SNAP_DENS_OFF, SNAP_BOX_OFF = 19848, 1089052, 6800
SNAP_N = 7217


def read_snapshot(path):
    raw = open(path, "rb").read()
    if raw[:8] != b"\x89HDF\r\n\x1a\n":
        raise ValueError("not an HDF5 file")
    pos = np.frombuffer(raw, "<f4", SNAP_N * 3, SNAP_COORD_OFF).reshape(SNAP_N, 3).copy()
    dens = np.frombuffer(raw, "<f4", SNAP_N, SNAP_DENS_OFF).copy()
    box = float(np.frombuffer(raw, "<f8", 1, SNAP_BOX_OFF)[0])
    if not (np.isfinite(pos).all() and np.isfinite(dens).all()):
        raise ValueError("non-finite snapshot values")
    if not (0 < box < 1e5 and pos.min() >= 0 and pos.max() <= box and dens.min() > 0):
        raise ValueError("snapshot values out of range: wrong offsets?")
    return pos, dens, box


def galaxy(ref_root, mod):
    td = os.path.join(ref_root, "tests", "test_data")
    pos, dens, box = read_snapshot(os.path.join(td, "galaxy_interaction.hdf5"))
    proj = np.load(os.path.join(td, "galaxy_interaction-proj.npy"))
    # the reference test's call: ProjectionCloud(pos, dens, boundbox=[0,box]*3)
    # -> grid_projection(extent=[box/2-37.5, box/2+37.5], 128, [0, box], None)
    from vortrace_b200 import grid as G  # numpy-only module
    length = 75.0
    extent = [box / 2.0 - length / 2.0, box / 2.0 + length / 2.0]
    gs, ge = G.generate_projection_grid(extent, 128, [0.0, box], None)
    out, _, _ = O.reference_project(mod, pos, dens, [0.0, box] * 3, gs.reshape(-1, 3),
                                    ge.reshape(-1, 3))
    np.testing.assert_array_almost_equal(out.reshape(128, 128), proj, decimal=14)
    np.savez_compressed(os.path.join(HERE, "galaxy_interaction.npz"), pos=pos, dens=dens,
                        box_size=np.float64(box), proj=proj)
    print("galaxy_interaction.npz written; max|ref-golden| =",
          np.abs(out.reshape(128, 128) - proj).max())


def lattice(n=5):
    c = np.arange(n, dtype=np.float64)
    xx, yy, zz = np.meshgrid(c, c, c, indexing="ij")
    pos = np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()])
    return pos, [-0.5, n - 0.5] * 3


LATTICE_RAYS = [
    ([-0.1, -0.1, -0.1], [4.1, 4.1, 4.1]),     # body diagonal through vertices
    ([0.5, 0.2, -0.1], [0.5, 0.2, 4.1]),       # along a face
    ([0.5, 0.5, -0.1], [0.5, 0.5, 4.1]),       # along an edge
    ([0.1, 0.1, 0.1], [0.9, 0.9, 0.9]),        # through one vertex
    ([0.50001, 0.50001, -0.1], [0.50001, 0.50001, 4.1]),
    ([2.0, 2.0, -0.5], [2.0, 2.0, 4.5]),
    ([1.0, 2.0, -0.5], [1.0, 2.0, 4.5]),
    ([3.0, 3.0, -0.5], [3.0, 3.0, 4.5]),
    ([0.5, 0.5, 0.5], [0.6, 0.6, 0.6]),        # same cell
    ([2.0, 2.0, -0.1], [2.0, 2.0, 4.1]),
    ([4.1, 0.2, 3.3], [-0.2, 3.7, 0.4]),
]


def small_walks(mod):
    rng = np.random.default_rng(20240601)
    cases = {}

    # uniform cloud, random rays, nf=2 (integrate/max/min)
    n = 1500
    pos = rng.uniform(0, 10, (n, 3))
    f = np.column_stack([rng.lognormal(0, 1, n), rng.uniform(0, 1, n)])
    st = rng.uniform(0, 10, (120, 3))
    en = rng.uniform(0, 10, (120, 3))
    cases["uniform"] = (pos, f, [0, 10] * 3, None, st, en, ["integrate", "max", "min"])

    # Plummer-clustered cloud, z-grid rays
    m = 2500
    a = 0.5
    u = rng.uniform(1e-6, 1, m)
    r = a / np.sqrt(u ** (-2.0 / 3.0) - 1)
    r = np.minimum(r, 4.0)
    v = rng.normal(size=(m, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    pos = 5.0 + r[:, None] * v
    pos = np.vstack([pos, rng.uniform(0, 10, (250, 3))])
    rho = (1 + np.sum((pos - 5) ** 2, axis=1) / a ** 2) ** -2.5
    xs = np.linspace(4.0, 6.0, 10)
    gx, gy = np.meshgrid(xs, xs, indexing="ij")
    st = np.column_stack([gx.ravel(), gy.ravel(), np.zeros(gx.size)])
    en = st.copy()
    en[:, 2] = 10.0
    cases["plummer"] = (pos, rho, [0, 10] * 3, None, st, en, ["integrate"])

    # volume rendering on a random cloud (RGBA in range)
    n = 1200
    pos = rng.uniform(0, 10, (n, 3))
    rgba = np.column_stack([rng.uniform(0, 1, (n, 3)), rng.uniform(0, 0.3, n)])
    st = rng.uniform(0, 10, (100, 3))
    en = rng.uniform(0, 10, (100, 3))
    cases["volume"] = (pos, rgba, [0, 10] * 3, None, st, en, ["volume"])

    # cubic lattice, degenerate rays (exact ties everywhere)
    pos, bb = lattice(5)
    st = np.array([c[0] for c in LATTICE_RAYS], float)
    en = np.array([c[1] for c in LATTICE_RAYS], float)
    cases["lattice"] = (pos, np.ones(len(pos)), bb, np.ones(len(pos)), st, en, ["integrate"])

    # float32-quantised lattice (tests/test_degenerate.py:172-194 in the reference)
    pos, bb = lattice(10)
    off = np.array([500.0, 500.0, 500.1])
    p32 = (pos + off).astype(np.float32)
    p32 -= off.astype(np.float32)
    pos = p32.astype(np.float64)
    st = np.array([[-0.1, -0.1, -0.1], [0.3, -0.1, 0.2], [9.1, 0.0, 4.5]])
    en = np.array([[9.1, 9.1, 9.1], [8.7, 9.2, 9.0], [0.0, 9.1, 4.5]])
    cases["lattice_f32"] = (pos, np.ones(len(pos)), bb, np.ones(len(pos)), st, en, ["integrate"])

    blob = {}
    for name, (pos, f, bb, vol, st, en, modes) in cases.items():
        blob[f"{name}/pos"] = pos
        blob[f"{name}/fields"] = np.asarray(f, np.float64)
        blob[f"{name}/bb"] = np.asarray(bb, np.float64)
        if vol is not None:
            blob[f"{name}/vol"] = np.asarray(vol, np.float64)
        blob[f"{name}/starts"] = st
        blob[f"{name}/ends"] = en
        blob[f"{name}/modes"] = np.array(modes)
        # the segment list does not depend on the reduction: store it once
        for i, mode in enumerate(modes):
            out, segs, oid = O.reference_project(mod, pos, f, bb, st, en, mode=mode, vol=vol,
                                                 detailed=True)
            cid, se, sx, off = segs
            blob[f"{name}/{mode}/out"] = np.asarray(out).reshape(len(st), -1)
            if i == 0:
                blob[f"{name}/cell_ids"] = np.asarray(cid, np.int64)
                blob[f"{name}/s_enter"] = np.asarray(se)
                blob[f"{name}/s_exit"] = np.asarray(sx)
                blob[f"{name}/offsets"] = np.asarray(off, np.int64)
                blob[f"{name}/orig_ids"] = np.asarray(oid, np.int64)
            else:
                assert np.array_equal(blob[f"{name}/cell_ids"], cid)
        print(name, "segments:", len(cid))
    np.savez_compressed(os.path.join(HERE, "small_walks.npz"), **blob)
    print("small_walks.npz written")


def periodic_walks(mod):
    rng = np.random.default_rng(20240707)
    blob = {}
    # uniform cloud in [0, 10)^3
    n = 2000
    pos = rng.uniform(0, 10, (n, 3))
    rho = rng.lognormal(0, 1, n)
    st = [rng.uniform(0, 10, (60, 3))]
    en = [rng.uniform(0, 10, (60, 3))]
    for ax in range(3):  # rays hugging the faces normal to each axis
        a = rng.uniform(0, 10, (8, 3))
        b = rng.uniform(0, 10, (8, 3))
        a[:, ax] = rng.uniform(0.005, 0.05, 8)
        b[:, ax] = rng.uniform(9.95, 9.995, 8)
        st.append(a)
        en.append(b)
    # rays whose ends sit next to one generator and next to its periodic
    # image: both ends in one cell, so the walk bisects for another cell
    for ax in range(3):
        order = np.argsort(pos[:, ax])[:4]
        for i in order:
            a = pos[i].copy()
            b = pos[i].copy()
            a[ax] += 0.01
            b[ax] += 10.0 - 0.01
            st.append(a[None])
            en.append(b[None])
    # rays leaving the domain
    a = rng.uniform(0, 10, (8, 3))
    b = rng.uniform(0, 10, (8, 3))
    a[:, 0] = -1.5
    b[:, 0] = 11.5
    st.append(a)
    en.append(b)
    st = np.vstack(st)
    en = np.vstack(en)
    out, segs, oid = O.reference_project(mod, pos, rho, [0, 10] * 3, st, en, detailed=True,
                                         periodic=True)
    cid, se, sx, off = segs
    blob.update({"uniform/pos": pos, "uniform/fields": rho, "uniform/bb": np.array([0, 10.0] * 3),
                 "uniform/starts": st, "uniform/ends": en,
                 "uniform/out": np.asarray(out).reshape(len(st), -1),
                 "uniform/cell_ids": np.asarray(cid, np.int64), "uniform/s_enter": np.asarray(se),
                 "uniform/s_exit": np.asarray(sx), "uniform/offsets": np.asarray(off, np.int64),
                 "uniform/orig_ids": np.asarray(oid, np.int64)})
    print("periodic uniform segments:", len(cid))
    pc = O.reference_cloud(mod, pos, rho, [0, 10] * 3, periodic=True)
    q = np.vstack([rng.uniform(-0.5, 10.5, (240, 3)),
                   np.array([[x, y, z] for x in (0.01, 9.99) for y in (0.02, 9.98)
                             for z in (0.03, 9.97)])])
    blob["uniform/knn_q"] = q
    for k in (1, 3, 10):
        ids = np.zeros((len(q), k), np.int64)
        r2 = np.zeros((len(q), k))
        for i, qq in enumerate(q):
            a, b = pc.queryTree(qq, k)
            ids[i], r2[i] = a, b
        blob[f"uniform/knn{k}_ids"] = ids
        blob[f"uniform/knn{k}_r2"] = r2
    # cubic lattice, box 5, spacing 0.5 (tests/test_periodic.py:10-18)
    c = np.arange(0.25, 5.0, 0.5)
    xx, yy, zz = np.meshgrid(c, c, c, indexing="ij")
    lpos = np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()])
    lst = np.array([[0.01, 2.5, 2.5], [0.5, 2.5, 2.5], [0.3, 0.4, 0.2], [4.9, 0.1, 2.6]])
    len_ = np.array([[4.99, 2.5, 2.5], [4.5, 2.5, 2.5], [4.6, 4.7, 4.9], [0.2, 4.8, 2.4]])
    lout, lsegs, loid = O.reference_project(mod, lpos, np.full(len(lpos), 2.5), [0, 5.0] * 3,
                                            lst, len_, detailed=True, periodic=True)
    blob.update({"lattice/pos": lpos, "lattice/bb": np.array([0, 5.0] * 3), "lattice/starts": lst,
                 "lattice/ends": len_, "lattice/out": np.asarray(lout).reshape(len(lst), -1),
                 "lattice/offsets": np.asarray(lsegs[3], np.int64)})
    np.savez_compressed(os.path.join(HERE, "periodic_walks.npz"), **blob)
    print("periodic_walks.npz written")


def slice_brute(mod):
    rng = np.random.default_rng(20240808)
    n = 3000
    pos = rng.uniform(0, 10, (n, 3))
    f = np.column_stack([rng.lognormal(0, 1, n), rng.uniform(0, 1, n)])
    blob = {"pos": pos, "fields": f, "bb": np.array([0, 10.0] * 3)}
    slices = [((37, 23), [0.5, 9.5, 1.0, 9.0], 3.3), ((16, 16), [0.0, 10.0, 0.0, 10.0], 0.0),
              ((9, 31), [2.0, 8.0, 2.0, 8.0], 10.0)]
    for periodic in (False, True):
        pc = O.reference_cloud(mod, pos, f, [0, 10] * 3, periodic=periodic)
        tag = "periodic" if periodic else "open"
        for i, (npix, ext, depth) in enumerate(slices):
            sl = mod.Slice(list(npix), list(ext), depth)
            sl.makeSlice(pc)
            blob[f"{tag}/slice{i}"] = np.asarray(sl.returnSlice()).reshape(npix[0] * npix[1], -1)
        if not periodic:
            for mode in ("Sum", "Max", "Min"):
                bp = mod.BruteProjection([12, 10, 25], [1.0, 9.0, 1.0, 9.0, 0.0, 10.0])
                bp.makeProjection(pc, getattr(mod.ReductionMode, mode))
                blob[f"open/brute_{mode.lower()}"] = np.asarray(bp.returnProjection()).reshape(
                    120, -1)
    for i, (npix, ext, depth) in enumerate(slices):
        blob[f"slice{i}/npix"] = np.array(npix)
        blob[f"slice{i}/extent"] = np.array(ext)
        blob[f"slice{i}/depth"] = np.array(depth)
    np.savez_compressed(os.path.join(HERE, "slice_brute.npz"), **blob)
    print("slice_brute.npz written")


# the five degenerate rays of the reference's tests/test_degenerate.py on the
# 5x5x5 lattice
DEGENERATE_RAYS = [
    ([-0.1] * 3, [4.1] * 3),
    ([0.5, 0.2, -0.1], [0.5, 0.2, 4.1]),
    ([0.5, 0.5, -0.1], [0.5, 0.5, 4.1]),
    ([0.1] * 3, [0.9] * 3),
    ([0.50001, 0.50001, -0.1], [0.50001, 0.50001, 4.1]),
]


def _tie_rays(rng, n):
    """Rays on a 6x6x6 lattice whose walks meet exact distance ties: rays
    along the axes at face, edge and interior offsets; rays between random
    points of the half-integer grid (both ends on cell faces, edges or
    vertices); rays between quarter-grid points; face diagonals."""
    st, en = [], []
    offs = [0.5, 1.0, 1.5, 2.25, 3.0]
    for ax in range(3):
        o = [d for d in range(3) if d != ax]
        for a in offs:
            for b in offs:
                p = np.zeros(3)
                q = np.zeros(3)
                p[o[0]], p[o[1]] = a, b
                q[o[0]], q[o[1]] = a, b
                p[ax], q[ax] = -0.5, n - 0.5
                st.append(p)
                en.append(q)
    half = np.arange(-0.5, n, 0.5)
    for _ in range(100):
        p, q = rng.choice(half, 3), rng.choice(half, 3)
        if np.array_equal(p, q):
            q[0] += 0.5
        st.append(p)
        en.append(q)
    quarter = np.arange(-0.25, n - 0.5, 0.25)
    for _ in range(60):
        p, q = rng.choice(quarter, 3), rng.choice(quarter, 3)
        if np.array_equal(p, q):
            q[1] += 0.25
        st.append(p)
        en.append(q)
    for _ in range(20):
        ax = rng.integers(3)
        c = rng.choice(half)
        p = rng.uniform(-0.4, n - 0.6, 3)
        p[ax] = c
        q = p.copy()
        o = [d for d in range(3) if d != ax]
        p[o[0]], p[o[1]] = -0.5, -0.5
        q[o[0]], q[o[1]] = n - 0.5, n - 0.5
        st.append(p)
        en.append(q)
    return np.array(st), np.array(en)


def tie_walks(mod):
    """Exact-tie geometry through the reference module: segment lists of
    lattice clouds (the degenerate rays of the reference's tests, axis rays,
    half- and quarter-grid rays, face diagonals, a float32-quantised
    lattice), the reference's k-NN order of exactly tied generators, and
    Slice / BruteProjection samples on lattice faces and vertices."""
    rng = np.random.default_rng(20241111)
    blob = {}
    cases = {}
    pos, bb = lattice(5)
    cases["lat5"] = (pos, bb, np.array([r[0] for r in DEGENERATE_RAYS + LATTICE_RAYS], float),
                     np.array([r[1] for r in DEGENERATE_RAYS + LATTICE_RAYS], float))
    pos, bb = lattice(6)
    st, en = _tie_rays(rng, 6)
    cases["lat6"] = (pos, bb, st, en)
    pos, bb = lattice(8)
    off = np.array([500.0, 500.0, 500.1])
    p32 = (pos + off).astype(np.float32)
    p32 -= off.astype(np.float32)
    half = np.arange(-0.5, 8, 0.5)
    st = np.array([rng.choice(half, 3) for _ in range(40)])
    en = np.array([rng.choice(half, 3) for _ in range(40)])
    en[np.all(st == en, axis=1), 0] += 0.5
    cases["lat8_f32"] = (p32.astype(np.float64), bb, st, en)
    for name, (pos, bb, st, en) in cases.items():
        f = 1.0 + 0.001 * np.arange(len(pos))   # distinct per cell
        keep = []
        for i in range(len(st)):   # rays the reference walks without error
            try:
                O.reference_project(mod, pos, f, bb, st[i:i + 1], en[i:i + 1],
                                    vol=np.ones(len(pos)))
                keep.append(i)
            except RuntimeError as e:
                print(name, "ray", i, "skipped:", e)
        st, en = st[keep], en[keep]
        out, segs, oid = O.reference_project(mod, pos, f, bb, st, en, vol=np.ones(len(pos)),
                                             detailed=True)
        cid, se, sx, so = segs
        blob.update({f"{name}/pos": pos, f"{name}/fields": f, f"{name}/bb": np.asarray(bb, float),
                     f"{name}/vol": np.ones(len(pos)), f"{name}/starts": st, f"{name}/ends": en,
                     f"{name}/out": np.asarray(out).reshape(len(st), -1),
                     f"{name}/cell_ids": np.asarray(cid, np.int64),
                     f"{name}/s_enter": np.asarray(se), f"{name}/s_exit": np.asarray(sx),
                     f"{name}/offsets": np.asarray(so, np.int64),
                     f"{name}/orig_ids": np.asarray(oid, np.int64)})
        print(name, len(st), "rays,", len(cid), "segments")
    # k-NN order of tied generators (queries on the half and quarter grids)
    pos, bb = lattice(6)
    pc = O.reference_cloud(mod, pos, np.ones(len(pos)), bb, vol=np.ones(len(pos)))
    q = np.vstack([np.array([rng.choice(np.arange(-0.5, 6, 0.5), 3) for _ in range(200)]),
                   np.array([rng.choice(np.arange(-0.25, 5.5, 0.25), 3) for _ in range(200)])])
    blob["knn/q"] = q
    for k in (1, 3, 8, 27):
        ids = np.zeros((len(q), k), np.int64)
        r2 = np.zeros((len(q), k))
        for i, qq in enumerate(q):
            a, b = pc.queryTree(qq, k)
            ids[i], r2[i] = a, b
        blob[f"knn/k{k}_ids"] = ids
        blob[f"knn/k{k}_r2"] = r2
    # Slice and BruteProjection sampling lattice faces, edges and vertices
    f = np.column_stack([1.0 + np.arange(len(pos)), np.arange(len(pos))[::-1] * 0.5])
    pc = O.reference_cloud(mod, pos, f, bb, vol=np.ones(len(pos)))
    blob["sample/fields"] = f
    for i, depth in enumerate((2.5, 2.0)):
        sl = mod.Slice([13, 13], [-0.5, 5.5, -0.5, 5.5], depth)
        sl.makeSlice(pc)
        blob[f"sample/slice{i}"] = np.asarray(sl.returnSlice()).reshape(169, -1)
    for mode in ("Sum", "Max", "Min"):
        bp = mod.BruteProjection([13, 13, 13], [-0.5, 5.5, -0.5, 5.5, -0.5, 5.5])
        bp.makeProjection(pc, getattr(mod.ReductionMode, mode))
        blob[f"sample/brute_{mode.lower()}"] = np.asarray(bp.returnProjection()).reshape(169, -1)
    np.savez_compressed(os.path.join(HERE, "tie_walks.npz"), **blob)
    print("tie_walks.npz written")


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    mod = O.load_reference_module()
    if mod is None:
        raise SystemExit("oracle/_ref/Cvortrace not built: run oracle/build_ref.sh first")
    warnings.simplefilter("ignore")
    which = sys.argv[2:] or ["galaxy", "small", "periodic", "slice", "ties"]
    if "galaxy" in which:
        galaxy(ref_root, mod)
    if "small" in which:
        small_walks(mod)
    if "periodic" in which:
        periodic_walks(mod)
    if "slice" in which:
        slice_brute(mod)
    if "ties" in which:
        tie_walks(mod)


if __name__ == "__main__":
    main()
