"""Exact-tie geometry at the segment level.

On lattices and quantised positions several generators are exactly
equidistant from a query, and the reference's answer depends on the order in
which its nanoflann tree meets them.  The fixtures (tests/golden/tie_walks.npz
and the lattice cases of small_walks.npz, made by tests/golden/make_golden.py
from the reference module) hold the reference's cell sequences, entry/exit
distances, integrals, k-NN lists and Slice/BruteProjection samples; every
walk kernel must reproduce them bit for bit (the device resolves exact ties
on the reference-order tree, tietree.cu)."""
import warnings

import numpy as np
import pytest

import vortrace_b200 as vt
from tests.conftest import make_cubic_lattice
from vortrace_b200 import vortrace as V

pytestmark = pytest.mark.gpu

KERNELS = ["plain", "batched", "batched_fp64", "thread_fp32"]


def cloud(pos, fields, bb, vol=None):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return vt.ProjectionCloud(pos, fields, boundbox=list(bb), vol=vol)


def check_segments(pc, c, out_key):
    vals, cid, s_enter, ds, off = pc.traced_projection(c["starts"], c["ends"],
                                                       return_midpoint=False, flatten=True)
    np.testing.assert_array_equal(off, c["offsets"])
    np.testing.assert_array_equal(cid, c["orig_ids"][c["cell_ids"]])
    np.testing.assert_array_equal(s_enter, c["s_enter"])
    np.testing.assert_array_equal(ds, c["s_exit"] - c["s_enter"])
    np.testing.assert_array_equal(np.asarray(vals).reshape(-1), c[out_key][:, 0])
    out = pc.projection(c["starts"], c["ends"])
    np.testing.assert_array_equal(out, c[out_key][:, 0])


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("case", ["lat5", "lat6", "lat8_f32"])
def test_tie_segments_bit_exact(tie_walks, case, kernel):
    c = tie_walks[case]
    pc = cloud(c["pos"], c["fields"], c["bb"], c["vol"])
    pc.kernel = kernel
    np.testing.assert_array_equal(pc.orig_ids, c["orig_ids"])
    check_segments(pc, c, "out")
    if case == "lat6":
        # the walks met exact ties and answered them on the reference-order tree
        assert pc.last_stats["ties"] > 0
        assert pc._cloud.info().tie_tree_nodes > 0


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("case", ["lattice", "lattice_f32"])
def test_small_walks_lattice_segments_bit_exact(small_walks, case, kernel):
    c = small_walks[case]
    pc = cloud(c["pos"], c["fields"], c["bb"], c.get("vol"))
    pc.kernel = kernel
    check_segments(pc, c, "integrate/out")


def test_tie_tree_built_ahead_and_dropped_on_rebuild(tie_walks):
    c = tie_walks["lat6"]
    pc = cloud(c["pos"], c["fields"], c["bb"], c["vol"])
    assert pc._cloud.info().tie_tree_nodes == 0
    L = pc._cloud._lib
    vt._lib.check(L.vt_cloud_build_tie_tree(pc._cloud._h))
    info = pc._cloud.info()
    assert info.tie_tree_nodes > 0 and 0 < info.tie_tree_depth <= 96
    check_segments(pc, c, "out")
    pc._cloud.buildTree()
    assert pc._cloud.info().tie_tree_nodes == 0
    check_segments(pc, c, "out")


@pytest.mark.parametrize("k", [1, 3, 8, 27])
def test_tie_knn_order(tie_walks, k):
    pos, f, vol, bb = make_cubic_lattice(6)
    pc = cloud(pos, f, bb, vol)
    c = tie_walks["knn"]
    ids, r2 = pc._cloud.knn(c["q"], k)
    np.testing.assert_array_equal(r2, c[f"k{k}_r2"])
    np.testing.assert_array_equal(pc.orig_ids[ids], c[f"k{k}_ids"])


def test_tie_slice_and_brute(tie_walks):
    pos, _, vol, bb = make_cubic_lattice(6)
    c = tie_walks["sample"]
    pc = cloud(pos, c["fields"], bb, vol)
    for i, depth in enumerate((2.5, 2.0)):
        out = pc.slice([-0.5, 5.5, -0.5, 5.5], 13, depth)
        np.testing.assert_array_equal(out.reshape(-1, 2), c[f"slice{i}"])
    for mode in ("sum", "max", "min"):
        bp = V.BruteProjection([13, 13, 13], [-0.5, 5.5, -0.5, 5.5, -0.5, 5.5])
        bp.makeProjection(pc._cloud, mode)
        np.testing.assert_array_equal(np.asarray(bp.returnProjection()).reshape(169, -1),
                                      c[f"brute_{mode}"])
