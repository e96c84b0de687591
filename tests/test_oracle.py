"""The CPU oracle (oracle/vt_oracle.c) pinned against the reference's golden
projection, the fixtures produced by the reference module, the reference's
C++ known-answer tests and, where it is built, the reference module itself."""
import math
import warnings

import numpy as np
import pytest

from oracle import oracle as O
from vortrace_b200 import grid as gr


def oracle_for(pos, fields, bb, vol=None):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        lp = O.load_points(pos, fields, bb, vol)
    return lp, O.OracleTree(lp["pts"], lp["fields"], lp["valid_rgba"])


def test_golden_projection(galaxy):
    # tests/test_vortrace.py:31-48 of the reference
    box = galaxy["box_size"]
    lp, t = oracle_for(galaxy["pos"], galaxy["dens"], [0.0, box] * 3)
    ext = [box / 2.0 - 37.5, box / 2.0 + 37.5]
    s, e = gr.generate_projection_grid(ext, 128, [0.0, box], None)
    out = t.project(s.reshape(-1, 3), e.reshape(-1, 3)).reshape(128, 128)
    np.testing.assert_array_almost_equal(out, galaxy["proj"], decimal=14)


@pytest.mark.parametrize("case", ["uniform", "plummer", "volume", "lattice", "lattice_f32"])
def test_reference_fixtures_bit_exact(small_walks, case):
    c = small_walks[case]
    lp, t = oracle_for(c["pos"], c["fields"], c["bb"], c.get("vol"))
    np.testing.assert_array_equal(lp["orig_ids"], c["orig_ids"])
    for mode in c["modes"]:
        out, (cid, se, sx, off) = t.project(c["starts"], c["ends"], str(mode), segments=True)
        np.testing.assert_array_equal(off, c["offsets"])
        np.testing.assert_array_equal(cid, c["cell_ids"])
        np.testing.assert_array_equal(se, c["s_enter"])
        np.testing.assert_array_equal(sx, c["s_exit"])
        np.testing.assert_array_equal(out, c[f"{mode}/out"])


@pytest.mark.parametrize("case", ["lat5", "lat6", "lat8_f32"])
def test_tie_fixtures_bit_exact(tie_walks, case):
    # exact-tie geometry: the walk's 1-NN answers depend on nanoflann's order
    c = tie_walks[case]
    lp, t = oracle_for(c["pos"], c["fields"], c["bb"], c["vol"])
    np.testing.assert_array_equal(lp["orig_ids"], c["orig_ids"])
    out, (cid, se, sx, off) = t.project(c["starts"], c["ends"], "integrate", segments=True)
    np.testing.assert_array_equal(off, c["offsets"])
    np.testing.assert_array_equal(cid, c["cell_ids"])
    np.testing.assert_array_equal(se, c["s_enter"])
    np.testing.assert_array_equal(sx, c["s_exit"])
    np.testing.assert_array_equal(out, c["out"])


@pytest.mark.parametrize("k", [1, 3, 8, 27])
def test_tie_knn_order(tie_walks, k):
    from tests.conftest import make_cubic_lattice
    pos, f, vol, bb = make_cubic_lattice(6)
    lp, t = oracle_for(pos, f, bb, vol)
    c = tie_walks["knn"]
    ids, r2 = t.knn(c["q"], k)
    np.testing.assert_array_equal(r2, c[f"k{k}_r2"])
    np.testing.assert_array_equal(lp["orig_ids"][ids], c[f"k{k}_ids"])


def test_split_point_known_answers():
    # tests/test_cpp.cpp:19-41 of the reference
    assert O.split_point_distance([0, 0, 0], [0, 0, 1], [0, 0, 0], [0, 0, 1]) == pytest.approx(0.5)
    assert O.split_point_distance([0, 0, 0], [0, 0, 2], [0, 0, 1], [0, 0, 3]) == pytest.approx(2.0)
    assert O.split_point_distance([0, 0, 0], [1, 1, 1], [0.25] * 3, [0.75] * 3) == pytest.approx(
        0.5 * math.sqrt(3.0))
    # bisector parallel to the ray: sentinel
    assert O.split_point_distance([0, 0, 0], [0, 0, 1], [1, 0, 0], [-1, 0, 0]) > 1e300


def test_nearest_neighbour_four_points():
    # tests/test_cpp.cpp:45-73
    pos = np.array([[0.25, 0.25, 0.5], [0.75, 0.25, 0.5], [0.25, 0.75, 0.5], [0.75, 0.75, 0.5]])
    t = O.OracleTree(pos)
    ids, _ = t.knn(np.array([[0.3, 0.3, 0.5], [0.7, 0.7, 0.5]]), 1)
    assert ids[:, 0].tolist() == [0, 3]


def test_filtering_and_single_cell():
    # tests/test_cpp.cpp:92-134
    lp = O.load_points(np.array([[0.5] * 3, [0.9] * 3, [10.0] * 3]), np.ones(3), [0, 1] * 3)
    assert len(lp["orig_ids"]) == 2
    t = O.OracleTree(np.array([[0.5, 0.5, 0.5]]))
    out = t.project(np.array([[0.5, 0.5, 0.0]]), np.array([[0.5, 0.5, 1.0]]))
    assert out[0, 0] == pytest.approx(1.0)


def test_volume_closed_form():
    # tests/test_volume_render.py:30-47: uniform RGBA -> C (1 - exp(-alpha L))
    rng = np.random.default_rng(42)
    pos = rng.random((500, 3)) * 100.0
    rgba = [0.8, 0.4, 0.2, 0.01]
    lp, t = oracle_for(pos, np.tile(rgba, (500, 1)), [0.0, 100.0] * 3)
    out, (_, se, sx, _) = t.project(np.array([[50, 50, 0.1]]), np.array([[50, 50, 99.9]]),
                                    "volume", segments=True)
    L = np.sum(sx - se)
    np.testing.assert_allclose(out[0], np.array(rgba[:3]) * (1 - np.exp(-0.01 * L)), rtol=1e-10)


def test_lattice_diagonal_length():
    # tests/test_degenerate.py:38-46: a ray through lattice vertices
    from tests.conftest import make_cubic_lattice
    pos, f, vol, bb = make_cubic_lattice(5)
    lp, t = oracle_for(pos, f, bb, vol)
    out = t.project(np.array([[-0.1] * 3]), np.array([[4.1] * 3]))
    assert out[0, 0] == pytest.approx(np.linalg.norm([4.2] * 3), rel=1e-6)


# ------------------------------------------------------- vs the reference
def _need(ref_module):
    if ref_module is None:
        pytest.skip("reference module not built (oracle/build_ref.sh)")


def test_knn_matches_reference(ref_module):
    _need(ref_module)
    rng = np.random.default_rng(3)
    pos = rng.uniform(0, 100, (20000, 3))
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = ref_module.PointCloud()
        pc.loadPoints(pos, np.ones(len(pos)), [0, 100] * 3)
    pc.buildTree()
    lp, t = oracle_for(pos, np.ones(len(pos)), [0, 100] * 3)
    q = rng.uniform(-10, 110, (500, 3))
    for k in (1, 3, 100):
        ids, r2 = t.knn(q, k)
        for i in range(len(q)):
            rid, rr2 = pc.queryTree(q[i], k)
            assert np.array_equal(np.asarray(rid, np.int64), ids[i])
            assert np.array_equal(np.asarray(rr2), r2[i])


@pytest.mark.parametrize("kind", ["uniform", "lattice"])
def test_walk_matches_reference(ref_module, kind):
    _need(ref_module)
    rng = np.random.default_rng(11)
    if kind == "uniform":
        pos = rng.uniform(0, 100, (30000, 3))
        f = rng.lognormal(0, 1, len(pos))
        bb, vol = [0, 100] * 3, None
        st = rng.uniform(0, 100, (2000, 3))
        en = rng.uniform(0, 100, (2000, 3))
    else:
        from tests.conftest import make_cubic_lattice
        pos, f, vol, bb = make_cubic_lattice(6)
        st = rng.uniform(-0.4, 5.4, (400, 3)).round(1)
        en = rng.uniform(-0.4, 5.4, (400, 3)).round(1)
        keep = np.linalg.norm(en - st, axis=1) > 0
        st, en = st[keep], en[keep]
    out, seg, oid = O.reference_project(ref_module, pos, f, bb, st, en, vol=vol, detailed=True)
    lp, t = oracle_for(pos, f, bb, vol)
    o2, seg2 = t.project(st, en, segments=True)
    np.testing.assert_array_equal(oid, lp["orig_ids"])
    for a, b in zip(seg, seg2):
        np.testing.assert_array_equal(np.asarray(a), b)
    np.testing.assert_array_equal(np.asarray(out).reshape(o2.shape), o2)


def test_load_points_matches_reference(ref_module):
    _need(ref_module)
    rng = np.random.default_rng(5)
    pos = rng.uniform(-20, 120, (3000, 3))
    vol = rng.uniform(0.1, 30.0, 3000)
    for v in (None, vol):
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            pc = ref_module.PointCloud()
            if v is None:
                pc.loadPoints(pos, np.ones(3000), [10, 90, 0, 100, 20, 60])
            else:
                pc.loadPoints(pos, np.ones(3000), [10, 90, 0, 100, 20, 60], v, False)
        lp = O.load_points(pos, np.ones(3000), [10, 90, 0, 100, 20, 60], v)
        np.testing.assert_array_equal(np.asarray(pc.get_orig_ids()), lp["orig_ids"])
        assert pc.get_pad() == lp["pad"]


def test_periodic_fixture_consistency():
    """The reference-generated periodic fixture: CSR offsets, segments that
    tile every ray, and the lattice's density x length."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "periodic_walks.npz"))
    st, en, off = z["uniform/starts"], z["uniform/ends"], z["uniform/offsets"]
    L = np.linalg.norm(en - st, axis=1)
    assert off[0] == 0 and np.all(np.diff(off) >= 1) and off[-1] == len(z["uniform/cell_ids"])
    ds = z["uniform/s_exit"] - z["uniform/s_enter"]
    for i in range(len(st)):
        np.testing.assert_allclose(np.sum(ds[off[i]:off[i + 1]]), L[i], rtol=1e-12)
    # same-cell rays (both ends next to one generator) cross other cells
    assert np.all(np.diff(off)[84:96] > 1)
    Ll = np.linalg.norm(z["lattice/ends"] - z["lattice/starts"], axis=1)
    np.testing.assert_allclose(z["lattice/out"][:, 0], 2.5 * Ll, rtol=1e-10)
