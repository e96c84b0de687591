"""ProjectionCloud behaviour on the CUDA path, following the reference's own
tests (tests/test_degenerate.py, test_traced_projection.py,
test_volume_render.py, test_multifield.py, test_padding.py,
test_vortrace.py of gusbeane/vortrace)."""
import warnings

import numpy as np
import pytest

import vortrace_b200 as vt
from tests.conftest import make_cubic_lattice

pytestmark = pytest.mark.gpu

KERNELS = ["plain", "batched"]


def pc_of(pos, fields, bb, vol=None, **kw):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return vt.ProjectionCloud(pos, fields, boundbox=bb, vol=vol, **kw)


@pytest.fixture
def lattice_cloud():
    pos, f, vol, bb = make_cubic_lattice()
    return pc_of(pos, f, bb, vol)


@pytest.fixture
def lattice_cloud_multifield():
    pos, f, vol, bb = make_cubic_lattice()
    return pc_of(pos, np.column_stack([f, 2 * f]), bb, vol)


# ---------------------------------------------------- degenerate geometry
DEGENERATE = {
    "diagonal_through_vertices": ([-0.1] * 3, [4.1] * 3),
    "ray_along_face": ([0.5, 0.2, -0.1], [0.5, 0.2, 4.1]),
    "ray_along_edge": ([0.5, 0.5, -0.1], [0.5, 0.5, 4.1]),
    "single_vertex": ([0.1] * 3, [0.9] * 3),
    "near_degenerate": ([0.50001, 0.50001, -0.1], [0.50001, 0.50001, 4.1]),
}


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("name", sorted(DEGENERATE))
def test_degenerate_integral_is_length(lattice_cloud, name, kernel):
    s, e = DEGENERATE[name]
    lattice_cloud.kernel = kernel
    dens, _, _, _ = lattice_cloud.traced_projection(np.array(s), np.array(e))
    np.testing.assert_allclose(dens, np.linalg.norm(np.subtract(e, s)), rtol=1e-6)
    out = lattice_cloud.projection(np.array([s]), np.array([e]))
    np.testing.assert_allclose(out[0], np.linalg.norm(np.subtract(e, s)), rtol=1e-6)


def test_selective_field():
    pos, f, vol, bb = make_cubic_lattice()
    f = np.zeros(len(pos))
    f[np.argmin(np.linalg.norm(pos - 2.0, axis=1))] = 1.0
    pc = pc_of(pos, f, bb, vol)
    dens, *_ = pc.traced_projection(np.array([2.0, 2.0, -0.1]), np.array([2.0, 2.0, 4.1]))
    assert dens > 0.0


def test_float32_quantised_positions():
    n = 10
    pos, f, vol, bb = make_cubic_lattice(n)
    off = np.array([500.0, 500.0, 500.1])
    p32 = (pos + off).astype(np.float32)
    p32 -= off.astype(np.float32)
    pc = pc_of(p32.astype(np.float64), f, bb, vol)
    s, e = [-0.1] * 3, [n - 0.9] * 3
    dens, *_ = pc.traced_projection(np.array(s), np.array(e))
    np.testing.assert_allclose(dens, np.linalg.norm(np.subtract(e, s)), rtol=1e-3)


def test_same_cell():
    pos, f, vol, bb = make_cubic_lattice()
    pc = pc_of(pos, f, bb, vol)
    res = pc.traced_projection(np.array([0.5] * 3), np.array([0.6] * 3))[0]
    np.testing.assert_allclose(res, np.linalg.norm([0.1] * 3), rtol=1e-6)


# ------------------------------------------------------ traced projection
def test_traced_single_ray_formats(lattice_cloud):
    s, e = np.array([2.0, 2.0, -0.5]), np.array([2.0, 2.0, 4.5])
    val, cid, sv, ds = lattice_cloud.traced_projection(s, e)
    assert np.isscalar(val) or np.ndim(val) == 0
    np.testing.assert_allclose(val, 5.0, rtol=1e-6)
    np.testing.assert_allclose(np.sum(ds), 5.0, rtol=1e-12)
    val2, *_ = lattice_cloud.traced_projection(s[None], e[None])
    np.testing.assert_allclose(val2, 5.0, rtol=1e-6)
    _, _, s_mid, _ = lattice_cloud.traced_projection(s, e, return_midpoint=True)
    _, _, s_ent, _ = lattice_cloud.traced_projection(s, e, return_midpoint=False)
    assert len(s_mid) == len(s_ent) and not np.array_equal(s_mid, s_ent)


def _rays(n=8):
    st = np.tile([2.0, 2.0, -0.5], (n, 1))
    en = np.tile([2.0, 2.0, 4.5], (n, 1))
    st[1], en[1] = [1.0, 2.0, -0.5], [1.0, 2.0, 4.5]
    st[2], en[2] = [3.0, 3.0, -0.5], [3.0, 3.0, 4.5]
    return st, en


def test_traced_batch_formats(lattice_cloud):
    st, en = _rays()
    vals, cl, sl, dl = lattice_cloud.traced_projection(st, en)
    assert vals.shape[0] == 8 and len(cl) == len(sl) == len(dl) == 8
    vals, cid, sv, ds, off = lattice_cloud.traced_projection(st, en, flatten=True)
    assert off[0] == 0 and off[-1] == len(cid) and len(off) == 9
    assert len(cid) == len(sv) == len(ds)


def test_traced_batch_matches_sequential(lattice_cloud):
    st, en = _rays(4)
    vals, cl, sl, dl = lattice_cloud.traced_projection(st, en)
    for i in range(4):
        v, c, s, d = lattice_cloud.traced_projection(st[i], en[i])
        np.testing.assert_allclose(vals[i], v, rtol=1e-12)
        np.testing.assert_array_equal(cl[i], c)
        np.testing.assert_array_equal(sl[i], s)
        np.testing.assert_array_equal(dl[i], d)
    np.testing.assert_allclose(vals, lattice_cloud.projection(st, en), rtol=1e-12)


def test_multifield_batch(lattice_cloud_multifield):
    st = np.tile([2.0, 2.0, -0.5], (4, 1))
    en = np.tile([2.0, 2.0, 4.5], (4, 1))
    vals, *_ = lattice_cloud_multifield.traced_projection(st, en)
    assert vals.shape == (4, 2)
    np.testing.assert_allclose(vals[:, 1], 2 * vals[:, 0], rtol=1e-12)


@pytest.mark.parametrize("red", ["max", "min"])
def test_traced_max_min_match_projection(lattice_cloud, red):
    st = np.array([[2.0, 2.0, -0.5], [1.0, 1.0, -0.5]])
    en = np.array([[2.0, 2.0, 4.5], [1.0, 1.0, 4.5]])
    vals, *_ = lattice_cloud.traced_projection(st, en, reduction=red)
    np.testing.assert_allclose(vals, lattice_cloud.projection(st, en, reduction=red), rtol=1e-12)


def test_traced_errors(lattice_cloud):
    with pytest.raises(ValueError):
        lattice_cloud.traced_projection(np.zeros((3, 3)), np.zeros((4, 3)))
    with pytest.raises(ValueError):
        lattice_cloud.traced_projection(np.zeros((3, 2)), np.zeros((3, 2)))
    with pytest.raises(ValueError):
        lattice_cloud.traced_projection(np.zeros(4), np.zeros(4))
    with pytest.raises(AttributeError, match="traced_projection"):
        lattice_cloud.single_projection(np.zeros(3), np.ones(3))
    with pytest.raises(ValueError, match="Unknown reduction"):
        lattice_cloud.traced_projection(np.zeros(3), np.ones(3), reduction="bogus")
    with pytest.raises(ValueError, match="identical shape"):
        lattice_cloud.projection(np.zeros((3, 3)), np.zeros((2, 3)))


# -------------------------------------------------------------- volume
def _uniform_rgba(rgba, n=500, box=100.0):
    rng = np.random.default_rng(42)
    return pc_of(rng.random((n, 3)) * box, np.tile(rgba, (n, 1)), [0.0, box] * 3), box


@pytest.mark.parametrize("kernel", KERNELS)
def test_volume_closed_forms(kernel):
    pc, box = _uniform_rgba([1.0, 0.5, 0.25, 0.0])
    pc.kernel = kernel
    s, e = np.array([box / 2, box / 2, 0.1]), np.array([box / 2, box / 2, box - 0.1])
    rgb, *_ = pc.traced_projection(s, e, reduction="volume")
    assert rgb.shape == (3,)
    np.testing.assert_allclose(rgb, 0.0, atol=1e-15)
    R, G, B, a = 0.8, 0.4, 0.2, 0.01
    pc, box = _uniform_rgba([R, G, B, a])
    pc.kernel = kernel
    rgb, _, _, ds = pc.traced_projection(s, e, reduction="volume")
    np.testing.assert_allclose(rgb, np.array([R, G, B]) * (1 - np.exp(-a * np.sum(ds))),
                               rtol=1e-10)
    pc, box = _uniform_rgba([1.0, 0.5, 0.25, 1000.0])
    rgb = pc.projection(s[None], e[None], reduction="volume")[0]
    np.testing.assert_allclose(rgb, [1.0, 0.5, 0.25], rtol=1e-6)


def test_volume_reversed_differs():
    rng = np.random.default_rng(123)
    n = 500
    f = np.column_stack([rng.random(n), rng.random(n), rng.random(n), 0.01 + 0.05 * rng.random(n)])
    pc = pc_of(rng.random((n, 3)) * 100.0, f, [0.0, 100.0] * 3)
    s, e = np.array([50.0, 50.0, 0.1]), np.array([50.0, 50.0, 99.9])
    fwd, *_ = pc.traced_projection(s, e, reduction="volume")
    rev, *_ = pc.traced_projection(e, s, reduction="volume")
    assert not np.allclose(fwd, rev, atol=1e-10)


def test_volume_validation():
    rng = np.random.default_rng(1)
    pos = rng.random((100, 3)) * 10
    bad_r = np.column_stack([rng.random(100) * 2, rng.random(100), rng.random(100),
                             rng.random(100) * 0.1])
    with pytest.raises(ValueError, match=r"R, G, B.*\[0, 1\]"):
        pc_of(pos, bad_r, [0, 10] * 3).grid_projection([2, 8], 8, [0, 10], None,
                                                       reduction="volume")
    neg_a = np.column_stack([rng.random(100), rng.random(100), rng.random(100),
                             -0.1 * np.ones(100)])
    with pytest.raises(ValueError, match="alpha >= 0"):
        pc_of(pos, neg_a, [0, 10] * 3).traced_projection([5, 5, 0.1], [5, 5, 9.9],
                                                         reduction="volume")
    for nf in (1, 2, 3):
        f = rng.random((100, nf)) if nf > 1 else rng.random(100)
        with pytest.raises(ValueError, match="4 fields"):
            pc_of(pos, f, [0, 10] * 3).projection(np.array([[5, 5, 0.1]]),
                                                  np.array([[5, 5, 9.9]]), reduction="volume")


# ---------------------------------------------- multi-field / snapshot
def test_snapshot_multifield_and_reductions(galaxy):
    pos, dens, box = galaxy["pos"], galaxy["dens"], galaxy["box_size"]
    bb = [0.0, box] * 3
    ext = [box / 2 - 37.5, box / 2 + 37.5]
    pc1 = pc_of(pos, dens, bb)
    pc2 = pc_of(pos, np.column_stack([dens, 2 * dens]), bb)
    d1 = pc1.grid_projection(ext, 64, [0.0, box], None)
    d2 = pc2.grid_projection(ext, 64, [0.0, box], None)
    assert d1.shape == (64, 64) and d2.shape == (64, 64, 2)
    np.testing.assert_allclose(d2[:, :, 1], 2 * d2[:, :, 0], rtol=1e-12)
    np.testing.assert_allclose(d2[:, :, 0], d1, rtol=1e-12)
    e2 = [box / 2 - 30, box / 2 + 30]
    dmax = pc1.grid_projection(e2, 32, [0.0, box], None, reduction="max")
    dmin = pc1.grid_projection(e2, 32, [0.0, box], None, reduction="min")
    dsum = pc1.grid_projection(e2, 32, [0.0, box], None)
    assert np.all(dmax > 0) and np.all(dmin <= dmax) and not np.allclose(dmax, dsum)
    s, e = np.array([box / 2, box / 2, 0.1]), np.array([box / 2, box / 2, box - 0.1])
    mx, cid, _, _ = pc1.traced_projection(s, e, reduction="max")
    np.testing.assert_allclose(mx, np.max(dens[cid]))
    mn, cid, _, _ = pc1.traced_projection(s, e, reduction="min")
    np.testing.assert_allclose(mn, np.min(dens[cid]))


# -------------------------------------------------------- padding / warns
def test_vol_padding_and_warnings():
    rng = np.random.default_rng(42)
    bb = [10.0, 90.0] * 3
    pos = np.vstack([rng.uniform(20, 80, (100, 3)), [[5.0, 50.0, 50.0]]])
    vol = np.full(len(pos), (4.0 / 3.0) * np.pi * 5.0 ** 3)
    pc = vt.ProjectionCloud(pos, np.ones(len(pos)), boundbox=bb, vol=vol)
    assert len(pc.orig_ids) == len(pos)
    pos = np.vstack([rng.uniform(20, 80, (100, 3)), [[-100.0, 50.0, 50.0]]])
    pc = vt.ProjectionCloud(pos, np.ones(len(pos)), boundbox=bb,
                            vol=np.full(len(pos), (4.0 / 3.0) * np.pi))
    assert len(pc.orig_ids) == 100 and 100 not in pc.orig_ids
    with pytest.warns(UserWarning, match="vol"):
        vt.ProjectionCloud(rng.uniform(0, 1, (50, 3)), np.ones(50), boundbox=[0, 1] * 3)
    with pytest.warns(UserWarning, match="1e-6"):
        vt.ProjectionCloud(rng.uniform(0, 1, (50, 3)), np.ones(50), boundbox=[0, 1] * 3,
                           vol=np.full(50, 1e-21))


def test_thin_box_uniform_padding():
    pos = np.array([[50.0, 50.0, 50.5], [50.0, 50.0, 40.0]])
    pc = pc_of(pos, np.ones(2), [0.0, 100.0, 0.0, 100.0, 50.0, 51.0])
    assert len(pc.orig_ids) == 2


def test_no_tree_and_empty_rays():
    pos, f, vol, bb = make_cubic_lattice(3)
    pc = pc_of(pos, f, bb, vol, _skip_build_tree=True)
    with pytest.raises(RuntimeError, match="no valid tree"):
        pc.projection(np.zeros((1, 3)), np.ones((1, 3)))
    pc = pc_of(pos, f, bb, vol)
    with pytest.raises(RuntimeError, match="has not yet been made"):
        pc.projection(np.zeros((0, 3)), np.zeros((0, 3)))


def test_verbose_messages(capfd):
    pos, f, vol, bb = make_cubic_lattice(3)
    vt.set_verbose(True)
    try:
        pc = pc_of(pos, f, bb, vol)
        pc.projection(np.array([[0.0, 0.0, 0.0]]), np.array([[2.0, 2.0, 2.0]]))
    finally:
        vt.set_verbose(False)
    out = capfd.readouterr().out
    assert "Tree build took" in out and "Projection generation took" in out
