"""The seeded benchmark generators are deterministic and have the stated
shapes and distributions (small sizes)."""
import numpy as np

from vortrace_b200 import workloads as W


def test_clustered_cloud_shape_and_determinism():
    a = W.clustered_cloud(20000, 1, nf=3)
    b = W.clustered_cloud(20000, 1, nf=3)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    pos, f = a
    assert pos.shape == (20000, 3) and f.shape == (20000, 3)
    r = np.linalg.norm(pos[:18000] - 50.0, axis=1)
    assert r.max() <= 40.0 + 1e-9          # truncated Plummer
    assert 1.5 < np.median(r) < 3.0         # half-mass radius of a=2 is ~2.6
    np.testing.assert_allclose(f[:, 1] / f[:, 0] > 0, True)
    assert np.all((f[:, 2] / f[:, 0] >= 0) & (f[:, 2] / f[:, 0] <= 0.02))


def test_transfer_function_valid_rgba():
    rho = np.logspace(-4, 3, 1000)
    rgba = W.transfer_rgba(rho)
    assert rgba.shape == (1000, 4)
    assert np.all((rgba[:, :3] >= 0) & (rgba[:, :3] <= 1)) and np.all(rgba[:, 3] >= 0)
    assert rgba[:, 3].max() <= 0.05 * 1.0001


def test_rotations_orthonormal():
    R = W.random_rotations(8, 4)
    for m in R:
        np.testing.assert_allclose(m @ m.T, np.eye(3), atol=1e-12)
        assert np.linalg.det(m) > 0


def test_uniform_100k_rays():
    w = W.uniform_100k()
    assert w["pos"].shape == (100000, 3) and w["starts"].shape == (128 * 128, 3)
    assert np.all(w["starts"][:, 2] == 0.0) and np.all(w["ends"][:, 2] == 100.0)


def test_nested_cloud_small():
    pos, rho, extra = W.nested_cloud(50000, 5)
    assert pos.shape == (50000, 3) and rho.max() == 1.0
    assert len(extra["a"]) == 8 and min(extra["a"]) >= 0.05 and max(extra["a"]) <= 2.0
