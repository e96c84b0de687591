"""Periodic clouds (loadPoints(..., periodic=True)) against the reference.

Fixtures: tests/golden/periodic_walks.npz, produced by the reference's own
module (tests/golden/make_golden.py): k-NN with the 27-image merge
(src/pointcloud.cpp:308-368), minimum-image split points
(src/ray.cpp:71-86) and the same-cell bisection (src/ray.cpp:220-246)."""
import os
import warnings

import numpy as np
import pytest
import scipy.sparse as sp

import vortrace_b200 as vt

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "periodic_walks.npz")


@pytest.fixture(scope="module")
def pw():
    return np.load(GOLDEN)


def cloud(pos, f, bb):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return vt.ProjectionCloud(pos, f, boundbox=list(bb), periodic=True)


@pytest.fixture(scope="module")
def uni(pw):
    return cloud(pw["uniform/pos"], pw["uniform/fields"], pw["uniform/bb"])


def test_periodic_knn_bit_exact(pw, uni):
    q = pw["uniform/knn_q"]
    for k in (1, 3, 10):
        ids, r2 = uni._cloud.knn(q, k)
        np.testing.assert_array_equal(r2, pw[f"uniform/knn{k}_r2"])
        np.testing.assert_array_equal(ids, pw[f"uniform/knn{k}_ids"])


@pytest.mark.parametrize("kernel", ["auto", "plain", "batched", "thread_fp32"])
def test_periodic_walks_bit_exact(pw, uni, kernel):
    st, en = pw["uniform/starts"], pw["uniform/ends"]
    uni.kernel = kernel
    out = uni.projection(st, en)
    np.testing.assert_array_equal(np.reshape(out, (len(st), -1)), pw["uniform/out"])
    _, cid, se, ds, off = uni.traced_projection(st, en, return_midpoint=False, flatten=True)
    np.testing.assert_array_equal(off, pw["uniform/offsets"])
    np.testing.assert_array_equal(cid, pw["uniform/orig_ids"][pw["uniform/cell_ids"]])
    np.testing.assert_array_equal(se, pw["uniform/s_enter"])
    np.testing.assert_array_equal(ds, pw["uniform/s_exit"] - pw["uniform/s_enter"])


def test_periodic_lattice_invariants(pw):
    # tests/test_periodic.py:126-200 in the reference: density x length
    pc = cloud(pw["lattice/pos"], np.full(len(pw["lattice/pos"]), 2.5), pw["lattice/bb"])
    st, en = pw["lattice/starts"], pw["lattice/ends"]
    L = np.linalg.norm(en - st, axis=1)
    out = pc.projection(st, en)
    np.testing.assert_allclose(out, 2.5 * L, rtol=1e-10)
    np.testing.assert_allclose(out, pw["lattice/out"][:, 0], rtol=1e-10)
    _, ids, _, ds = pc.traced_projection(st, en)
    for i in range(len(st)):
        assert len(ids[i]) == len(set(ids[i]))
        np.testing.assert_allclose(np.sum(ds[i]), L[i], rtol=1e-12)


def test_periodic_same_cell_without_second_cell_raises(pw, uni):
    # both ends and every dyadic sample in one cell (src/ray.cpp:243-246)
    g = pw["uniform/pos"][0]
    st = (g + [1e-4, 0.0, 0.0])[None]
    en = (g + [2e-4, 0.0, 0.0])[None]
    uni.kernel = "auto"
    with pytest.raises(RuntimeError, match="Could not find intermediate cell by bisection"):
        uni.projection(st, en)


def test_periodic_adjoint(pw):
    import torch
    from vortrace_b200 import autograd as VA
    pc = cloud(pw["uniform/pos"], pw["uniform/fields"], pw["uniform/bb"])
    st, en = pw["uniform/starts"], pw["uniform/ends"]
    off = pw["uniform/offsets"]
    ray = np.repeat(np.arange(len(st)), np.diff(off))
    A = sp.csr_matrix((pw["uniform/s_exit"] - pw["uniform/s_enter"], (ray, pw["uniform/cell_ids"])),
                      shape=(len(st), len(pw["uniform/pos"])))
    A.sum_duplicates()
    w = np.random.default_rng(5).normal(size=len(st))
    want = A.T @ w
    for _ in range(2):  # re-walk adjoint, then the segment tape
        f = torch.tensor(pw["uniform/fields"], dtype=torch.float64, device="cuda",
                         requires_grad=True)
        img = VA.project(pc, f, st, en)
        np.testing.assert_array_equal(img.detach().cpu().numpy(), pw["uniform/out"][:, 0])
        (img * torch.as_tensor(w, device="cuda")).sum().backward()
        np.testing.assert_allclose(f.grad.cpu().numpy(), want, rtol=1e-12,
                                   atol=1e-14 * np.abs(want).max())
