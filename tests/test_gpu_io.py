"""Cloud persistence (vortrace_b200.io, ProjectionCloud.save/load, the tree
blob): a restored tree gives the same bits as a freshly built one."""
import warnings

import numpy as np
import pytest

import vortrace_b200 as vt
from vortrace_b200 import io as vio

pytestmark = pytest.mark.gpu


def make(periodic=False, seed=3):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 10, (30000, 3))
    f = np.column_stack([rng.lognormal(0, 1, 30000), rng.uniform(0, 1, 30000)])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = vt.ProjectionCloud(pos, f, boundbox=[0, 10] * 3, periodic=periodic)
    s = rng.uniform(0, 10, (3000, 3))
    e = rng.uniform(0, 10, (3000, 3))
    return pc, s, e


@pytest.mark.parametrize("periodic", [False, True])
def test_save_load_cloud_restores_tree(tmp_path, periodic):
    pc, s, e = make(periodic)
    ref = pc.projection(s, e)
    blob = pc.save_tree_bytes()
    assert blob[:8] == b"VTB2TREE"
    path = tmp_path / "cloud.npz"
    pc.save(path)
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        pc2 = vt.ProjectionCloud.load(path)
    assert not any("rebuilding the tree" in str(w.message) for w in caught)
    assert pc2.periodic == periodic
    np.testing.assert_array_equal(pc2.projection(s, e), ref)
    assert pc2.save_tree_bytes() == blob
    # without the tree: rebuilt on load, same bits
    vio.save_cloud(tmp_path / "notree.npz", pc, save_tree=False)
    with np.load(tmp_path / "notree.npz") as z:
        assert "_kdtree" not in z
    np.testing.assert_array_equal(vio.load_cloud(tmp_path / "notree.npz").projection(s, e), ref)


def test_foreign_and_mismatched_blobs(tmp_path):
    pc, s, e = make()
    ref = pc.projection(s, e)
    path = tmp_path / "foreign.npz"
    np.savez(path, pos=pc.pos_orig, fields=pc.fields_orig, boundbox=np.asarray(pc.boundbox),
             periodic=np.bool_(False), _kdtree=np.void(b"\x01nanoflann-index" * 64))
    with pytest.warns(UserWarning, match="rebuilding the tree"):
        pc2 = vio.load_cloud(path)
    np.testing.assert_array_equal(pc2.projection(s, e), ref)
    other, _, _ = make(seed=4)
    with pytest.raises(ValueError, match="built on other points"):
        other._cloud.loadTreeFromBytes(pc.save_tree_bytes())
    with pytest.raises(ValueError, match="wrong size|too short|does not fit"):
        pc._cloud.loadTreeFromBytes(pc.save_tree_bytes()[:-8])
