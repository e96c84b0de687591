"""Autotuner (vt_cloud_autotune) and the forward+adjoint baseline knob
(VT_PARAM_ADJOINT_KERNEL): they change the speed, never the results."""
import warnings

import numpy as np
import pytest

import vortrace_b200 as vt
from vortrace_b200 import _lib as L
from vortrace_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    pos, f = W.clustered_cloud(200_000, 21, nf=3)
    s, e = W.z_grid([44.0, 56.0], 256)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = vt.ProjectionCloud(pos, f, boundbox=W.BOX)
    return pc, s, e


def test_autotune_choice_keeps_results(case):
    pc, s, e = case
    pc.kernel = "plain"
    ref = pc.projection(s, e)
    res = pc.autotune(s, e, max_sample=16384)
    assert res["kernel"] in ("thread_fp32", "batched_fp64", "batched")
    # 8 kernel x shared-memory depth pairs, then 2 occupancies
    assert res["tried"] == 10 and res["sample_rays"] == 16384 and res["mcrossings_per_s"] > 0
    assert res["blocks_per_sm"] in (0, 4, 3) and res["leaf_size"] == 8
    pc.kernel = "auto"
    np.testing.assert_array_equal(pc.projection(s, e), ref)
    with pytest.raises(ValueError):
        pc.autotune(s[:0], e[:0])


def test_autotune_leaf_size_rebuilds_and_keeps_results(case):
    pc, s, e = case
    pc.kernel = "plain"
    ref = pc.projection(s, e)
    # a taped forward on the tree before tuning
    import torch
    from vortrace_b200 import autograd as ag
    f = torch.tensor(pc.fields_orig.reshape(len(pc.pos_orig), -1), device="cuda",
                     requires_grad=True)
    img = ag.project(pc, f, s[:4096], e[:4096])
    res = pc.autotune(s, e, max_sample=16384, leaf_size=True)
    # three leaf sizes x (8 + 2) configurations
    assert res["tried"] == 30 and res["leaf_size"] in (6, 8, 12)
    info = pc._cloud.info()
    assert info.tree_built
    pc.kernel = "auto"
    np.testing.assert_array_equal(pc.projection(s, e), ref)
    # the tape recorded on the old tree is not used: the adjoint re-walks
    img.sum().backward()
    g_after = f.grad.clone()
    f.grad = None
    ag.project(pc, f, s[:4096], e[:4096]).sum().backward()
    np.testing.assert_allclose(g_after.cpu().numpy(), f.grad.cpu().numpy(), rtol=1e-12,
                               atol=1e-12 * float(f.grad.abs().max()))
    # back to the default leaf size for the other tests of the module
    pc._cloud.set_param(L.PARAM_LEAF_SIZE, 8)
    pc._cloud.set_param(L.PARAM_TUNE_LEAF_SIZE, 0)
    pc._cloud.buildTree()


def test_adjoint_kernel_parameter(case):
    pc, s, e = case
    lib, h = pc._cloud._lib, pc._cloud._h
    g = np.random.default_rng(2).normal(size=(len(s), 3))
    out = pc.projection(s, e)
    grads = []
    for k in (L.KERNEL_AUTO, L.KERNEL_PLAIN_FP64, L.KERNEL_BATCHED):
        pc._cloud.set_param(L.PARAM_ADJOINT_KERNEL, k)
        grad = np.zeros((len(pc.orig_ids), 3))
        L.check(lib.vt_project_adjoint(h, L.dptr(s), L.dptr(e), len(s), L.REDUCE_SUM,
                                       L.dptr(np.ascontiguousarray(out)), L.dptr(g), L.dptr(grad)))
        grads.append(grad)
    pc._cloud.set_param(L.PARAM_ADJOINT_KERNEL, L.KERNEL_AUTO)
    for gr in grads[1:]:
        np.testing.assert_allclose(gr, grads[0], rtol=1e-12, atol=1e-14 * np.abs(grads[0]).max())
    with pytest.raises(ValueError):
        pc._cloud.set_param(L.PARAM_ADJOINT_KERNEL, 7)


def test_graph_replays_projection(case):
    """A captured forward gives the projection's bits on every launch and
    follows new rays written into its buffers; a failing ray is reported."""
    import torch
    from vortrace_b200.graph import ProjectionGraph
    pc, s, e = case
    pc.kernel = "auto"
    ref = pc.projection(s, e)
    S = torch.as_tensor(s, device="cuda")
    E = torch.as_tensor(e, device="cuda")
    g = ProjectionGraph(pc, S, E)
    for _ in range(2):
        g.launch()
        st = g.finish()
        np.testing.assert_array_equal(g.out.cpu().numpy(), ref)
        assert st["rays"] == len(s) and st["crossings"] > 0
    s2, e2 = s[::-1].copy(), e[::-1].copy()
    g.starts.copy_(torch.as_tensor(s2, device="cuda"))
    g.ends.copy_(torch.as_tensor(e2, device="cuda"))
    g.launch()
    g.finish()
    np.testing.assert_array_equal(g.out.cpu().numpy(), ref[::-1])
    g.starts[5, 0] = float("nan")
    g.launch()
    with pytest.raises(ValueError, match="finite"):
        g.finish()
    del g
