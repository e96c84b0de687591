"""Projection grids generated on the device (vt_grid_rays_device,
vt_project_grid): the rays are bit-identical to the host generator's
(vortrace/grid.py:35-44, :100-192 with center=None), and grid_projection
through the device path gives the same image bits as projecting the host
generator's rays."""
import ctypes as C
import warnings

import numpy as np
import pytest

import vortrace_b200 as vt
from vortrace_b200 import _lib as L
from vortrace_b200 import grid as gr

pytestmark = pytest.mark.gpu

CASES = [
    ([40.0, 60.0], 1024, [0.0, 100.0]),
    ([[0, 100], [0, 100]], (7, 13), [0, 100]),
    ([[-3.3, 7.1], [2.0, 2.5]], (1, 5), [5.0, -2.5]),
    ([[1.0, 1.0], [0.1, 0.3]], (3, 1), [0.0, 1.0]),
    ([[0.0, 1e-300], [0.0, 1.0]], (5, 2), [0.0, 1.0]),
    ([[-1e6, 2.5e6], [1.0 / 3.0, 2.0 / 3.0]], (997, 3), [-7.0, 11.0]),
]


def device_rays(extent, nres, bounds):
    import torch
    lib = L.load()
    ext = gr._as_extent(np.asarray(extent)).astype(np.float64)
    nx, ny = gr._as_nres(nres)
    e4 = np.ascontiguousarray([ext[0][0], ext[0][1], ext[1][0], ext[1][1]], np.float64)
    b = np.ascontiguousarray(bounds, np.float64)
    s = torch.empty((nx * ny, 3), dtype=torch.float64, device="cuda")
    e = torch.empty_like(s)
    stream = torch.cuda.current_stream().cuda_stream
    L.check(lib.vt_grid_rays_device(L.dptr(e4), nx, ny, L.dptr(b), C.c_void_p(s.data_ptr()),
                                    C.c_void_p(e.data_ptr()), C.c_void_p(stream)))
    torch.cuda.synchronize()
    return s.cpu().numpy(), e.cpu().numpy()


@pytest.mark.parametrize("extent,nres,bounds", CASES)
def test_device_rays_bit_identical(extent, nres, bounds):
    hs, he = gr.generate_projection_grid(extent, nres, bounds, None)
    ds, de = device_rays(extent, nres, bounds)
    assert np.array_equal(ds.view(np.uint64), hs.reshape(-1, 3).view(np.uint64))
    assert np.array_equal(de.view(np.uint64), he.reshape(-1, 3).view(np.uint64))


def test_device_rays_reject_bad_arguments():
    lib = L.load()
    e4 = np.array([0.0, 1.0, 0.0, 1.0])
    b = np.array([0.0, 1.0])
    assert lib.vt_grid_rays_device(L.dptr(e4), 0, 4, L.dptr(b), None, None, None) == \
        L.VT_ERR_INVALID
    bad = np.array([0.0, np.inf, 0.0, 1.0])
    assert lib.vt_grid_rays_device(L.dptr(bad), 2, 2, L.dptr(b), None, None, None) == \
        L.VT_ERR_INVALID


@pytest.fixture(scope="module")
def cloud():
    rng = np.random.default_rng(11)
    pos = rng.uniform(0.0, 100.0, (30000, 3))
    fields = np.column_stack([rng.lognormal(0.0, 1.0, 30000), rng.uniform(0.0, 1.0, 30000)])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return vt.ProjectionCloud(pos, fields, boundbox=[0.0, 100.0] * 3)


@pytest.mark.parametrize("kernel", ["auto", "plain", "thread_fp32", "batched"])
@pytest.mark.parametrize("extent,nres,bounds,proj", [
    ([20.0, 80.0], 256, [0.0, 100.0], None),
    ([[10, 90], [30, 70]], (96, 40), [100, 0], None),
    ([5.0, 95.0], (33, 65), [0.0, 100.0], "xz"),
])
def test_grid_projection_device_path(cloud, kernel, extent, nres, bounds, proj):
    cloud.kernel = kernel
    img = cloud.grid_projection(extent, nres, bounds, None, proj=proj)
    nx, ny = gr._as_nres(nres)
    assert cloud.last_stats["rays"] == nx * ny
    hs, he = gr.generate_projection_grid(extent, nres, bounds, None, proj=proj)
    ref = cloud.projection(hs.reshape(-1, 3), he.reshape(-1, 3))
    assert img.shape == (nx, ny, 2)
    assert np.array_equal(img.reshape(-1, 2), ref)
    cloud.kernel = "auto"


def test_grid_projection_float32_extent_uses_host_rays(cloud):
    ext = np.array([20.1, 79.7], np.float32)
    img = cloud.grid_projection(ext, 64, [0.0, 100.0], None, reduction="max")
    hs, he = gr.generate_projection_grid(ext, 64, [0.0, 100.0], None)
    ref = cloud.projection(hs.reshape(-1, 3), he.reshape(-1, 3), reduction="max")
    assert np.array_equal(img.reshape(-1, 2), ref)


@pytest.mark.parametrize("reduction", ["integrate", "volume"])
def test_autograd_grid_project_device_rays(reduction):
    """autograd.grid_project with center=None takes its rays from the device
    generator: same image bits and gradient as projecting the host rays."""
    import torch
    from vortrace_b200 import autograd as VA
    rng = np.random.default_rng(5)
    n = 20000
    pos = rng.uniform(0.0, 100.0, (n, 3))
    if reduction == "volume":
        f = np.column_stack([rng.uniform(0, 1, (n, 3)), rng.uniform(0.0, 0.2, n)])
    else:
        f = np.column_stack([rng.lognormal(0.0, 1.0, n), rng.uniform(0.0, 1.0, n)])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = vt.ProjectionCloud(pos, f, boundbox=[0.0, 100.0] * 3)
    ft = torch.tensor(f, device="cuda", requires_grad=True)
    img = VA.grid_project(pc, ft, [[10, 90], [20, 80]], (48, 40), [0, 100], None,
                          reduction=reduction)
    w = torch.as_tensor(rng.normal(size=tuple(img.shape)), device="cuda")
    (img * w).sum().backward()
    g_dev = ft.grad.clone()
    ft.grad = None
    hs, he = gr.generate_projection_grid([[10, 90], [20, 80]], (48, 40), [0, 100], None)
    ref = VA.project(pc, ft, hs.reshape(-1, 3), he.reshape(-1, 3), reduction=reduction)
    assert img.shape[:2] == (48, 40)
    assert torch.equal(img.reshape(ref.shape), ref)
    (ref * w.reshape(ref.shape)).sum().backward()
    torch.testing.assert_close(g_dev, ft.grad, rtol=1e-12, atol=1e-15)
