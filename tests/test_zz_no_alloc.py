"""vt_project_device_noalloc: the projection entry point that allocates no
device memory (for callers whose device memory is owned by another allocator
or that cannot afford cudaMalloc/cudaFree in their loop).  Called through the
C ABI on the caller's device buffers, it must give the same image as
vt_project_device, bit for bit (the integrate tolerance of the parity tests),
on two calls in a row -- the second reuses the static scratch the first left
behind.  Collected last so a failure here never hides another test."""
import ctypes as C
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_project_device_twice():
    import torch

    import vortrace_b200 as vt
    from vortrace_b200 import _lib as L
    from vortrace_b200 import workloads as W

    lib = L.load()
    pos, f = W.clustered_cloud(200_000, 21, nf=3)
    s, e = W.z_grid([44.0, 56.0], 96)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = vt.ProjectionCloud(pos, f, boundbox=W.BOX)
    h = pc._cloud._h
    dev = torch.device("cuda", 0)
    d_s = torch.from_numpy(s).to(dev)
    d_e = torch.from_numpy(e).to(dev)
    n = s.shape[0]
    ref = torch.empty((n, 3), dtype=torch.float64, device=dev)
    out = torch.empty_like(ref)
    stream = torch.cuda.current_stream(dev).cuda_stream
    L.check(lib.vt_project_device(h, d_s.data_ptr(), d_e.data_ptr(), n, L.REDUCE_SUM,
                                  L.KERNEL_AUTO, ref.data_ptr(), stream, None))
    for _ in range(2):
        out.fill_(float("nan"))
        L.check(lib.vt_project_device_noalloc(h, d_s.data_ptr(), d_e.data_ptr(), n,
                                              L.REDUCE_SUM, out.data_ptr(), stream))
        torch.cuda.synchronize(dev)
        assert torch.equal(out, ref)
    # sizes beyond the scratch's limit are refused before any work
    rc = lib.vt_project_device_noalloc(h, d_s.data_ptr(), d_e.data_ptr(), (1 << 20) + 1,
                                       L.REDUCE_SUM, out.data_ptr(), stream)
    assert rc == L.VT_ERR_INVALID
    assert b"no-allocation limit" in lib.vt_last_error()
