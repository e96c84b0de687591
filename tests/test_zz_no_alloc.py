"""vt_project_device_noalloc: the projection entry point that allocates no
device memory (for callers whose device memory is owned by another allocator
or that cannot afford cudaMalloc/cudaFree in their loop).  Called through the
C ABI on the caller's device buffers, it must give the same image as
vt_project_device, bit for bit (the integrate tolerance of the parity tests),
on two calls in a row -- the second reuses the static scratch the first left
behind -- also when rays are handed to the global-stack kernel, whose stacks
and queue live in that scratch; it must report the walk's errors from the
static diagnosis slot and recover afterwards; and a series of calls must
leave the device's free memory unchanged.  Collected last so a failure here
never hides another test."""
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup():
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
    dev = torch.device("cuda", 0)
    return torch, L, lib, pc, dev, torch.from_numpy(s).to(dev), torch.from_numpy(e).to(dev)


def _ref(torch, L, lib, h, d_s, d_e, n, nout, dev, kernel):
    ref = torch.empty((n, nout), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = L.Stats()
    import ctypes as C
    L.check(lib.vt_project_device(h, d_s.data_ptr(), d_e.data_ptr(), n, L.REDUCE_SUM, kernel,
                                  ref.data_ptr(), stream, C.byref(st)))
    return ref, st


def test_noalloc_matches_project_device_twice():
    torch, L, lib, pc, dev, d_s, d_e = _setup()
    h = pc._cloud._h
    n = d_s.shape[0]
    stream = torch.cuda.current_stream(dev).cuda_stream
    ref, _ = _ref(torch, L, lib, h, d_s, d_e, n, 3, dev, L.KERNEL_AUTO)
    out = torch.empty_like(ref)
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


def test_noalloc_hand_over_errors_and_free_memory():
    torch, L, lib, pc, dev, d_s, d_e = _setup()
    h = pc._cloud._h
    n = d_s.shape[0]
    stream = torch.cuda.current_stream(dev).cuda_stream
    # every ray deeper than 2 pending points goes to the global-stack kernel,
    # whose queue and stacks are slices of the static scratch
    pc._cloud.set_param(L.PARAM_LOCAL_STACK, 2)
    ref, st = _ref(torch, L, lib, h, d_s, d_e, n, 3, dev, L.KERNEL_BATCHED)
    assert st.slow_rays > 0
    out = torch.empty_like(ref)

    def call():
        out.fill_(float("nan"))
        rc = lib.vt_project_device_noalloc(h, d_s.data_ptr(), d_e.data_ptr(), n, L.REDUCE_SUM,
                                           out.data_ptr(), stream)
        torch.cuda.synchronize(dev)
        return rc

    def series():
        assert call() == L.VT_OK
        assert torch.equal(out, ref)
        # a stack capacity of 2 is exceeded by the handed-over rays
        pc._cloud.set_param(L.PARAM_STACK_CAP, 2)
        assert call() == 15
        assert b"stack capacity (2)" in lib.vt_last_error()
        pc._cloud.set_param(L.PARAM_STACK_CAP, 4096)
        # a per-ray failure diagnosed from the static slot
        pc._cloud.set_param(L.PARAM_MAX_ITERATIONS, 1)
        assert call() == 10
        assert b"maximum iteration count" in lib.vt_last_error()
        pc._cloud.set_param(L.PARAM_MAX_ITERATIONS, 100000)
        assert call() == L.VT_OK
        assert torch.equal(out, ref)

    series()   # first use loads every kernel the series needs
    free0 = torch.cuda.mem_get_info(dev)[0]
    series()
    series()
    assert torch.cuda.mem_get_info(dev)[0] == free0


def test_noalloc_exact_ties_need_the_tree_built_ahead(tie_walks):
    import torch

    import vortrace_b200 as vt
    from vortrace_b200 import _lib as L

    lib = L.load()
    c = tie_walks["lat6"]
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    d_s = torch.from_numpy(np.ascontiguousarray(c["starts"])).to(dev)
    d_e = torch.from_numpy(np.ascontiguousarray(c["ends"])).to(dev)
    n = d_s.shape[0]
    out = torch.empty((n, 1), dtype=torch.float64, device=dev)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = vt.ProjectionCloud(c["pos"], c["fields"], boundbox=list(c["bb"]), vol=c["vol"])
    h = pc._cloud._h
    # an exact tie needs the reference-order tree, which this entry point
    # does not build
    rc = lib.vt_project_device_noalloc(h, d_s.data_ptr(), d_e.data_ptr(), n, L.REDUCE_SUM,
                                       out.data_ptr(), stream)
    assert rc == L.VT_ERR_RUNTIME
    assert b"vt_cloud_build_tie_tree" in lib.vt_last_error()
    L.check(lib.vt_cloud_build_tie_tree(h))
    for _ in range(2):
        out.fill_(float("nan"))
        L.check(lib.vt_project_device_noalloc(h, d_s.data_ptr(), d_e.data_ptr(), n,
                                              L.REDUCE_SUM, out.data_ptr(), stream))
        torch.cuda.synchronize(dev)
        np.testing.assert_array_equal(out.cpu().numpy()[:, 0], c["out"][:, 0])
