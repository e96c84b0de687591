"""Gradients of projections w.r.t. the per-cell fields (adjoint kernels).

References:
  * the sparse reference gradient A^T g, A[r, c] = sum of ds of ray r in cell
    c, assembled from the oracle's segment lists (bit-identical to the
    reference's makeDetailedProjection);
  * for 'volume', the reverse-mode compositing adjoint evaluated in numpy on
    those segment lists with exact suffix sums;
  * central finite differences through the forward kernel (rtol 1e-6).
"""
import warnings

import numpy as np
import pytest
import scipy.sparse as sp

import vortrace_b200 as vt
from oracle import oracle as O
from vortrace_b200 import _lib as L
from vortrace_b200 import workloads as W

pytestmark = pytest.mark.gpu

FD_RTOL = 1e-6


def setup(pos, fields, bb, starts, ends, mode):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = vt.ProjectionCloud(pos, fields, boundbox=bb)
        lp = O.load_points(pos, fields, bb)
    ot = O.OracleTree(lp["pts"], lp["fields"], lp["valid_rgba"])
    out, segs = ot.project(starts, ends, mode, segments=True)
    return pc, lp, out, segs


def adjoint(pc, starts, ends, mode, out, gout, kernel_fields=None):
    nf = pc._nfields
    grad = np.zeros((len(pc.orig_ids), nf))
    L.check(pc._cloud._lib.vt_project_adjoint(pc._cloud._h, L.dptr(np.ascontiguousarray(starts)),
                                              L.dptr(np.ascontiguousarray(ends)), len(starts),
                                              mode, L.dptr(np.ascontiguousarray(out)),
                                              L.dptr(np.ascontiguousarray(gout)),
                                              L.dptr(grad)))
    return grad


def sparse_sum_gradient(segs, nrays, npart, gout):
    cid, se, sx, off = segs
    ray = np.repeat(np.arange(nrays), np.diff(off))
    A = sp.csr_matrix((sx - se, (ray, cid)), shape=(nrays, npart))
    A.sum_duplicates()
    return A.T @ gout


def volume_reference_gradient(segs, fields, nrays, gout):
    cid, se, sx, off = segs
    grad = np.zeros_like(fields)
    for r in range(nrays):
        c = cid[off[r]:off[r + 1]]
        ds = (sx - se)[off[r]:off[r + 1]]
        rgb, a = fields[c, :3], fields[c, 3]
        o = 1.0 - np.exp(-a * ds)
        T = np.concatenate([[1.0], np.cumprod(1.0 - o)[:-1]])
        contrib = (T * o)[:, None] * rgb
        suffix = np.cumsum(contrib[::-1], axis=0)[::-1] - contrib  # sum over later segments
        g = gout[r]
        np.add.at(grad, (c, slice(0, 3)), (T * o)[:, None] * g[None, :])
        ga = ds * np.sum(g[None, :] * (T[:, None] * rgb * (1.0 - o)[:, None] - suffix), axis=1)
        np.add.at(grad[:, 3], c, ga)
    return grad


def fd_column(pc, fields_int, starts, ends, red, wts, cell, comp, h):
    """Central difference of L = sum(W * img) w.r.t. fields_int[cell, comp].

    Summed as sum(W * (img+ - img-)): rays that miss the cell give exactly
    zero, so the rounding of the full loss does not enter the difference."""
    f = fields_int.copy()
    imgs = []
    for sgn in (1.0, -1.0):
        f[cell, comp] = fields_int[cell, comp] + sgn * h
        L.check(pc._cloud._lib.vt_cloud_set_fields(pc._cloud._h, L.dptr(f)))
        imgs.append(pc.projection(starts, ends, reduction=red).reshape(wts.shape))
    L.check(pc._cloud._lib.vt_cloud_set_fields(pc._cloud._h, L.dptr(fields_int)))
    return np.sum(wts * (imgs[0] - imgs[1])) / (2.0 * h)


@pytest.fixture(scope="module")
def sum_case():
    pos, rho = W.clustered_cloud(200_000, 11, nf=1)
    s, e = W.z_grid([44.0, 56.0], 48)
    return pos, rho, s, e


def test_sum_adjoint_matches_sparse_reference(sum_case):
    pos, rho, s, e = sum_case
    pc, lp, out, segs = setup(pos, rho, W.BOX, s, e, "integrate")
    g = np.random.default_rng(0).normal(size=(len(s), 1))
    grad = adjoint(pc, s, e, L.REDUCE_SUM, out, g)
    ref = sparse_sum_gradient(segs, len(s), len(lp["orig_ids"]), g)
    np.testing.assert_allclose(grad, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())


def test_sum_adjoint_multifield_and_hand_over(sum_case):
    pos, rho, s, e = sum_case
    f3 = np.column_stack([rho, 2 * rho, rho ** 2])
    pc, lp, out, segs = setup(pos, f3, W.BOX, s, e, "integrate")
    g = np.random.default_rng(1).normal(size=(len(s), 3))
    ref = sparse_sum_gradient(segs, len(s), len(lp["orig_ids"]), g)
    a = adjoint(pc, s, e, L.REDUCE_SUM, out, g)
    np.testing.assert_allclose(a, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())
    # every ray deeper than one pending point goes through the global-stack
    # kernel, which must skip the segments already scattered
    pc._cloud.set_param(L.PARAM_LOCAL_STACK, 1)
    b = adjoint(pc, s, e, L.REDUCE_SUM, out, g)
    pc._cloud.set_param(L.PARAM_LOCAL_STACK, 1 << 30)
    np.testing.assert_allclose(b, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())


def _taped_forward(pc, tape, dS, dE, mode=L.REDUCE_SUM):
    import ctypes as C
    import torch
    n = dS.shape[0]
    nout = 3 if mode == L.REDUCE_VOLUME else pc._nfields
    out = torch.empty((n, nout), dtype=torch.float64, device="cuda")
    st = L.Stats()
    stream = torch.cuda.current_stream().cuda_stream
    L.check(pc._cloud._lib.vt_project_device_tape(pc._cloud._h, tape.h, dS.data_ptr(),
                                                  dE.data_ptr(), n, mode, L.KERNEL_AUTO,
                                                  out.data_ptr(), stream, C.byref(st)))
    return out


def _tape_adjoint(pc, tape, dS, dE, out, g, mode=L.REDUCE_SUM):
    import torch
    gd = torch.as_tensor(np.ascontiguousarray(g), device="cuda")
    grad = torch.zeros((len(pc.orig_ids), pc._nfields), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    L.check(pc._cloud._lib.vt_tape_adjoint_device(pc._cloud._h, tape.h, dS.data_ptr(),
                                                  dE.data_ptr(), dS.shape[0], mode,
                                                  out.data_ptr(), gd.data_ptr(),
                                                  grad.data_ptr(), stream))
    return grad.cpu().numpy()


@pytest.mark.parametrize("nf", [1, 2, 3])
def test_tape_adjoint_matches_sparse_reference(sum_case, nf):
    """The taped forward gives the same image bits, records exactly one
    entry per segment (also for rays finished by the global-stack kernel),
    and its scatter adjoint equals the sparse reference gradient.  The first
    taped forward on a fresh cloud has no size estimate: its tape does not
    fit, and the adjoint re-walks the rays instead."""
    import torch
    pos, rho, s, e = sum_case
    f = np.column_stack([rho, 2 * rho, rho ** 2][:nf])
    pc, lp, out, segs = setup(pos, f, W.BOX, s, e, "integrate")
    nseg = int(segs[3][-1])
    g = np.random.default_rng(3 + nf).normal(size=(len(s), nf))
    ref = sparse_sum_gradient(segs, len(s), len(lp["orig_ids"]), g)
    tol = dict(rtol=1e-12, atol=1e-14 * np.abs(ref).max())
    tape = L.Tape(pc._cloud._lib, pc._cloud._h)
    dS = torch.as_tensor(s, device="cuda").contiguous()
    dE = torch.as_tensor(e, device="cuda").contiguous()
    sizes = []
    for it in range(3):
        img = _taped_forward(pc, tape, dS, dE)
        np.testing.assert_array_equal(img.cpu().numpy(), out)
        sizes.append(int(pc._cloud._lib.vt_tape_size(tape.h)))
        grad = _tape_adjoint(pc, tape, dS, dE, img, g)
        bad = np.argwhere(~np.isclose(grad, ref, rtol=tol["rtol"], atol=tol["atol"]))
        np.testing.assert_allclose(grad, ref, **tol, err_msg=(
            f"forward {it} (tape size {sizes[-1]} of {nseg} segments), elements [cell, field] "
            f"{bad[:8].tolist()}, got {grad[tuple(bad[:8].T)].tolist()}, "
            f"want {ref[tuple(bad[:8].T)].tolist()}"))
    assert sizes[0] == 0 and sizes[1] == nseg and sizes[2] == nseg
    # rays deeper than one pending point are finished by the global-stack
    # kernel, which must not record their first segments twice
    pc._cloud.set_param(L.PARAM_LOCAL_STACK, 1)
    try:
        img = _taped_forward(pc, tape, dS, dE)
        assert int(pc._cloud._lib.vt_tape_size(tape.h)) == nseg
        np.testing.assert_array_equal(img.cpu().numpy(), out)
        np.testing.assert_allclose(_tape_adjoint(pc, tape, dS, dE, img, g), ref, **tol)
    finally:
        pc._cloud.set_param(L.PARAM_LOCAL_STACK, 1 << 30)


def test_null_stream_adjoint_follows_the_default_stream(sum_case):
    """A NULL stream selects the handle's stream, which is ordered with the
    legacy default stream (PyTorch's default) both ways: a zero fill of the
    gradient queued there behind a long kernel lands before the scatter adds
    into the buffer, and a read there sees the finished scatter."""
    import torch
    pos, rho, s, e = sum_case
    pc, lp, out, segs = setup(pos, rho, W.BOX, s, e, "integrate")
    g = np.random.default_rng(7).normal(size=(len(s), 1))
    ref = sparse_sum_gradient(segs, len(s), len(lp["orig_ids"]), g)
    tape = L.Tape(pc._cloud._lib, pc._cloud._h)
    dS = torch.as_tensor(s, device="cuda").contiguous()
    dE = torch.as_tensor(e, device="cuda").contiguous()
    assert torch.cuda.current_stream().cuda_stream == 0  # the legacy default stream
    for _ in range(2):  # the second forward's tape fits (sized by the first)
        img = _taped_forward(pc, tape, dS, dE)
    assert int(pc._cloud._lib.vt_tape_size(tape.h)) == int(segs[3][-1])
    gd = torch.as_tensor(np.ascontiguousarray(g), device="cuda")
    grad = torch.full((len(pc.orig_ids), 1), 1e30, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    torch.cuda._sleep(100_000_000)  # about 50 ms of GPU time on the default stream
    grad.zero_()                    # queued behind it
    L.check(pc._cloud._lib.vt_tape_adjoint_device(pc._cloud._h, tape.h, dS.data_ptr(),
                                                  dE.data_ptr(), dS.shape[0], L.REDUCE_SUM,
                                                  img.data_ptr(), gd.data_ptr(), grad.data_ptr(),
                                                  None))
    np.testing.assert_allclose(grad.cpu().numpy(), ref, rtol=1e-12,
                               atol=1e-14 * np.abs(ref).max())


def test_tape_volume_adjoint(vol_case):
    """Volume forward with a tape (48 bytes per segment) gives the same image
    (1e-12) and its scatter adjoint matches the reverse-mode compositing
    reference; the first call on a fresh cloud falls back to re-walking."""
    import torch
    pos, rgba, s, e = vol_case
    pc, lp, out, segs = setup(pos, rgba, W.BOX, s, e, "volume")
    nseg = int(segs[3][-1])
    g = np.random.default_rng(9).normal(size=(len(s), 3))
    ref = volume_reference_gradient(segs, lp["fields"], len(s), g)
    tape = L.Tape(pc._cloud._lib, pc._cloud._h)
    dS = torch.as_tensor(s, device="cuda").contiguous()
    dE = torch.as_tensor(e, device="cuda").contiguous()
    sizes = []
    for _ in range(3):
        img = _taped_forward(pc, tape, dS, dE, L.REDUCE_VOLUME)
        np.testing.assert_allclose(img.cpu().numpy(), out, rtol=1e-12, atol=1e-300)
        sizes.append(int(pc._cloud._lib.vt_tape_size(tape.h)))
        grad = _tape_adjoint(pc, tape, dS, dE, img, g, L.REDUCE_VOLUME)
        np.testing.assert_allclose(grad, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())
    assert sizes == [0, nseg, nseg]


def test_sum_adjoint_finite_differences(sum_case):
    pos, rho, s, e = sum_case
    pc, lp, out, segs = setup(pos, rho, W.BOX, s, e, "integrate")
    wts = np.random.default_rng(2).normal(size=len(s))
    grad = adjoint(pc, s, e, L.REDUCE_SUM, out, wts[:, None])[:, 0]
    fint = lp["fields"].copy()
    hit = np.nonzero(grad)[0]
    cells = np.random.default_rng(3).choice(hit, 16, replace=False)
    for c in cells:
        fd = fd_column(pc, fint, s, e, "integrate", wts, c, 0, 1e-3 * max(1.0, abs(fint[c, 0])))
        np.testing.assert_allclose(fd, grad[c], rtol=FD_RTOL)


@pytest.fixture(scope="module")
def vol_case():
    pos, f = W.clustered_cloud(100_000, 12, nf=3)
    rgba = W.transfer_rgba(f[:, 0] * 30.0)
    s, e = W.z_grid([45.0, 55.0], 32)
    return pos, rgba, s, e


def test_volume_adjoint_matches_reference(vol_case):
    pos, rgba, s, e = vol_case
    pc, lp, out, segs = setup(pos, rgba, W.BOX, s, e, "volume")
    g = np.random.default_rng(4).normal(size=(len(s), 3))
    grad = adjoint(pc, s, e, L.REDUCE_VOLUME, out, g)
    ref = volume_reference_gradient(segs, lp["fields"], len(s), g)
    scale = np.abs(ref).max(axis=0)
    np.testing.assert_allclose(grad, ref, rtol=1e-9, atol=1e-12 * scale.max())


def test_volume_adjoint_finite_differences(vol_case):
    pos, rgba, s, e = vol_case
    pc, lp, out, segs = setup(pos, rgba, W.BOX, s, e, "volume")
    wts = np.random.default_rng(5).normal(size=(len(s), 3))
    grad = adjoint(pc, s, e, L.REDUCE_VOLUME, out, wts)
    fint = lp["fields"].copy()
    rng = np.random.default_rng(6)
    inner = np.all((fint[:, :3] > 0.01) & (fint[:, :3] < 0.99), axis=1) & (fint[:, 3] > 1e-3)
    hit = np.nonzero((np.abs(grad).sum(1) > 0) & inner)[0]
    checked = 0
    for c in rng.choice(hit, min(64, len(hit)), replace=False):
        comp = int(rng.integers(0, 4))
        h = 1e-5 * max(1.0, abs(fint[c, comp]))
        fd = fd_column(pc, fint, s, e, "volume", wts, c, comp, h)
        if abs(grad[c, comp]) < 1e-8 * np.abs(grad).max():
            continue  # below FD resolution
        np.testing.assert_allclose(fd, grad[c, comp], rtol=FD_RTOL)
        checked += 1
    assert checked >= 16


def test_autograd_function(sum_case, vol_case):
    import torch
    from vortrace_b200 import autograd as VA
    pos, rho, s, e = sum_case
    pc, lp, out, segs = setup(pos, rho, W.BOX, s, e, "integrate")
    f = torch.tensor(rho, dtype=torch.float64, device="cuda", requires_grad=True)
    img = VA.project(pc, f, s, e)
    np.testing.assert_array_equal(img.detach().cpu().numpy(), out[:, 0])
    wts = torch.randn(len(s), dtype=torch.float64, device="cuda")
    (img * wts).sum().backward()
    ref = sparse_sum_gradient(segs, len(s), len(lp["orig_ids"]), wts.cpu().numpy()[:, None])
    want = np.zeros(len(rho))
    want[lp["orig_ids"]] = ref[:, 0]
    np.testing.assert_allclose(f.grad.cpu().numpy(), want, rtol=1e-12,
                               atol=1e-14 * np.abs(want).max())
    pos, rgba, s, e = vol_case
    pc, lp, out, segs = setup(pos, rgba, W.BOX, s, e, "volume")
    fv = torch.tensor(rgba, dtype=torch.float64, device="cuda", requires_grad=True)
    imgv = VA.project(pc, fv, s, e, reduction="volume")
    np.testing.assert_allclose(imgv.detach().cpu().numpy(), out, rtol=1e-12, atol=1e-300)
    wv = torch.randn(len(s), 3, dtype=torch.float64, device="cuda")
    (imgv * wv).sum().backward()
    ref = volume_reference_gradient(segs, lp["fields"], len(s), wv.cpu().numpy())
    want = np.zeros_like(rgba)
    want[lp["orig_ids"]] = ref
    np.testing.assert_allclose(fv.grad.cpu().numpy(), want, rtol=1e-9,
                               atol=1e-12 * np.abs(want).max())
