"""Field gradients at the size of the volume-rendering configuration: the
2,000,000-point clustered cloud, RGBA from the three-band transfer function,
a 512x512 'volume' image, loss = sum(W * img) with W ~ N(0, 1) per pixel and
channel.  The gradient of the differentiable path (taped forward + scatter
adjoint, through torch.autograd) is compared with

  * the reverse-mode compositing gradient evaluated in numpy on the oracle's
    segment lists (bit-identical to the reference's makeDetailedProjection),
    for every cell (rtol 1e-9), and
  * central finite differences of the loss on 64 random cells (rtol 1e-6).
"""
import warnings

import numpy as np
import pytest

import vortrace_b200 as vt
from oracle import oracle as O
from tests.test_gpu_adjoint import FD_RTOL, fd_column
from vortrace_b200 import workloads as W

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def volume_gradient_chunked(segs, fields, nrays, gout, chunk=8192):
    """Reverse-mode compositing gradient (the formulas of the reference's
    front-to-back compositing, src/reduction.cpp:55-83, differentiated), rays
    processed in chunks as rows of a padded array: per ray the same
    transmittance products and suffix sums as a per-ray loop (padding adds
    exact zeros / ones)."""
    cid, se, sx, off = segs
    ds_all = sx - se
    npart = fields.shape[0]
    grad = np.zeros_like(fields)
    for r0 in range(0, nrays, chunk):
        r1 = min(nrays, r0 + chunk)
        cnt = np.diff(off[r0:r1 + 1])
        m = int(cnt.max()) if len(cnt) else 0
        if m == 0:
            continue
        rows = np.repeat(np.arange(r1 - r0), cnt)
        cols = np.arange(int(off[r1] - off[r0])) - np.repeat(off[r0:r1] - off[r0], cnt)
        seg = slice(int(off[r0]), int(off[r1]))
        c = cid[seg]
        ds = np.zeros((r1 - r0, m))
        a = np.zeros((r1 - r0, m))
        rgb = np.zeros((r1 - r0, m, 3))
        ds[rows, cols] = ds_all[seg]
        a[rows, cols] = fields[c, 3]
        rgb[rows, cols] = fields[c, :3]
        o = 1.0 - np.exp(-a * ds)
        T = np.ones_like(o)
        T[:, 1:] = np.cumprod(1.0 - o, axis=1)[:, :-1]
        contrib = (T * o)[:, :, None] * rgb
        suffix = np.cumsum(contrib[:, ::-1], axis=1)[:, ::-1] - contrib
        g = gout[r0:r1][:, None, :]
        d_rgb = (T * o)[:, :, None] * g
        d_a = ds * np.sum(g * (T[:, :, None] * rgb * (1.0 - o)[:, :, None] - suffix), axis=2)
        for k in range(3):
            grad[:, k] += np.bincount(c, weights=d_rgb[rows, cols, k], minlength=npart)
        grad[:, 3] += np.bincount(c, weights=d_a[rows, cols], minlength=npart)
    return grad


def test_volume_2m_gradient():
    import torch

    from vortrace_b200 import autograd as VA

    w = W.volume_2m()
    s, e = w["starts"], w["ends"]
    n = len(s)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = vt.ProjectionCloud(w["pos"], w["fields"], boundbox=W.BOX)
        lp = O.load_points(w["pos"], w["fields"], W.BOX)
    ot = O.OracleTree(lp["pts"], lp["fields"], lp["valid_rgba"])
    out, segs = ot.project(s, e, "volume", segments=True)
    del ot
    wts = np.random.default_rng(33).normal(size=(n, 3))

    f = torch.tensor(w["fields"], dtype=torch.float64, device="cuda", requires_grad=True)
    img = VA.project(pc, f, s, e, reduction="volume")
    np.testing.assert_allclose(img.detach().cpu().numpy(), out, rtol=1e-12, atol=1e-300)
    (img * torch.as_tensor(wts, device="cuda")).sum().backward()
    grad_orig = f.grad.cpu().numpy()
    grad = grad_orig[lp["orig_ids"]]            # internal (filtered) order

    ref = volume_gradient_chunked(segs, lp["fields"], n, wts)
    np.testing.assert_allclose(grad, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())

    # central finite differences on 64 random cells the image resolves
    fint = lp["fields"].copy()
    inner = np.all((fint[:, :3] > 0.01) & (fint[:, :3] < 0.99), axis=1) & (fint[:, 3] > 1e-3)
    rng = np.random.default_rng(34)
    comp = rng.integers(0, 4, len(fint))
    resolvable = np.abs(grad[np.arange(len(fint)), comp]) >= 1e-8 * np.abs(grad).max()
    cells = rng.choice(np.nonzero(inner & resolvable)[0], 64, replace=False)
    for c in cells:
        k = int(comp[c])
        h = 1e-5 * max(1.0, abs(fint[c, k]))
        fd = fd_column(pc, fint, s, e, "volume", wts, c, k, h)
        np.testing.assert_allclose(fd, grad[c, k], rtol=FD_RTOL)
