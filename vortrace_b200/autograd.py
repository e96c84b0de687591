"""Differentiable projections: gradients of images w.r.t. the per-cell fields.

The reference has no gradients.  Here the forward is the walk kernel and the
backward is the hand-written adjoint kernel (vt_project_adjoint_device):

* ``'integrate'``: dL/dfield[c, f] = sum over segments of ray r in cell c of
  dL/dimg[r, f] * ds.  When a gradient is needed the forward records a
  segment tape (16 bytes per crossing, vt_project_device_tape) and the
  backward is a scatter of it (vt_tape_adjoint_device); a tape that did not
  fit falls back to re-walking the rays;
* ``'volume'``: reverse-mode front-to-back compositing; the transmittance in
  front of every segment and the colour composited up to it come from the
  forward's tape (48 bytes per crossing), or are recomputed by re-walking the
  ray when the tape did not fit.

The cell geometry does not depend on the fields, so the segment lists are
the same in the forward and the backward walk.  PyTorch is only the autograd
shell; all arithmetic runs in libvortrace_b200.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .vortrace import ProjectionCloud


def _dev_ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def _take_tape(pc: ProjectionCloud) -> L.Tape:
    """A free tape of this cloud (its device buffer is reused), or a new one."""
    pool = pc.__dict__.setdefault("_tapes", [])
    return pool.pop() if pool else L.Tape(pc._cloud._lib, pc._cloud._h)


def _give_back_tape(pc: ProjectionCloud, tape: L.Tape) -> None:
    pool = pc.__dict__.setdefault("_tapes", [])
    if not pool:  # keep one free tape per cloud; others free their memory
        pool.append(tape)


class _ProjectFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fields_internal, pc: ProjectionCloud, starts, ends, mode, kernel):
        lib = pc._cloud._lib
        h = pc._cloud._h
        dev = starts.device
        f = fields_internal.detach().to(device=dev, dtype=torch.float64).contiguous()
        stream = torch.cuda.current_stream(dev).cuda_stream
        L.check(lib.vt_cloud_set_fields_device(h, _dev_ptr(f), stream))
        n = starts.shape[0]
        nout = 3 if mode == L.REDUCE_VOLUME else f.shape[1]
        out = torch.empty((n, nout), dtype=torch.float64, device=dev)
        st = L.Stats()
        tape = None
        if mode in (L.REDUCE_SUM, L.REDUCE_VOLUME) and ctx.needs_input_grad[0]:
            tape = _take_tape(pc)
            L.check(lib.vt_project_device_tape(h, tape.h, _dev_ptr(starts), _dev_ptr(ends), n,
                                               mode, kernel, _dev_ptr(out), stream,
                                               C.byref(st)))
        else:
            L.check(lib.vt_project_device(h, _dev_ptr(starts), _dev_ptr(ends), n, mode, kernel,
                                          _dev_ptr(out), stream, C.byref(st)))
        ctx.tape = tape
        pc.last_stats = st.as_dict()
        ctx.pc = pc
        ctx.mode = mode
        ctx.fields = f
        ctx.save_for_backward(starts, ends, out)
        return out

    @staticmethod
    def backward(ctx, gout):
        starts, ends, out = ctx.saved_tensors
        pc = ctx.pc
        lib = pc._cloud._lib
        h = pc._cloud._h
        dev = starts.device
        stream = torch.cuda.current_stream(dev).cuda_stream
        # the cloud may have been given other fields since the forward
        L.check(lib.vt_cloud_set_fields_device(h, _dev_ptr(ctx.fields), stream))
        g = gout.to(dtype=torch.float64).contiguous()
        grad = torch.zeros_like(ctx.fields)
        if ctx.tape is not None:
            L.check(lib.vt_tape_adjoint_device(h, ctx.tape.h, _dev_ptr(starts), _dev_ptr(ends),
                                               starts.shape[0], ctx.mode, _dev_ptr(out),
                                               _dev_ptr(g), _dev_ptr(grad), stream))
            _give_back_tape(pc, ctx.tape)
            ctx.tape = None
        else:
            L.check(lib.vt_project_adjoint_device(h, _dev_ptr(starts), _dev_ptr(ends),
                                                  starts.shape[0], ctx.mode, _dev_ptr(out),
                                                  _dev_ptr(g), _dev_ptr(grad), stream))
        return grad, None, None, None, None, None


def _rays_on(p, dev) -> torch.Tensor:
    """(R, 3) float64 rays on ``dev``: device tensors are used in place,
    host arrays copied once."""
    if isinstance(p, torch.Tensor):
        return p.to(device=dev, dtype=torch.float64).reshape(-1, 3).contiguous()
    a = np.ascontiguousarray(p, np.float64)
    return torch.as_tensor(a, device=dev).reshape(-1, 3).contiguous()


def project(pc: ProjectionCloud, fields: torch.Tensor, pos_start, pos_end, *,
            reduction: str = "integrate", kernel: str = "auto") -> torch.Tensor:
    """Differentiable :meth:`ProjectionCloud.projection`.

    ``fields``: tensor of shape (N,) or (N, nfields) over the ORIGINAL
    particles (the order of ``pos`` given to the cloud); only the particles
    kept by the bounding-box filter influence the result.  ``pos_start`` /
    ``pos_end``: (R, 3) rays, host arrays or tensors (device tensors are used
    without a copy).  Returns (R,) or (R, nout) float64 on the
    device of ``fields`` (must be a CUDA tensor).
    """
    mode = {"integrate": L.REDUCE_SUM, "sum": L.REDUCE_SUM, "volume": L.REDUCE_VOLUME,
            "max": L.REDUCE_MAX, "min": L.REDUCE_MIN}.get(reduction)
    if mode is None:
        raise ValueError(f"Unknown reduction {reduction!r}")
    if mode not in (L.REDUCE_SUM, L.REDUCE_VOLUME):
        raise ValueError("gradients are defined for 'integrate' and 'volume' only")
    if not fields.is_cuda:
        raise ValueError("fields must be a CUDA tensor")
    dev = fields.device
    f2 = fields.reshape(fields.shape[0], -1)
    if f2.shape[1] != pc._nfields:
        raise ValueError(f"fields has {f2.shape[1]} columns, the cloud {pc._nfields}")
    if mode == L.REDUCE_VOLUME and pc._nfields != 4:
        raise ValueError("Volume rendering requires exactly 4 fields "
                         f"(R, G, B, alpha), got {pc._nfields}")
    oid = torch.as_tensor(pc.orig_ids, device=dev, dtype=torch.long)
    fi = f2.index_select(0, oid)
    S, E = (_rays_on(p, dev) for p in (pos_start, pos_end))
    out = _ProjectFn.apply(fi, pc, S, E, mode, L.KERNELS[kernel])
    return out[:, 0] if (out.shape[1] == 1 and fields.dim() == 1) else out


def grid_project(pc: ProjectionCloud, fields: torch.Tensor, extent, nres, bounds, center, *,
                 reduction: str = "integrate", **angles) -> torch.Tensor:
    """Differentiable :meth:`ProjectionCloud.grid_projection`."""
    from . import grid as gr
    from .vortrace import device_grid_args
    args = None
    if center is None and fields.is_cuda:
        args = device_grid_args(extent, nres, bounds, angles.get("proj"))
    if args is not None:
        # the unrotated grid's rays made on the device (vt_grid_rays_device)
        e4, nx, ny, b = args
        dev = fields.device
        ps = torch.empty((nx * ny, 3), dtype=torch.float64, device=dev)
        pe = torch.empty_like(ps)
        stream = torch.cuda.current_stream(dev).cuda_stream
        with torch.cuda.device(dev):
            L.check(pc._cloud._lib.vt_grid_rays_device(L.dptr(e4), nx, ny, L.dptr(b),
                                                       _dev_ptr(ps), _dev_ptr(pe), stream))
        shape = (nx, ny)
    else:
        ps, pe = gr.generate_projection_grid(extent, nres, bounds, center, **angles)
        shape = ps.shape[:-1]
        ps, pe = ps.reshape(-1, 3), pe.reshape(-1, 3)
    out = project(pc, fields, ps, pe, reduction=reduction)
    return out.reshape(*shape, *out.shape[1:])
