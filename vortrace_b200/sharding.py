"""Ray sharding over GPUs (one process per GPU, torch.distributed).

The walk shards by rays: every rank holds the whole cloud and tree (16M
points take under 1 GB of HBM) and walks a contiguous block of the rays.
The forward needs no exchange until the image is assembled (all-gather);
the adjoint of a shared loss needs one all-reduce (sum) of the N x nfields
FP64 field gradient.

The projector is passed in (``project(starts, ends) -> (n, nout) array`` and
``adjoint(starts, ends, out, gout) -> (npart, nf) array``), so the same code
drives the CUDA library on GPU ranks and any CPU implementation on gloo ranks.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous block of n items owned by `rank` (sizes differ by <= 1)."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def sharded_project(project, starts, ends, group=None):
    """Walk this rank's block of rays and all-gather the full result."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n = starts.shape[0]
    a, b = shard_range(n, rank, world)
    local = np.ascontiguousarray(project(starts[a:b], ends[a:b]))
    nout = local.shape[1] if local.ndim == 2 else 1
    cap = -(-n // world)
    buf = np.zeros((cap, nout))
    buf[: b - a] = local.reshape(b - a, nout)
    t = torch.from_numpy(buf)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    out = np.empty((n, nout))
    for r, p in enumerate(parts):
        ra, rb = shard_range(n, r, world)
        out[ra:rb] = p.cpu().numpy()[: rb - ra]
    return out


def sharded_adjoint(adjoint, starts, ends, out, gout, group=None):
    """Field gradient of a loss over all rays: local adjoint + all-reduce."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    a, b = shard_range(starts.shape[0], rank, world)
    g = np.ascontiguousarray(adjoint(starts[a:b], ends[a:b], out[a:b], gout[a:b]))
    t = torch.from_numpy(g)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()
