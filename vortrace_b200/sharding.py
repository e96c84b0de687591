"""Ray sharding over GPUs (one process per GPU, torch.distributed).

The walk shards by rays: every rank holds the whole cloud and tree (16M
points take under 1 GB of HBM) and walks a contiguous block of the rays.
The forward needs no exchange until the image is assembled (one all-gather
of the rank blocks, on the device); the adjoint of a loss over all rays
needs one all-reduce (sum) of the N x nfields FP64 field gradient, also on
the device.  Nothing crosses to the host: the rank's block of rays, its
image rows, the gathered image and the gradient stay in device memory, and
NCCL moves them between GPUs.

``sharded_projection`` is differentiable.  Its projector defaults to
:func:`vortrace_b200.autograd.project` (the taped forward and the scatter
adjoint of libvortrace_b200); any differentiable ``projector(fields, starts,
ends) -> (n, nout)`` can stand in for it, which is how the collectives are
tested with gloo ranks on the CPU.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous block of n items owned by `rank` (sizes differ by <= 1)."""
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _world(group):
    return dist.get_world_size(group), dist.get_rank(group)


class _GatherRows(torch.autograd.Function):
    """All-gather of the ranks' contiguous row blocks into the full (n, k)
    tensor on every rank; the backward hands each rank the gradient rows of
    its own block (the other rows belong to the other ranks' walks)."""

    @staticmethod
    def forward(ctx, local, n, group):
        world, rank = _world(group)
        a, b = shard_range(n, rank, world)
        if local.shape[0] != b - a:
            raise ValueError(f"rank {rank} holds {local.shape[0]} rows, its block is {b - a}")
        ctx.block = (a, b)
        cap = -(-n // world) if world else 0
        k = local.shape[1]
        send = local.new_zeros((cap, k))
        send[: b - a] = local
        recv = local.new_empty((world * cap, k))
        dist.all_gather_into_tensor(recv, send, group=group)
        parts = []
        for r in range(world):
            ra, rb = shard_range(n, r, world)
            parts.append(recv[r * cap: r * cap + (rb - ra)])
        return torch.cat(parts, 0)

    @staticmethod
    def backward(ctx, g):
        a, b = ctx.block
        return g[a:b], None, None


class _SumGradOverRanks(torch.autograd.Function):
    """Identity in the forward; the backward sums the incoming gradient over
    the ranks (one all-reduce), so every rank ends with the gradient of the
    loss over all rays."""

    @staticmethod
    def forward(ctx, x, group):
        ctx.group = group
        return x.view_as(x)

    @staticmethod
    def backward(ctx, g):
        g = g.contiguous()
        dist.all_reduce(g, op=dist.ReduceOp.SUM, group=ctx.group)
        return g, None


def _rows(x, a, b, device):
    """Rows [a, b) of a ray array as a float64 tensor on `device` (device
    tensors are sliced in place; host arrays copy only this block)."""
    if isinstance(x, torch.Tensor):
        return x[a:b].to(device=device, dtype=torch.float64)
    return torch.as_tensor(x[a:b], dtype=torch.float64, device=device)


def sharded_projection(pc, fields, starts, ends, *, reduction="integrate", kernel="auto",
                       group=None, projector=None):
    """Differentiable projection of all rays, each rank walking its block.

    ``fields``: (N,) or (N, nfields) tensor over the original particles, the
    same on every rank (a CUDA tensor for the default projector).
    ``starts`` / ``ends``: (R, 3), the full ray set (host arrays or
    tensors); each rank walks rows ``shard_range(R, rank, world)``.
    Returns the full (R,) or (R, nout) image on every rank.  Backward: the
    gradient w.r.t. ``fields`` of a loss over the whole image, summed over
    the ranks' walks by one all-reduce.
    """
    world, rank = _world(group)
    n = starts.shape[0]
    if ends.shape[0] != n:
        raise ValueError("starts and ends must hold the same number of rays")
    a, b = shard_range(n, rank, world)
    if projector is None:
        from . import autograd as ag

        def projector(f, s, e):
            return ag.project(pc, f, s, e, reduction=reduction, kernel=kernel)
    f = _SumGradOverRanks.apply(fields, group)
    s = _rows(starts, a, b, fields.device)
    e = _rows(ends, a, b, fields.device)
    local = projector(f, s, e)
    flat = local.dim() == 1
    full = _GatherRows.apply(local.reshape(b - a, -1), n, group)
    return full[:, 0] if flat else full
