"""Multi-rank ray sharding on CPU: two gloo ranks, each walking its block of
rays (the reference's segment matrix stands in for the walk), must each end
with the single-process image and the field gradient of a loss over all
rays (A^T W), through the same all-gather and gradient all-reduce that run
on the device with NCCL."""
import os
import socket

import numpy as np
import pytest

from vortrace_b200.sharding import shard_range


def test_shard_range_partitions():
    for n in (0, 1, 7, 100, 1001):
        for w in (1, 2, 3, 8):
            blocks = [shard_range(n, r, w) for r in range(w)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(blocks[i][1] == blocks[i + 1][0] for i in range(w - 1))
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    rng = np.random.default_rng(8)
    pos = rng.uniform(0, 10, (3000, 3))
    rho = rng.lognormal(0, 1, 3000)
    st = rng.uniform(0, 10, (301, 3))
    en = rng.uniform(0, 10, (301, 3))
    return pos, rho, st, en


def _oracle_matrix(pos, rho, st, en):
    """The reference's segment lists as a dense (rays x particles) matrix of
    segment lengths, columns in the original particle order: image = A @
    rho, gradient of sum(W * image) = A^T W."""
    import warnings
    from oracle import oracle as O
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        lp = O.load_points(pos, rho, [0, 10] * 3)
    t = O.OracleTree(lp["pts"], lp["fields"])
    img, (cid, se, sx, off) = t.project(st, en, "integrate", segments=True, nthreads=1)
    ray = np.repeat(np.arange(len(st)), np.diff(off))
    A = np.zeros((len(st), len(pos)))
    np.add.at(A, (ray, np.asarray(lp["orig_ids"])[cid]), sx - se)
    return A, img


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from vortrace_b200.sharding import sharded_projection
        pos, rho, st, en = _case()
        A, _ = _oracle_matrix(pos, rho, st, en)
        At = torch.from_numpy(A)
        calls = []

        def projector(f, s, e):
            # this rank's rows of the reference matrix, found from its rays
            a = int(np.flatnonzero((st == s[0].numpy()).all(1))[0])
            calls.append((a, s.shape[0]))
            return At[a:a + s.shape[0]] @ f

        f = torch.from_numpy(rho).requires_grad_(True)
        img = sharded_projection(None, f, st, en, projector=projector)
        W = torch.from_numpy(np.random.default_rng(1).normal(size=len(st)))
        (W * img).sum().backward()
        q.put((rank, calls, img.detach().numpy(), f.grad.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_single_process():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in range(2)], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pos, rho, st, en = _case()
    A, ref = _oracle_matrix(pos, rho, st, en)
    W = np.random.default_rng(1).normal(size=len(st))
    # each rank walked its own contiguous block, once
    for k, calls, _, _ in res:
        a, b = shard_range(len(st), k, 2)
        assert calls == [(a, b - a)]
    for _, _, img, grad in res:
        # every rank holds the whole image and the gradient over all rays
        np.testing.assert_allclose(img, ref[:, 0], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(grad, A.T @ W, rtol=1e-12, atol=1e-15)


def _single(fn):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        fn()
    finally:
        dist.destroy_process_group()


def test_argument_rules():
    import torch

    from vortrace_b200.sharding import _GatherRows, sharded_projection

    def body():
        f = torch.ones(4, dtype=torch.float64)
        st = np.zeros((3, 3))
        with pytest.raises(ValueError, match="same number of rays"):
            sharded_projection(None, f, st, np.zeros((2, 3)), projector=lambda *a: None)
        with pytest.raises(ValueError, match="its block is 3"):
            _GatherRows.apply(torch.zeros((2, 1), dtype=torch.float64), 3, None)
        # one rank: the projector sees every ray, as float64 tensors on the
        # device of the fields, and the image comes back unchanged
        seen = []

        def proj(fl, s, e):
            seen.append((s.dtype, s.device, tuple(s.shape), tuple(e.shape)))
            return fl[:3] * 2.0
        out = sharded_projection(None, f, st, st, projector=proj)
        assert seen == [(torch.float64, f.device, (3, 3), (3, 3))]
        assert out.shape == (3,) and torch.equal(out, torch.full((3,), 2.0, dtype=torch.float64))
    _single(body)
