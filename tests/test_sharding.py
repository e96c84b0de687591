"""Multi-rank ray sharding on CPU: two gloo ranks, each walking its block of
rays with the oracle, must reproduce the single-process image and the
single-process field gradient (sparse reference A^T g)."""
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


def _oracle_ops(pos, rho):
    import warnings
    import scipy.sparse as sp
    from oracle import oracle as O
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        lp = O.load_points(pos, rho, [0, 10] * 3)
    t = O.OracleTree(lp["pts"], lp["fields"])
    npart = len(lp["orig_ids"])

    def project(s, e):
        return t.project(s, e, "integrate", nthreads=1)

    def adjoint(s, e, out, g):
        _, (cid, se, sx, off) = t.project(s, e, "integrate", segments=True, nthreads=1)
        ray = np.repeat(np.arange(len(s)), np.diff(off))
        A = sp.csr_matrix((sx - se, (ray, cid)), shape=(len(s), npart))
        return np.asarray(A.T @ g)

    return project, adjoint


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from vortrace_b200.sharding import sharded_adjoint, sharded_project
        pos, rho, st, en = _case()
        project, adjoint = _oracle_ops(pos, rho)
        out = sharded_project(project, st, en)
        g = np.random.default_rng(1).normal(size=(len(st), 1))
        grad = sharded_adjoint(adjoint, st, en, out, g)
        q.put((rank, out, grad))
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
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pos, rho, st, en = _case()
    project, adjoint = _oracle_ops(pos, rho)
    ref = project(st, en)
    g = np.random.default_rng(1).normal(size=(len(st), 1))
    ref_grad = adjoint(st, en, ref, g)
    for _, out, grad in res:
        np.testing.assert_array_equal(out, ref)
        np.testing.assert_allclose(grad, ref_grad, rtol=1e-12, atol=1e-15)
