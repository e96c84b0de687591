"""Device-resident ray sharding on one GPU: a one-rank NCCL group runs the
same all-gather of the image rows and all-reduce of the field gradient that
N ranks run, on CUDA tensors.  The image and the gradient must equal the
unsharded differentiable projection's bit for bit (one rank: the collectives
copy and sum nothing else)."""
import os
import socket
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("reduction", ["integrate", "volume"])
def test_one_rank_nccl_matches_unsharded(reduction):
    import torch
    import torch.distributed as dist

    import vortrace_b200 as vt
    from vortrace_b200 import autograd as ag
    from vortrace_b200 import workloads as W
    from vortrace_b200.sharding import sharded_projection

    dev = torch.device("cuda", 0)
    pos, f = W.clustered_cloud(100_000, 31, nf=3)
    fields = W.transfer_rgba(f[:, 0]) if reduction == "volume" else f
    s, e = W.z_grid([44.0, 56.0], 48)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = vt.ProjectionCloud(pos, fields, boundbox=W.BOX)
    ft = torch.tensor(fields, device=dev, requires_grad=True)
    img_ref = ag.project(pc, ft, s, e, reduction=reduction)
    wgt = torch.randn(img_ref.shape, dtype=torch.float64, device=dev,
                      generator=torch.Generator(device=dev).manual_seed(3))
    (wgt * img_ref).sum().backward()
    g_ref = ft.grad.clone()
    ft.grad = None

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=dev)
    try:
        d_s = torch.from_numpy(s).to(dev)
        d_e = torch.from_numpy(e).to(dev)
        img = sharded_projection(pc, ft, d_s, d_e, reduction=reduction)
        (wgt * img).sum().backward()
        torch.cuda.synchronize(dev)
        assert img.device == dev and ft.grad.device == dev
        assert torch.equal(img, img_ref.detach())
        # the scatter adjoint adds with atomics: same sums, any order
        gr = g_ref.cpu().numpy()
        np.testing.assert_allclose(ft.grad.cpu().numpy(), gr, rtol=1e-12,
                                   atol=1e-12 * np.abs(gr).max())
    finally:
        dist.destroy_process_group()
