"""Launch one walk kernel a few times on a benchmark workload, for profilers.

    python -m vortrace_b200.profile_walk --config clustered_2m --npix 512 \
        --kernel thread_fp32 --smem-levels 3 --launches 5

Builds the workload's cloud (``vortrace_b200.workloads``), then runs
``vt_project_device`` with the given kernel ``--launches`` times on the same
device-resident rays and prints the crossings and the last launch's walk
time.  No autotuning and no other kernel runs between the launches, so a
profiler's ``-k regex:<kernel> -s <n> -c 1`` selects the (n+1)-th launch of
that kernel.
"""
from __future__ import annotations

import argparse
import ctypes as C
import warnings

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--config", default="clustered_2m")
    ap.add_argument("--npix", type=int, default=None)
    ap.add_argument("--kernel", default="thread_fp32")
    ap.add_argument("--smem-levels", type=int, default=3)
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--launches", type=int, default=5)
    a = ap.parse_args(argv)

    import torch

    from . import _lib as L
    from . import workloads as W
    from .vortrace import ProjectionCloud

    w = W.CONFIGS[a.config]() if not a.npix else W.CONFIGS[a.config](npix=a.npix)
    mode = {"integrate": L.REDUCE_SUM, "volume": L.REDUCE_VOLUME}[w["reduction"]]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = ProjectionCloud(w["pos"], w["fields"], boundbox=w["boundbox"])
    lib, h = pc._cloud._lib, pc._cloud._h
    pc._cloud.set_param(L.PARAM_SMEM_LEVELS, a.smem_levels)
    pc._cloud.set_param(L.PARAM_BLOCKS_PER_SM, a.blocks_per_sm)
    dev = torch.device("cuda", 0)
    d_s = torch.from_numpy(np.ascontiguousarray(w["starts"])).to(dev)
    d_e = torch.from_numpy(np.ascontiguousarray(w["ends"])).to(dev)
    n = d_s.shape[0]
    nout = 3 if mode == L.REDUCE_VOLUME else pc._nfields
    out = torch.empty((n, nout), dtype=torch.float64, device=dev)
    st = L.Stats()
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(a.launches):
        L.check(lib.vt_project_device(h, d_s.data_ptr(), d_e.data_ptr(), n, mode,
                                      L.KERNELS[a.kernel], out.data_ptr(), stream, C.byref(st)))
    print(f"{a.config} npix={a.npix} kernel={a.kernel} rays={n} crossings={st.crossings} "
          f"walk_ms={st.walk_ms:.3f}", flush=True)


if __name__ == "__main__":
    main()
