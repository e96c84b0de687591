#!/usr/bin/env python
"""Benchmark of the exact Voronoi ray walk on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config clustered_2m]

One step = one projection of the workload's rays through the cloud (the
cloud and its device tree are built once, outside the timed region, as the
reference's timing of Projection::makeProjection excludes buildTree).
Prints one JSON line (rank 0).

Metric: cell crossings per second (Mcrossings/s) of the batched kernel
(VT_KERNEL_AUTO after vt_cloud_autotune on the workload's rays: persistent,
one ray per thread in a coherent sorted order with the bounded guarded-FP32
or FP64 k-NN, or one ray per warp for small batches), forward; the same
line reports forward+adjoint, the bounded-FP64 variant of the batched
kernel and the plain FP64 one-ray-per-thread kernel.  Multi-GPU (torchrun): every rank projects its own
view of the cloud (the grid rotated about the cloud centre by 2*pi*rank/N):
weak scaling, no data-path collective; value = all ranks' crossings / max
over ranks of the timed device time.

``--impl reference`` times the reference's own CPU implementation (its
Cvortrace module compiled from its sources into oracle/_ref, OpenMP over all
host cores; the C restatement in oracle/ when that module is absent) on a
bounded sample of the same rays.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
import warnings

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcrossings/s fwd & fwd+bwd: batched guarded-FP32 vs plain FP64 GPU kernel"
UNIT = "Mcrossings/s"
# Algorithmic bytes per cell crossing, B_x = Q*(n_node*16 + n_pt*24) + nf*8 + 48,
# measured with the nanoflann restatement (oracle/measure_bx.py, 8192-ray sample).
BX = {"clustered_2m": 3262.25, "uniform_100k": 2915.74, "volume_2m": 3273.36,
      "batched_1m": 3201.12, "nested_16m": 3320.48}
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per crossing of
# the walk kernel, from one single-pass ncu capture of the same launch
# (clustered_2m, 1024x1024 rays, guarded-FP32 kernel at 9 blocks per SM with
# 3 tree levels in shared memory, vortrace_b200.profile_walk: 63.70 GB read
# + 66.01 GB written for 198,903,587 crossings; the writes are local memory,
# as the image is 25 MB: the spill and stack slots of 170K resident threads
# outgrow the L2), keyed by
# (workload, AUTO kernel); other launches of the kernel are taken to scale
# with their crossings.
DRAM_BYTES_PER_CROSSING = {("clustered_2m", "thread_fp32"): 652.15}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.lines = []
        self.proc = None
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.idx)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.th:
            self.th.join(timeout=5)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = max(smax, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(name, rank, world, npix=None):
    from vortrace_b200 import workloads as W
    from vortrace_b200 import grid as gr
    w = W.CONFIGS[name]() if not npix else W.CONFIGS[name](npix=npix)
    if world > 1 and rank > 0:
        # weak scaling: each rank projects its own view (rotated about the centre)
        c = np.array([50.0, 50.0, 50.0])
        R = gr.rotation_matrix(2 * np.pi * rank / world, 0.0, 0.0)
        w["starts"] = np.ascontiguousarray((w["starts"] - c) @ R.T + c)
        w["ends"] = np.ascontiguousarray((w["ends"] - c) @ R.T + c)
    return w


def cpu_reference_run(w, steps, nsample, warmup=0):
    """Time the reference's own CPU path on a sample of the rays.

    Returns (Mcrossings/s, crossings per step, seconds per step, kind,
    rays in the sample)."""
    from oracle import oracle as O
    n = w["starts"].shape[0]
    idx = np.linspace(0, n - 1, min(nsample, n)).astype(np.int64)
    S = np.ascontiguousarray(w["starts"][idx])
    E = np.ascontiguousarray(w["ends"][idx])
    mod = O.load_reference_module()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        if mod is not None:
            kind = "reference"
            pc = mod.PointCloud()
            pc.loadPoints(np.ascontiguousarray(w["pos"], np.float64),
                          np.ascontiguousarray(w["fields"], np.float64), list(w["boundbox"]))
            pc.buildTree()
            mode = {"integrate": mod.ReductionMode.Sum,
                    "volume": mod.ReductionMode.VolumeRender}[w["reduction"]]
            pr = mod.Projection(S, E)
            pr.makeDetailedProjection(pc, mode)
            crossings = int(pr.returnSegments()[3][-1])

            def step():
                p = mod.Projection(S, E)
                p.makeProjection(pc, mode)
                return p.returnProjection()
        else:
            kind = "port"
            lp = O.load_points(w["pos"], w["fields"], w["boundbox"])
            t = O.OracleTree(lp["pts"], lp["fields"], lp["valid_rgba"])
            _, segs = t.project(S, E, w["reduction"], segments=True)
            crossings = int(segs[3][-1])

            def step():
                return t.project(S, E, w["reduction"])
    for _ in range(warmup):
        step()
    times = []
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    sec = statistics.mean(times)
    return crossings / sec / 1e6, crossings, sec, kind, len(idx)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    w = make_workload(args.config, 0, 1)
    val, cross, sec, kind, ns = cpu_reference_run(w, args.steps, args.cpu_sample,
                                                  warmup=args.warmup)
    cores = host_cores()
    n = w["starts"].shape[0]
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 4), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.config}: {w['meta']}",
                   "sample": f"{ns} of {n} rays (evenly spaced)", "crossings_per_step": cross},
        "cpu_baseline": {"value": round(val, 4), "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{ns} of {n} rays of {args.config}, OpenMP over all host "
                                   "cores, tree build excluded"},
        "e2e": {"value": round(val, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def oracle_sample_parity(w, pc, kernel, nsample=4096):
    """Outside the timed region: the walk kernel's CSR segments of an evenly
    spaced sample of the workload's rays against the oracle (the C
    restatement of the reference, pinned to the reference module), and its
    per-ray values against the oracle's."""
    from oracle import oracle as O
    n = w["starts"].shape[0]
    idx = np.linspace(0, n - 1, min(nsample, n)).astype(np.int64)
    S = np.ascontiguousarray(w["starts"][idx])
    E = np.ascontiguousarray(w["ends"][idx])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        lp = O.load_points(w["pos"], w["fields"], w["boundbox"])
    t = O.OracleTree(lp["pts"], lp["fields"], lp["valid_rgba"])
    oout, (ocid, ose, osx, ooff) = t.project(S, E, w["reduction"], segments=True)
    del t
    old = pc.kernel
    pc.kernel = kernel
    try:
        vals, cid, se, ds, off = pc.traced_projection(S, E, return_midpoint=False,
                                                      reduction=w["reduction"], flatten=True)
    finally:
        pc.kernel = old
    seg_ok = (np.array_equal(off, ooff) and np.array_equal(cid, lp["orig_ids"][ocid])
              and np.array_equal(se, ose) and np.array_equal(ds, osx - ose))
    v = np.asarray(vals).reshape(len(idx), -1)
    o = oout.reshape(len(idx), -1)
    rel = np.abs(v - o) / np.maximum(np.abs(o), 1e-300)
    return {"sample_rays": int(len(idx)), "sample_crossings": int(ooff[-1]),
            "segments_bit_identical_to_oracle": bool(seg_ok),
            "values_bit_identical_to_oracle": bool(np.array_equal(v, o)),
            "values_max_rel_err_vs_oracle": float(rel.max()) if rel.size else 0.0}, idx, o


def counters_run(w, kernel, tune, mode):
    """One forward of the guarded-FP32 kernel through the library built
    with the search counters (libvortrace_b200_counters.so), outside the
    timed region, on a tree and launch configured as the autotuner chose:
    nodes visited, FP64 re-checks and the queries that needed one."""
    from vortrace_b200 import _lib as L
    from vortrace_b200 import build as B
    if not os.path.exists(B.LIB_COUNTERS):
        return None
    lib = L.load_variant(B.LIB_COUNTERS)
    pos = np.ascontiguousarray(w["pos"], np.float64)
    f = np.ascontiguousarray(w["fields"], np.float64)
    nf = 1 if f.ndim == 1 else f.shape[1]
    sb = np.ascontiguousarray(w["boundbox"], np.float64)
    h = C.c_void_p()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        L.check(lib.vt_cloud_create(L.dptr(pos), pos.shape[0], L.dptr(f), pos.shape[0], nf,
                                    L.dptr(sb), None, 0, 0, C.byref(h)), lib)
    try:
        L.check(lib.vt_cloud_set_param(h, L.PARAM_LEAF_SIZE, int(tune["leaf_size"])), lib)
        L.check(lib.vt_cloud_build_tree(h), lib)
        L.check(lib.vt_cloud_set_param(h, L.PARAM_SMEM_LEVELS, int(tune["smem_levels"])), lib)
        L.check(lib.vt_cloud_set_param(h, L.PARAM_BLOCKS_PER_SM, int(tune["blocks_per_sm"])),
                lib)
        S = np.ascontiguousarray(w["starts"])
        E = np.ascontiguousarray(w["ends"])
        n = S.shape[0]
        nout = 3 if mode == L.REDUCE_VOLUME else nf
        out = np.empty((n, nout))
        st = L.Stats()
        L.check(lib.vt_project(h, L.dptr(S), L.dptr(E), n, mode, kernel, L.dptr(out),
                               C.byref(st)), lib)
    finally:
        lib.vt_cloud_destroy(h)
    q32 = max(1, st.fp32_queries)
    return {"kernel": "k_batched guarded-FP32 (library built with VT_BATCHED_COUNTERS=1)",
            "queries": int(st.queries), "fp32_split_queries": int(st.fp32_queries),
            "nodes_per_query": round(st.search_steps / max(1, st.queries), 3),
            "fp64_rechecks_per_query": round(st.fp64_checks / q32, 4),
            "queries_with_fp64_recheck_fraction": round(st.fp64_check_queries / q32, 6),
            "fp64_full_resolves": int(st.fp64_resolves),
            "fp64_full_resolve_fraction": round(st.fp64_resolves / max(1, st.queries), 8),
            "search_simd_efficiency": round(st.search_lane_steps /
                                            max(1, 32 * st.search_warp_steps), 4),
            "trip_cycle_shares": [round(x / max(1, sum(st.trip_cycles)), 4)
                                  for x in st.trip_cycles]}


def measure(name, args, rank, world, dev, K, W, *, kp=None, wp=None, full=True,
            npix=None):
    """All legs of one workload.  K/W: timed and warm-up steps of the
    headline legs; kp/wp: of the baseline legs (default max(2, K//2) / 1).
    full: also the end-to-end leg through host buffers and the CPU leg."""
    import torch

    import vortrace_b200 as vt
    from vortrace_b200 import _lib as L

    kp = kp if kp is not None else max(2, K // 2)
    wp = wp if wp is not None else 1
    w = make_workload(name, rank, world, npix)
    mode = {"integrate": L.REDUCE_SUM, "volume": L.REDUCE_VOLUME}[w["reduction"]]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pc = vt.ProjectionCloud(w["pos"], w["fields"], boundbox=w["boundbox"])
    lib = pc._cloud._lib
    h = pc._cloud._h
    build_cold = pc._cloud.info().tree_build_ms
    pc._cloud.buildTree()   # warm: module loading and CUB scratch already done
    info = pc._cloud.info()
    nf = int(info.nfields)
    nout = 3 if mode == L.REDUCE_VOLUME else nf
    S = np.ascontiguousarray(w["starts"])
    E = np.ascontiguousarray(w["ends"])
    n = S.shape[0]
    d_s = torch.from_numpy(S).to(dev)
    d_e = torch.from_numpy(E).to(dev)
    d_out = torch.empty((n, nout), dtype=torch.float64, device=dev)
    d_gout = torch.ones((n, nout), dtype=torch.float64, device=dev)
    d_grad = torch.zeros((int(info.npart), nf), dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    st = L.Stats()

    def fwd(kernel):
        L.check(lib.vt_project_device(h, d_s.data_ptr(), d_e.data_ptr(), n, mode, kernel,
                                      d_out.data_ptr(), stream.cuda_stream, C.byref(st)))
        return st.crossings, st.walk_ms

    def bwd():
        L.check(lib.vt_project_adjoint_device(h, d_s.data_ptr(), d_e.data_ptr(), n, mode,
                                              d_out.data_ptr(), d_gout.data_ptr(),
                                              d_grad.data_ptr(), stream.cuda_stream))

    # forward with a segment tape + scatter adjoint (the autograd path of
    # 'integrate' and 'volume'), with any walk kernel
    tape = L.Tape(lib, h)

    def fwd_tape(kernel):
        L.check(lib.vt_project_device_tape(h, tape.h, d_s.data_ptr(), d_e.data_ptr(), n, mode,
                                           kernel, d_out.data_ptr(), stream.cuda_stream,
                                           C.byref(st)))

    def bwd_tape():
        L.check(lib.vt_tape_adjoint_device(h, tape.h, d_s.data_ptr(), d_e.data_ptr(), n, mode,
                                           d_out.data_ptr(), d_gout.data_ptr(),
                                           d_grad.data_ptr(), stream.cuda_stream))

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize(dev)

    def timed(fn, steps):
        """Per-step device time (ms) with CUDA events on the launching stream;
        L2 flushed before every step (outside the events)."""
        ms = []
        for i in range(steps):
            flush.fill_(i & 0xff)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms

    def reduce(x, op):
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def leg(fn, steps, warm):
        for _ in range(warm):
            fn()
        barrier()
        ms = timed(fn, steps)
        barrier()
        import torch.distributed as dist
        return reduce(sum(ms), dist.ReduceOp.MAX if world > 1 else None)

    def rate(t_ms, steps):
        return tot_cross * steps / (t_ms / 1e3) / 1e6

    def grad_sum():
        # a loss over every rank's rays: each forward+adjoint step ends with
        # the field gradient summed over the ranks on the device (one NCCL
        # all-reduce of the N x nf FP64 gradient)
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(d_grad, op=dist.ReduceOp.SUM)

    # --- autotune (outside the timed region): the AUTO kernel, the
    # shared-memory tree depth, the resident blocks per SM and the leaf size
    # from timings on a sample of this workload's rays
    # (a sample of up to 2^20 rays: the whole 1024^2 image, a quarter of the
    # 2048^2 one; leaf sizes are not tuned here: on a 262,144-ray sample of
    # nested_16m leaf 6 with the FP64 search won, 5% slower than leaf 8 at
    # full size)
    tune = pc.autotune(S, E, reduction={L.REDUCE_VOLUME: "volume"}.get(mode, "integrate"),
                       max_sample=min(n, 1 << 20))
    auto_kernel = tune["kernel"] if n >= tune["sample_rays"] else (
        "batched" if n < 65536 else "thread_fp32")

    # --- forward, batched kernel (the headline), clocks sampled meanwhile
    for _ in range(W):
        fwd(L.KERNEL_AUTO)
    barrier()
    sampler = ClockSampler(int(str(dev).split(":")[-1]))
    sampler.start()
    walk_ms = []

    def f_b():
        walk_ms.append(fwd(L.KERNEL_AUTO)[1])

    fwd_ms = timed(f_b, K)
    barrier()
    clocks = sampler.stop()
    crossings, _ = fwd(L.KERNEL_AUTO)
    img_auto = d_out.clone()
    import torch.distributed as dist
    t_fwd = reduce(sum(fwd_ms), dist.ReduceOp.MAX if world > 1 else None)
    tot_cross = reduce(float(crossings), dist.ReduceOp.SUM if world > 1 else None)
    value = rate(t_fwd, K)

    taped = mode in (L.REDUCE_SUM, L.REDUCE_VOLUME)
    # --- forward + adjoint: taped forward (AUTO) + scatter adjoint
    t_fb = leg(lambda: (fwd_tape(L.KERNEL_AUTO), bwd_tape(), grad_sum()), K, max(2, W // 2))
    fb_value = rate(t_fb, K)
    tape_entries = int(lib.vt_tape_size(tape.h))
    # --- forward + adjoint that re-walks the rays (no tape), AUTO kernel
    t_rw = leg(lambda: (fwd(L.KERNEL_AUTO), bwd(), grad_sum()), kp, wp)
    rw_value = rate(t_rw, kp)
    # --- the batched kernel with the bounded FP64 k-NN
    t_f64 = leg(lambda: fwd(L.KERNEL_BATCHED_FP64), kp, wp)
    f64_value = rate(t_f64, kp)
    # --- plain FP64 one-ray-per-thread kernel (the baseline kernel)
    t_pl = leg(lambda: fwd(L.KERNEL_PLAIN_FP64), kp, wp)
    pl_value = rate(t_pl, kp)
    fwd(L.KERNEL_PLAIN_FP64)
    img_plain = d_out.clone()
    # --- the plain kernel's forward + adjoint, like for like: taped plain
    # forward + the same scatter adjoint
    t_ptb = leg(lambda: (fwd_tape(L.KERNEL_PLAIN_FP64), bwd_tape(), grad_sum()), kp, wp)
    ptb_value = rate(t_ptb, kp)
    # --- ... and with the plain kernel re-walking for the adjoint
    pc._cloud.set_param(L.PARAM_ADJOINT_KERNEL, L.KERNEL_PLAIN_FP64)
    t_pfb = leg(lambda: (fwd(L.KERNEL_PLAIN_FP64), bwd(), grad_sum()), kp, wp)
    pc._cloud.set_param(L.PARAM_ADJOINT_KERNEL, L.KERNEL_AUTO)
    pfb_value = rate(t_pfb, kp)

    rec = {
        "workload": f"{name}: {w['meta']}", "rays_per_gpu": n, "reduction": w["reduction"],
        "crossings_per_step": int(tot_cross), "value": round(value, 4),
        "ms_per_step": round(t_fwd / K, 3), "steps": K, "warmup": W,
        "baseline_steps": kp, "baseline_warmup": wp,
        "rays_per_s": round(n * world * K / (t_fwd / 1e3), 1),
        "kernel": f"VT_KERNEL_AUTO = {auto_kernel}", "autotune": tune,
        "fwd_bwd_mcrossings_per_s": round(fb_value, 4),
        "fwd_bwd_adjoint": (f"segment tape ({48 if mode == L.REDUCE_VOLUME else 16} "
                            "B/crossing) + scatter" if taped and tape_entries > 0
                            else "re-walk"),
        "fwd_bwd_gradient_exchange": ("all-reduce (sum) of the N x nf FP64 field gradient "
                                      f"over {world} ranks on the device (NCCL), every step"
                                      if world > 1 else "none (1 rank)"),
        "fwd_bwd_rewalk_mcrossings_per_s": round(rw_value, 4),
        "bounded_fp64_mcrossings_per_s": round(f64_value, 4),
        "plain_fp64_mcrossings_per_s": round(pl_value, 4),
        "speedup_vs_plain_fp64": round(value / pl_value, 3),
        "plain_fp64_taped_fwd_bwd_mcrossings_per_s": round(ptb_value, 4),
        "fwd_bwd_speedup_vs_plain_fp64_taped": round(fb_value / ptb_value, 3),
        "plain_fp64_fwd_bwd_mcrossings_per_s": round(pfb_value, 4),
        "fwd_bwd_speedup_vs_plain_fp64_rewalk": round(fb_value / pfb_value, 3),
        "tree_build_ms": {"first": round(build_cold, 2), "warm": round(info.tree_build_ms, 2)},
        "clocks": clocks,
    }

    # --- roofline of the dominant kernel (k_batched + the tiny k_slow)
    bx = BX.get(name)
    mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(mp):
        with open(mp) as f:
            peak, peak_src = float(json.load(f)["hbm_gbs"]), "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    launch_ms = statistics.mean(walk_ms) if walk_ms else None
    if bx and launch_ms:
        achieved = crossings * bx / (launch_ms / 1e3) / 1e9
        dpc = DRAM_BYTES_PER_CROSSING.get((name, auto_kernel))
        rec["roofline"] = {
            "bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "traffic": round(dpc * crossings) if dpc else None,
            "peak_source": peak_src, "bytes_per_crossing": bx,
            "launch_ms": round(launch_ms, 3),
            "kernel": {"thread_fp32": "k_batched (guarded-FP32 k-NN, coherent ray order)",
                       "batched_fp64": "k_batched (bounded FP64 k-NN, coherent ray order)",
                       "batched": "k_warp (one ray per warp)"}.get(auto_kernel, auto_kernel)}

    # --- parity (outside the timed region; one process: rank 0 of N = 1)
    if rank == 0 and world == 1:
        par = {"image_bit_identical_to_plain_fp64": bool(torch.equal(img_auto, img_plain))}
        try:
            sp, idx, o = oracle_sample_parity(w, pc, auto_kernel)
            par.update(sp)
            got = img_auto.cpu().numpy()[idx].reshape(len(idx), -1)
            par["image_rows_bit_identical_to_oracle"] = bool(np.array_equal(got, o))
        except Exception as e:   # keep the timing line
            par["oracle_error"] = str(e)
        rec["parity"] = par
        try:
            rec["counters"] = counters_run(w, L.KERNEL_THREAD_FP32, tune, mode)
        except Exception as e:
            rec["counters"] = {"error": str(e)}

    e2e = None
    if full:
        # --- end to end through the C ABI with host buffers (pinned)
        hS = torch.from_numpy(S).pin_memory().numpy()
        hE = torch.from_numpy(E).pin_memory().numpy()
        hO = torch.empty((n, nout), dtype=torch.float64).pin_memory().numpy()
        st2 = L.Stats()

        def e2e_step():
            L.check(lib.vt_project(h, L.dptr(hS), L.dptr(hE), n, mode, L.KERNEL_AUTO,
                                   L.dptr(hO), C.byref(st2)))

        e2e_step()
        barrier()
        e2e_s = []
        for i in range(K):
            flush.fill_(i & 0xff)
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            e2e_step()
            e2e_s.append(time.perf_counter() - t0)
        barrier()
        t_e2e = reduce(sum(e2e_s), dist.ReduceOp.MAX if world > 1 else None)
        e2e = {"value": round(tot_cross * K / t_e2e / 1e6, 4), "unit": UNIT,
               "h2d_bytes_per_step": int(2 * n * 3 * 8), "d2h_bytes_per_step": int(n * nout * 8)}
    del tape
    return rec, e2e, w


def run_ours(args):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from vortrace_b200 import _lib as L

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    L.load().vt_set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    K, W = args.steps, args.warmup
    rec, e2e, w = measure(args.config, args, rank, world, dev, K, W, npix=args.npix)
    n = rec["rays_per_gpu"]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            v, c, sec, kind, ns = cpu_reference_run(w, 2, args.cpu_sample)
            cpu = {"value": round(v, 4), "unit": UNIT, "cores": host_cores(), "kind": kind,
                   "sample": f"{ns} of {n} rays of {args.config} (evenly spaced), "
                             f"{c} crossings, 2 steps, OpenMP over all host cores"}
        except Exception as e:  # keep the GPU line even if the CPU leg fails
            cpu = {"value": None, "unit": UNIT, "cores": host_cores(), "kind": "unavailable",
                   "sample": f"CPU baseline failed: {e}"}
    del w

    target = None
    if rank == 0 and world == 1 and args.target and args.target != args.config:
        # the >= 3x target configuration (16M-point nested cloud), fewer steps
        try:
            target, _, _ = measure(args.target, args, 0, 1, dev, args.target_steps, 3,
                                   kp=2, wp=1, full=False)
        except Exception as e:
            target = {"workload": args.target, "error": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": rec["value"], "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": rec["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": rec["workload"], "rays_per_gpu": n,
                       "crossings_per_step": rec["crossings_per_step"],
                       "reduction": rec["reduction"],
                       "l2": "flushed before every timed step (256 MB write)",
                       "tree_build_ms": rec["tree_build_ms"],
                       "parallelism": f"rays sharded by view, {world} rank(s)"},
        }
        for k in ("fwd_bwd_mcrossings_per_s", "fwd_bwd_adjoint",
                  "fwd_bwd_rewalk_mcrossings_per_s", "kernel", "autotune",
                  "bounded_fp64_mcrossings_per_s", "plain_fp64_mcrossings_per_s",
                  "speedup_vs_plain_fp64", "plain_fp64_taped_fwd_bwd_mcrossings_per_s",
                  "fwd_bwd_speedup_vs_plain_fp64_taped", "plain_fp64_fwd_bwd_mcrossings_per_s",
                  "fwd_bwd_speedup_vs_plain_fp64_rewalk", "rays_per_s", "parity", "counters"):
            if k in rec:
                line[k] = rec[k]
        line.update({
            "e2e": e2e,
            # per timed forward step: k_ray_keys, the walk kernel, k_slow, and
            # for batches of fewer than 8 x 20 x 148 warps' rays also
            # k_ray_cost, k_batch_keys and k_permute_batches (longest batches
            # first); CUB's radix-sort kernels not counted
            "gpu_launches": (3 + (3 if n < 8 * 20 * 148 * 32 else 0)) * K,
            "roofline": rec.get("roofline"),
            "cpu_baseline": cpu,
            "clocks": rec["clocks"],
        })
        if target is not None:
            line["target_config"] = target
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="clustered_2m")
    ap.add_argument("--cpu-sample", type=int, default=32768)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--npix", type=int, default=None,
                    help="override the grid resolution (smaller profiling case)")
    ap.add_argument("--target", default="nested_16m",
                    help="second workload reported as target_config at N=1 ('' to skip)")
    ap.add_argument("--target-steps", type=int, default=3)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
