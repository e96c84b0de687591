"""Build libvortrace_b200.so in-tree with nvcc (sm_100a only).

    python -m vortrace_b200.build [--force] [--verbose-ptxas]

Every .cu file under csrc/ is compiled for ``-gencode
arch=compute_100a,code=sm_100a`` with ``--fmad=false`` (FP64 expressions must
round like the reference's x86-64 build) and linked into
``vortrace_b200/libvortrace_b200.so`` next to this file.  A second build with
the search counters of the batched kernel compiled in
(``-DVT_BATCHED_COUNTERS=1``: nodes visited, FP64 re-checks, queries with a
re-check) goes to ``libvortrace_b200_counters.so``; the benchmark reads its
counters in a launch outside the timed region.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvortrace_b200.so")
LIB_COUNTERS = os.path.join(HERE, "libvortrace_b200_counters.so")
COUNTER_DEFINES = ("VT_BATCHED_COUNTERS=1",)
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-O3", "--expt-relaxed-constexpr", "-I" + INCLUDE]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: cannot build libvortrace_b200")


def host_compiler() -> list[str]:
    # the system g++ (the environment's CXX may point at a toolchain without
    # the libraries nvcc expects)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return ["-ccbin", cand]
    return []


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return _sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + sorted(
        glob.glob(os.path.join(CSRC, "*.h"))) + [os.path.join(INCLUDE, "vortrace_b200.h"),
                                                 os.path.abspath(__file__)]


def up_to_date(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(force: bool = False, ptxas_verbose: bool = False, jobs: int = 0,
          out: str | None = None, defines: tuple = ()) -> str:
    """Compile and link; ``out``/``defines`` build a variant elsewhere (for
    tuning sweeps, e.g. defines=("VT_BATCHED_MINB=6",))."""
    lib = out or LIB
    if not force and (out is None or out == LIB_COUNTERS) and up_to_date(lib):
        return lib
    bdir = BUILD if out is None else (BUILD + "_counters" if out == LIB_COUNTERS
                                      else lib + ".objs")
    os.makedirs(bdir, exist_ok=True)
    cc = nvcc()
    objs, procs = [], []
    for src in _sources():
        obj = os.path.join(bdir, os.path.basename(src)[:-3] + ".o")
        cmd = [cc, *ARCH, *FLAGS, *host_compiler(), *[f"-D{d}" for d in defines], "-c", src,
               "-o", obj]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                                            text=True)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"--- nvcc failed on {src}\n{out}\n")
        elif out.strip():
            sys.stderr.write(out)
    if failed:
        raise RuntimeError("libvortrace_b200 build failed")
    tmp = lib + ".tmp"
    subprocess.run([cc, *ARCH, *host_compiler(), "-shared", *objs, "-o", tmp], check=True)
    os.replace(tmp, lib)
    return lib


def build_counters(force: bool = False) -> str:
    """The library with the batched kernel's search counters compiled in."""
    return build(force=force, out=LIB_COUNTERS, defines=COUNTER_DEFINES)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--no-counters", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.verbose_ptxas))
    if not a.no_counters:
        print(build_counters(force=a.force))


if __name__ == "__main__":
    main()
