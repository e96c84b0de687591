"""Measure the reference search's work per cell crossing on a workload and
derive the algorithmic bytes per crossing used by the roofline:

    B_x = Q * (n_node * 16 + n_pt * 24) + nf * 8 + 48

Q = k-NN queries per crossing, n_node = tree nodes visited per query, n_pt =
point distance evaluations per query (counted in the nanoflann restatement of
vt_oracle.c, which visits exactly the nodes nanoflann visits), 16 B per node
(split value + split dimension / child word), 24 B per FP64 point, nf * 8 B of
field gather and 48 B for the two generator points of the bisector.

    python oracle/measure_bx.py clustered_2m [nrays_sample]
"""
from __future__ import annotations

import json
import os
import sys
import warnings

import numpy as np

sys.path[0] = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
from oracle import oracle as O  # noqa: E402
from vortrace_b200 import workloads as W  # noqa: E402


def measure(name, nsample=8192):
    w = W.CONFIGS[name]()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        lp = O.load_points(w["pos"], w["fields"], w["boundbox"])
    t = O.OracleTree(lp["pts"], lp["fields"], lp["valid_rgba"])
    n = w["starts"].shape[0]
    idx = np.linspace(0, n - 1, min(nsample, n)).astype(np.int64)
    out, (cid, se, sx, off) = t.project(w["starts"][idx], w["ends"][idx], w["reduction"],
                                        segments=True)
    t.project(w["starts"][idx], w["ends"][idx], w["reduction"])
    c = O.OracleTree.last_counters()
    cross = int(off[-1])
    q = c["queries"] / cross
    nn = c["nodes"] / c["queries"]
    npt = c["points"] / c["queries"]
    nf = t.nf
    bx = q * (nn * 16 + npt * 24) + nf * 8 + 48
    return {"workload": name, "rays_sampled": int(len(idx)), "crossings": cross,
            "crossings_per_ray": cross / len(idx), "Q": q, "n_node": nn,
            "n_leaf": c["leaves"] / c["queries"], "n_pt": npt, "nf": nf, "B_x": bx}


if __name__ == "__main__":
    name = sys.argv[1] if len(sys.argv) > 1 else "clustered_2m"
    ns = int(sys.argv[2]) if len(sys.argv) > 2 else 8192
    print(json.dumps(measure(name, ns), indent=1))
