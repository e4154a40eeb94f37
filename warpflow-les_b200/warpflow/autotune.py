"""Autotuner for the many-sweep relax of small multigrid levels.

For each level size it times the implementations of libwfb200 (0: one CTA
with the level in shared memory; 1: a thread-block cluster with a cluster
barrier per half-sweep; 2: a cluster with point-to-point halo pushes; 3: the
same with two halo planes and one exchange per sweep; 4: point-to-point
with thinner slabs, clusters of up to 16 CTAs) on a 300-sweep relax
and installs the fastest through
``wf_set_coarse_strategy``.  Results can be cached as JSON and re-applied.
The library's built-in table is the same measurement taken on a B200.
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

from . import _abi
from .config import case_from_dict
from .multigrid import Multigrid
from .topology import build_topology

SIZES = (6, 8, 10, 12, 14, 16, 20, 24, 28, 32)
CLUSTER_SIZES = set(SIZES)   # sizes with cluster kernels
TB_SIZES = {8, 10, 12, 14, 16, 20, 24, 28, 32}
THIN_SIZES = {12, 16, 20, 24, 28, 32}
SMEM_SIZES = {4, 8, 12, 16, 20, 24}


def _time_relax(mg, sweeps, reps=3):
    mg._relax(0, sweeps)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        mg._relax(0, sweeps)
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps * 1e3  # us


def set_strategy(n, strategy, fp32=False):
    _abi.call("wf_set_coarse_strategy", int(n), 1 if fp32 else 0, int(strategy))


def tune(sizes=SIZES, sweeps=300, device="cuda:0"):
    """Time every applicable strategy for each size; install and return
    {n: {"best": s, "us": {s: time}}}."""
    if os.environ.get("WF_COARSE"):
        raise RuntimeError("unset WF_COARSE to autotune (it forces one strategy)")
    out = {}
    for n in sizes:
        cfg = case_from_dict({"grid": {"nx": n, "ny": n, "nz": n},
                              "numerics": {"mg_levels": 1}})
        mg = Multigrid(cfg, build_topology(cfg), device, 1.0 / n, 1.0 / n, 1.0 / n)
        lev = mg.levels[0]
        lev.rhs.assign(np.random.default_rng(n).standard_normal(lev.shape))
        cands = [s for s in (0, 1, 2, 3, 4)
                 if (s == 0 and n in SMEM_SIZES) or (s in (1, 2) and n in CLUSTER_SIZES)
                 or (s == 3 and n in TB_SIZES) or (s == 4 and n in THIN_SIZES)]
        times = {}
        for s in cands:
            set_strategy(n, s)
            lev.phi.zero_()
            times[s] = _time_relax(mg, sweeps)
        best = min(times, key=times.get)
        set_strategy(n, best)
        set_strategy(n, best, fp32=True)
        out[n] = {"best": best, "us": {str(k): round(v, 1) for k, v in times.items()}}
    return out


def save(table, path):
    with open(path, "w") as fh:
        json.dump({str(k): v for k, v in table.items()}, fh, indent=1)


def load_and_apply(path):
    with open(path) as fh:
        table = json.load(fh)
    for n, rec in table.items():
        set_strategy(int(n), rec["best"])
        set_strategy(int(n), rec["best"], fp32=True)
    return table
