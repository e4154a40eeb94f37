"""Autotuner for the many-sweep relax of small multigrid levels.

For each level size it times the implementations of libwfb200 (0: one CTA
with the level in shared memory; 1: a thread-block cluster with a cluster
barrier per half-sweep; 2: a cluster with point-to-point halo pushes; 3: the
same with two halo planes and one exchange per sweep; 4: point-to-point
with thinner slabs, clusters of up to 16 CTAs) on a 300-sweep relax
and installs the fastest through
``wf_set_coarse_strategy``.

``tune_buckets`` makes the ensemble's choice per case size: it times an
ensemble step of ``ncases`` equal-sized cases bucketed (every kernel launch
serves all of them) against one graph branch per case, and installs the
faster through ``wf_set_bucket_cap``.

``tune_shapes`` chooses launch shapes per grid size: the CTA of the
convection pass (``k_conv``: threads along k and j) and the cells per
thread and rows per CTA of the split red-black half-sweep
(``k_rbgs_split``).  Each candidate is timed on the kernel alone, its
output must equal the default shape's bit for bit (only the mapping of
cells to threads changes), and the fastest is installed through
``wf_set_launch_shape``.  Shapes are read when a launch is issued, so tune
before building the solvers that should use them.

Results can be cached as JSON (``save``; one file holds all three tables)
and re-applied (``load_and_apply``).  The library's built-in tables are the
same measurements taken on a B200.
"""
from __future__ import annotations

import ctypes
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


def set_bucket_cap(n, cap, fp32=True):
    """Largest bucket for ensemble cases of size n (1: a branch per case,
    0: the library's default)."""
    _abi.call("wf_set_bucket_cap", int(n), 1 if fp32 else 0, int(cap))


def bucket_cap(n, fp32=True):
    out = ctypes.c_int32()
    _abi.call("wf_bucket_cap", int(n), 1 if fp32 else 0, ctypes.byref(out))
    return out.value


def _time_ensemble(ens, reps):
    for _ in range(2):
        ens.launch()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        ens.launch()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def tune_buckets(sizes=(32, 48, 64, 80, 96), ncases=8, precision="mixed", reps=5,
                 device="cuda:0"):
    """For each size, time one ensemble step of `ncases` cases of that size
    in one bucket and as separate branches; install the faster and return
    {n: {"cap": c, "ms": {"bucket": t, "branches": t}}}.  The cases start
    from rest with the benchmark's noise and advance while being timed;
    both forms start from the same state."""
    from .ensemble import Ensemble, cavity_case
    fp32 = precision == "mixed"
    out = {}
    for n in sizes:
        cfgs = [cavity_case(n, 100.0 + 900.0 * i / max(1, ncases - 1), 1.0,
                            precision=precision) for i in range(ncases)]
        cap = max(2, int(ncases))
        times = {}
        for label, c in (("bucket", cap), ("branches", 1)):
            set_bucket_cap(n, c, fp32)
            ens = Ensemble(cfgs, device=device, nstreams=1)
            times[label] = _time_ensemble(ens, reps)
            ens.close()
        best = cap if times["bucket"] < times["branches"] else 1
        set_bucket_cap(n, best, fp32)
        out[n] = {"cap": best, "ms": {k: round(v, 3) for k, v in times.items()}}
    return out


SHAPE_CONV, SHAPE_SPLIT = 0, 1
# k_conv: threads along k, along j, planes i per thread
CONV_SHAPES = tuple((a, b, c) for a, b in ((32, 8), (16, 16), (64, 4), (32, 4), (16, 8),
                                           (128, 2), (32, 2), (8, 32))
                    for c in (1, 2, 4, 8))
# k_rbgs_split: cells per thread, rows per CTA
SPLIT_SHAPES = tuple((c, r, 1) for c in (1, 2, 4, 8) for r in (1, 2, 4, 8))
_KIND = {"conv": SHAPE_CONV, "split": SHAPE_SPLIT}


def set_shape(kind, n, a, b, c=1):
    """Launch shape of `kind` ("conv" or "split") for size n; (0, 0, 0)
    restores the default."""
    _abi.call("wf_set_launch_shape", _KIND[kind], int(n), int(a), int(b), int(c))


def shape(kind, n):
    a, b, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    _abi.call("wf_launch_shape", _KIND[kind], int(n), ctypes.byref(a), ctypes.byref(b),
              ctypes.byref(c))
    return a.value, b.value, c.value


def _time_fn(fn, reps):
    fn()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps * 1e3  # us


def tune_shapes(sizes=(80,), conv=CONV_SHAPES, split=SPLIT_SHAPES, reps=10, device="cuda:0"):
    """Time every candidate shape of the convection pass (the three
    components, one launch each) and, for sizes whose finest level relaxes
    on the split copy (FP64, n >= 80, even), of the split half-sweep (12
    half-sweeps: a 12-sweep relax less a 6-sweep one).  Install the fastest
    per size and return {"conv": {n: rec}, "split": {n: rec}}, rec =
    {"best": [a, b, c], "us": {"axbxc": time}}.  Raises if a shape changes
    a result."""
    from .ensemble import cavity_case
    from .solver import FlowSolver
    out = {"conv": {}, "split": {}}
    for n in sizes:
        cfg = cavity_case(n, precision="fp64")
        sol = FlowSolver(cfg, build_topology(cfg), device)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        dtp = ctypes.c_void_p(sol._sc.data_ptr())   # wf_scalars.dt is the first member

        def conv_pass():
            for comp in range(3):
                _abi.call("wf_conv", ctypes.byref(sol.case), comp, 0.5, dtp, stream)

        times, ref = {}, None
        for a, b, c in conv:
            set_shape("conv", n, a, b, c)
            t = _time_fn(conv_pass, reps)
            got = [sol.f[k].numpy() for k in ("ustar", "vstar", "wstar")]
            if ref is None:
                ref = got
            elif any(not np.array_equal(x, y) for x, y in zip(got, ref)):
                set_shape("conv", n, 0, 0, 0)
                raise RuntimeError("k_conv shape %dx%dx%d changed the result at n=%d"
                                   % (a, b, c, n))
            times["%dx%dx%d" % (a, b, c)] = t
        best = min(times, key=times.get)
        a, b, c = (int(x) for x in best.split("x"))
        set_shape("conv", n, a, b, c)
        out["conv"][n] = {"best": [a, b, c], "us": {k: round(v, 2) for k, v in times.items()}}

        mg = sol.mg
        lev = mg.levels[0]
        if n >= 80 and n % 2 == 0 and split:
            rhs = np.random.default_rng(n).standard_normal(lev.shape)
            lev.rhs.assign(rhs)
            times, ref = {}, None
            for c, r, _ in split:
                set_shape("split", n, c, r)
                lev.phi.zero_()
                mg._relax(0, 6)
                got = lev.phi.numpy()
                if ref is None:
                    ref = got
                elif not np.array_equal(got, ref):
                    set_shape("split", n, 0, 0, 0)
                    raise RuntimeError("k_rbgs_split shape %dx%d changed the result at n=%d"
                                       % (c, r, n))
                t12 = _time_fn(lambda: mg._relax(0, 12), reps)
                t6 = _time_fn(lambda: mg._relax(0, 6), reps)
                times["%dx%dx1" % (c, r)] = (t12 - t6) / 12
            best = min(times, key=times.get)
            c, r, _ = (int(x) for x in best.split("x"))
            set_shape("split", n, c, r)
            out["split"][n] = {"best": [c, r, 1],
                               "us": {k: round(v, 3) for k, v in times.items()}}
        sol.close()
    return out


def save(table, path, buckets=None, shapes=None):
    """Write the relax-strategy table (and the bucket and shape tables) as
    JSON."""
    doc = {"coarse": {str(k): v for k, v in table.items()}}
    if buckets is not None:
        doc["buckets"] = {str(k): v for k, v in buckets.items()}
    if shapes is not None:
        doc["shapes"] = {kind: {str(n): rec for n, rec in recs.items()}
                         for kind, recs in shapes.items()}
    with open(path, "w") as fh:
        json.dump(doc, fh, indent=1)


def load_and_apply(path, fp32_buckets=True):
    """Install a cached JSON table; returns the document."""
    with open(path) as fh:
        doc = json.load(fh)
    sections = ("coarse", "buckets", "shapes")
    coarse = doc.get("coarse", {} if any(k in doc for k in sections) else doc)
    for n, rec in coarse.items():
        set_strategy(int(n), rec["best"])
        set_strategy(int(n), rec["best"], fp32=True)
    for n, rec in doc.get("buckets", {}).items():
        set_bucket_cap(int(n), rec["cap"], fp32_buckets)
    for kind, recs in doc.get("shapes", {}).items():
        for n, rec in recs.items():
            set_shape(kind, int(n), *rec["best"])
    return doc
