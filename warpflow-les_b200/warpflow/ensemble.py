"""Many independent cavity cases advanced together on one GPU.

Each case keeps its fields and multigrid hierarchy resident on the device.
A step of the ensemble is one launch of one CUDA graph holding every case's
step (the projection loops inside it are device-driven, so cases that need
more outer iterations do not hold the others back on the host): small cases
of one size share every kernel launch as a bucket, large cases run as
concurrent branches -- a small case's latency-bound coarse solve overlaps
with a large case's bandwidth-bound sweeps.  All scalar blocks come back
with one device-to-host copy.  Once a case retires, the remaining cases'
own graphs are launched on a pool of streams instead.

The 64-case benchmark ensemble (N in {32, 48, 64, 80, 96}, Re in
[100, 1000], lid velocity in [0.5, 1.5], seeded) is built by
``random_ensemble``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi
from .config import case_from_dict
from .fields import cuda_device
from .solver import STEP_SERIAL, FlowSolver

ENS_BUCKETS = 4   # WF_ENS_BUCKETS
from .topology import build_topology


def cavity_case(n, re=400.0, ulid=1.0, levels=3, precision="mixed", sgs=True,
                variable_dt=True, dt_init=3.0e-4, noise=0.01, name="cavity"):
    """A CaseConfig of the lid-driven cavity benchmark."""
    return case_from_dict({
        "case": name,
        "grid": {"nx": n, "ny": n, "nz": n},
        "physics": {"reynolds": float(re), "sgs": {"enabled": bool(sgs), "cw": 0.46}},
        "initial": {"type": "rest", "noise": float(noise)},
        "boundaries": {"lid_velocity": float(ulid)},
        "numerics": {"mg_levels": int(levels), "mg_precision": precision},
        "time": {"variable_dt": bool(variable_dt), "dt_init": float(dt_init)},
    })


@dataclass
class EnsembleSpec:
    n: int
    re: float
    ulid: float


def random_ensemble(count=64, seed=0, sizes=(32, 48, 64, 80, 96), re=(100.0, 1000.0),
                    ulid=(0.5, 1.5)):
    """Seeded case parameters: N uniform over `sizes`, Re and lid velocity
    uniform in their ranges."""
    rng = np.random.default_rng(seed)
    return [EnsembleSpec(int(rng.choice(sizes)), float(rng.uniform(*re)),
                         float(rng.uniform(*ulid))) for _ in range(count)]


class Ensemble:
    """A set of FlowSolvers stepped concurrently.

    ``step()`` advances every active case by one time step and returns one
    info dict per case (or the exception a case raised, which retires it).

    With ``single_graph`` (default) all cases' steps also form ONE CUDA graph
    (``wf_ensemble_create``), and a step of the whole ensemble is one graph
    launch.  With ``buckets`` cases of the same size and numerics share
    their launches: each bucket is one branch of the graph whose every
    kernel serves all its cases (``WF_ENS_BUCKETS``); without it every case
    is a branch of its own.  ``buckets="auto"`` (default) buckets when all
    cases have the same size and numerics, else gives each case a branch.
    Measured on B200: 13 equal cases per size step 1.1-1.7x faster bucketed
    (32^3 1.07 vs 1.84 ms, 96^3 12.5 vs 12.6 ms), while the 64-case mix of
    sizes 32..96 steps 15 % faster with a branch per case (24.8 vs 28.5 ms
    with every size bucketed): independent branches of different lengths
    overlap one another, a bucket waits for its cases at every launch.  Once
    a case has retired, or for a subset, the cases' own graphs are launched
    on a pool of ``nstreams`` streams instead.
    """

    def __init__(self, cfgs, device="cuda:0", nstreams=32, single_graph=True, buckets="auto"):
        self.device = cuda_device(device)
        # Concurrent cases: kernels that wait for their predecessor while
        # resident would hold SMs other streams could use.
        concurrent = nstreams > 1 or single_graph
        self.solvers = [FlowSolver(cfg, build_topology(cfg), self.device,
                                   serial=concurrent) for cfg in cfgs]
        self.active = [True] * len(self.solvers)
        self._graph = None
        if buckets == "auto":
            kinds = {(sv.n, sv.case.nlev, sv.case.mg_fp32, sv.case.sgs, sv.case.variable_dt)
                     for sv in self.solvers}
            buckets = len(kinds) == 1
        self.buckets = bool(buckets and single_graph)
        if single_graph and len(self.solvers) > 1:
            arr = (_abi.WfCase * len(self.solvers))(*[sv.case for sv in self.solvers])
            self._graph = ctypes.c_void_p()
            mode = STEP_SERIAL | (ENS_BUCKETS if self.buckets else 0)
            _abi.call("wf_ensemble_create", arr, len(self.solvers), mode,
                      ctypes.byref(self._graph))
        ns = max(1, min(nstreams, len(self.solvers)))
        self.streams = [torch.cuda.Stream(self.device) for _ in range(ns)]
        nsc = ctypes.sizeof(_abi.WfScalars)
        self._nsc = nsc
        self._host = torch.empty(max(1, len(self.solvers)) * nsc, dtype=torch.uint8,
                                 pin_memory=True)

    def __len__(self):
        return len(self.solvers)

    def layout(self):
        """(bucket of each case, launch counts per bucket: prologue, calmas
        pass, multigrid part, epilogue) of the one-graph step; without
        buckets every case is its own."""
        if self._graph is None:
            return list(range(len(self))), [s.launch_counts() for s in self.solvers]
        n = len(self.solvers)
        nb = ctypes.c_int32()
        of = (ctypes.c_int32 * n)()
        counts = (ctypes.c_int32 * (4 * n))()
        _abi.call("wf_ensemble_layout", self._graph, ctypes.byref(nb), of, counts)
        bucket = list(of) if self.buckets else list(range(n))
        return bucket, [tuple(counts[4 * b:4 * b + 4]) for b in range(nb.value)]

    def launches_per_step(self):
        """Kernel launches of the last one-graph step: per bucket (or case),
        the prologue and epilogue once, the calmas pass per outer iteration
        and the multigrid part per solve of its busiest case."""
        bucket, counts = self.layout()
        total = 0
        for b, (c0, c1, c2, c3) in enumerate(counts):
            members = [self.solvers[i] for i in range(len(self)) if bucket[i] == b]
            it = max(s.outer_iters for s in members)
            nmg = max(s.last_nmg for s in members)
            total += c0 + c3 + it * c1 + nmg * c2
        return total

    def cells(self, which=None):
        idx = self._which(which)
        return sum(self.solvers[i].n ** 3 for i in idx)

    def _which(self, which):
        if which is None:
            return [i for i, a in enumerate(self.active) if a]
        return list(which)

    def launch(self, which=None):
        """Enqueue one step of the selected cases (default: all active)."""
        idx = self._which(which)
        main = torch.cuda.current_stream(self.device)
        if self._graph is not None and idx == list(range(len(self.solvers))):
            _abi.call("wf_ensemble_step", self._graph, ctypes.c_void_p(main.cuda_stream))
            return idx
        start = torch.cuda.Event()
        start.record(main)
        used = set()
        for slot, i in enumerate(idx):
            s = self.streams[slot % len(self.streams)]
            used.add(s)
            s.wait_event(start)
            with torch.cuda.stream(s):
                self.solvers[i].launch_step()
        for s in used:
            main.wait_stream(s)
        return idx

    def finish(self, idx):
        """Gather the scalar blocks of the launched cases (one copy) and
        apply them; a case that raised is retired and its exception returned
        in its slot."""
        if not idx:
            return []
        blob = torch.cat([self.solvers[i]._sc for i in idx])
        host = self._host[:blob.numel()]
        host.copy_(blob, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        out = []
        base = host.data_ptr()
        for k, i in enumerate(idx):
            view = _abi.WfScalars.from_address(base + k * self._nsc)
            try:
                out.append(self.solvers[i].apply_scalars(view))
            except RuntimeError as e:
                self.active[i] = False
                out.append(e)
        return out

    def step(self, which=None):
        return self.finish(self.launch(which))

    def close(self):
        if self._graph is not None:
            _abi.load().wf_ensemble_destroy(self._graph)
            self._graph = None
        for s in self.solvers:
            s.close()
