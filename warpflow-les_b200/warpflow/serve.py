"""Continuous-batching server for cavity solves.

Requests (N, Re, lid velocity, step count) arrive over time.  The server
admits a queued request as soon as its device memory -- fields plus
multigrid hierarchy, computed exactly by ``case_bytes``, and the shared
coarse-level operator of its kind -- fits in the HBM budget next to the
cases already resident, keeps every admitted case resident until its last
step, and advances all resident cases together one step at a time
(``Ensemble``-style concurrent graph launches).  A finished case's solver
stays resident and serves the next request of the same size: it is reset
on the device (``FlowSolver.reset``: fields re-initialised, 1/Re and the
lid velocity written to its scalar block), so steady-state admission
allocates nothing and captures no graph; only requests of a kind with no
idle solver build one, on a worker thread.  Requests
that arrive while others run join at the next step boundary; finished
cases leave at a step boundary and free their memory for the queue.
Latency is measured from arrival to the end of the request's last step.

``Admission`` holds the queueing policy and the memory ledger with no GPU
dependency, so it is tested on the CPU.
"""
from __future__ import annotations

import collections
import concurrent.futures
import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _abi
from .ensemble import cavity_case
from .fields import cuda_device
from .multigrid import COARSE_OP_MAX_BYTES
from .solver import FlowSolver
from .topology import build_topology

NFIELDS = 13


def coarse_op_elems(n, levels=3, precision="mixed"):
    """(shared operator elements, per-case scratch elements) of the
    coarse-level operator of an n^3 unit-cube case, from the library's own
    sizing (wf_mg_coarse_op_elems, host-only), or (0, 0) when the coarsest
    level runs as sweeps."""
    if levels < 2:
        return 0, 0
    c = _abi.WfCase()
    c.n, c.nlev, c.n_coarse = n, levels, 300
    c.dx = c.dy = c.dz = 1.0 / n
    c.mg_fp32 = 1 if precision == "mixed" else 0
    op, sc = ctypes.c_int64(), ctypes.c_int64()
    if _abi.load().wf_mg_coarse_op_elems(ctypes.byref(c), ctypes.byref(op),
                                         ctypes.byref(sc)) != 0:
        return 0, 0
    word = 4 if precision == "mixed" else 8
    if op.value * word > COARSE_OP_MAX_BYTES:
        return 0, 0
    return op.value, sc.value


def operator_bytes(n, levels=3, precision="mixed"):
    """Device bytes of the coarse-level operator shared by every case of
    the same size, depth and precision (kept for the life of the process)."""
    return coarse_op_elems(n, levels, precision)[0] * (4 if precision == "mixed" else 8)


def case_bytes(n, levels=3, precision="mixed"):
    """Device bytes a FlowSolver of an n^3 case allocates for itself: 13
    padded FP64 fields, FP64 multigrid levels (phi, rhs with one ring, level
    0 included), the FP32 copies of every level in mixed precision, a
    scratch of two level arrays per level in the multigrid's precision, the
    coarse-level operator's per-case scratch (the operator itself is shared:
    operator_bytes), and two scalar blocks plus one residual slot."""
    fields = NFIELDS * (n + 6) ** 3 * 8
    mg = 0
    for l in range(levels):
        m = (n >> l) + 2
        mg += 2 * m ** 3 * 8
        if precision == "mixed":
            mg += 2 * m ** 3 * 4 + 2 * m ** 3 * 4
        else:
            mg += 2 * m ** 3 * 8
    word = 4 if precision == "mixed" else 8
    mg += coarse_op_elems(n, levels, precision)[1] * word
    return fields + mg + 2 * ctypes.sizeof(_abi.WfScalars) + 8


OPERATOR_EDGES = (4, 8, 12, 16, 20, 24)   # coarsest edges with a coarse-level operator


def levels_for(n, coarse_max=32):
    """Multigrid depth for a request: 3 levels (the reference cases') unless
    the coarse grid would exceed `coarse_max` cells per axis; then one level
    more where that turns a coarsest edge without a coarse-level operator
    into one with it (128^3: 32^3 coarse sweeps -> a 16^3 operator, 1.75x
    faster per step; 112^3 stays at 3 levels, its 14^3 coarse level would
    be slower than 28^3)."""
    levels = 3
    while (n >> (levels - 1)) > coarse_max and n % (1 << levels) == 0:
        levels += 1
    if (n >> (levels - 1)) not in OPERATOR_EDGES and n % (1 << levels) == 0 \
            and (n >> levels) in OPERATOR_EDGES:
        levels += 1
    return levels


@dataclass
class Request:
    rid: int
    n: int
    re: float
    ulid: float
    n_steps: int
    arrival: float            # seconds after the stream starts
    levels: int = 3
    precision: str = "mixed"

    @property
    def bytes(self):
        return case_bytes(self.n, self.levels, self.precision)


@dataclass
class Completion:
    rid: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    cells: int
    info: dict = field(default_factory=dict)
    error: str = ""

    @property
    def latency(self):
        return self.finished - self.arrival


class Admission:
    """FIFO admission against a memory budget (no GPU needed).

    The ledger holds every running case's own bytes, the idle solvers kept
    resident for reuse (a finished case's solver serves the next request of
    its size: ``idle`` counts them per (N, levels, precision)), and, once
    per kind, the shared coarse-level operator, which stays allocated for
    the life of the process once a case of that kind has been built.  A
    request of a kind with an idle solver takes it and needs no new bytes;
    otherwise idle solvers of other kinds are evicted (largest first) until
    the request fits; the caller drains ``evicted`` and frees those
    solvers, and ``reused`` tells which admitted requests take an idle one."""

    def __init__(self, budget_bytes, max_active=None):
        self.budget = int(budget_bytes)
        self.max_active = max_active
        self.queue = collections.deque()
        self.resident = {}     # rid -> bytes
        self.shared = {}       # (n, levels, precision) -> operator bytes
        self.idle = collections.Counter()   # (n, levels, precision) -> idle solvers
        self.evicted = []      # kinds whose idle solver the caller must free
        self.reused = set()    # rids admitted onto an idle solver
        self.peak = 0

    @staticmethod
    def kind(req):
        return (req.n, req.levels, req.precision)

    @property
    def used(self):
        return (sum(self.resident.values()) + sum(self.shared.values()) +
                sum(cnt * case_bytes(*k) for k, cnt in self.idle.items()))

    def keep_idle(self, kind):
        """Charge one more idle solver of `kind` (built before the stream,
        for instance); False if it does not fit the budget."""
        extra = 0 if kind in self.shared else operator_bytes(*kind)
        if self.used + case_bytes(*kind) + extra > self.budget:
            return False
        self.idle[kind] += 1
        if extra:
            self.shared[kind] = extra
        self.peak = max(self.peak, self.used)
        return True

    def _extra(self, req):
        key = (req.n, req.levels, req.precision)
        return 0 if key in self.shared else operator_bytes(*key)

    def submit(self, req):
        if req.bytes + self._extra(req) + sum(self.shared.values()) > self.budget:
            raise ValueError("request %d needs %d bytes, more than the whole budget %d"
                             % (req.rid, req.bytes, self.budget))
        self.queue.append(req)

    def admit(self, now):
        """Pop the requests that have arrived by `now` and fit, in arrival
        order; stop at the first one that does not fit (no overtaking)."""
        out = []
        while self.queue and self.queue[0].arrival <= now:
            req = self.queue[0]
            if self.max_active is not None and len(self.resident) >= self.max_active:
                break
            kind = self.kind(req)
            if self.idle[kind] > 0:
                self.idle[kind] -= 1
                self.reused.add(req.rid)
            else:
                extra = self._extra(req)
                while self.used + req.bytes + extra > self.budget:
                    others = [k for k, cnt in self.idle.items() if cnt > 0]
                    if not others:
                        break
                    big = max(others, key=lambda k: case_bytes(*k))
                    self.idle[big] -= 1
                    self.evicted.append(big)
                if self.used + req.bytes + extra > self.budget:
                    break
                if extra:
                    self.shared[kind] = extra
            self.queue.popleft()
            self.resident[req.rid] = req.bytes
            self.peak = max(self.peak, self.used)
            out.append(req)
        return out

    def release(self, rid, keep=None):
        """A case left; with `keep` (its kind) its solver stays resident idle."""
        if self.resident.pop(rid, None) is not None and keep is not None:
            self.idle[keep] += 1


def poisson_stream(count=256, rate=20.0, seed=0, sizes=tuple(range(32, 129, 16)),
                   re=(100.0, 1000.0), ulid=(1.0, 1.0), steps=(100, 2000),
                   precision="mixed", step_scale=1.0):
    """Seeded request stream: exponential inter-arrival times at `rate`
    requests/s, N uniform over `sizes`, Re uniform, step counts uniform over
    the integer range (scaled by `step_scale`, at least 1)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(count):
        t += float(rng.exponential(1.0 / rate))
        n = int(rng.choice(sizes))
        ns = int(rng.integers(steps[0], steps[1] + 1))
        out.append(Request(rid=rid, n=n, re=float(rng.uniform(*re)),
                           ulid=float(rng.uniform(*ulid)),
                           n_steps=max(1, int(round(ns * step_scale))), arrival=t,
                           levels=levels_for(n), precision=precision))
    return out


class CavityServer:
    """Runs a request stream to completion with continuous batching."""

    def __init__(self, device="cuda:0", budget_bytes=150 * 10 ** 9, nstreams=16,
                 max_active=None, keep_fields=False):
        self.device = cuda_device(device)
        self.adm = Admission(budget_bytes, max_active)
        self.streams = [torch.cuda.Stream(self.device) for _ in range(nstreams)]
        self.keep_fields = keep_fields
        self.results = {}
        self.fields = {}
        self.pool = {}         # (n, levels, precision) -> idle resident solvers
        self.built = 0         # solvers constructed (start-up included)
        self.cell_steps = 0
        self.step_batches = 0
        self._nsc = ctypes.sizeof(_abi.WfScalars)
        self._host = torch.empty(4096 * self._nsc, dtype=torch.uint8, pin_memory=True)

    @staticmethod
    def _cfg(req):
        return cavity_case(req.n, req.re, req.ulid, levels=req.levels,
                           precision=req.precision, name="req%d" % req.rid)

    def _build(self, req):
        cfg = self._cfg(req)
        self.built += 1
        return FlowSolver(cfg, build_topology(cfg), self.device,
                          serial=len(self.streams) > 1)

    def warmup(self, requests):
        """Server start-up, before the stream's clock runs: build and step
        once a solver of every (N, levels, precision) that `requests` use, so
        that the CUDA context, the library's kernels and the shared
        coarse-level operators are loaded when the first request arrives;
        each such solver stays resident as an idle one for the first request
        of its kind, as far as the budget allows."""
        seen = set()
        for r in requests:
            key = (r.n, r.levels, r.precision)
            if key in seen:
                continue
            seen.add(key)
            sol = self._build(Request(rid=-1, n=r.n, re=r.re, ulid=r.ulid, n_steps=1,
                                      arrival=0.0, levels=r.levels, precision=r.precision))
            sol.step()
            if self.adm.keep_idle(key):
                self.pool.setdefault(key, []).append(sol)
            else:
                sol.close()
        torch.cuda.synchronize(self.device)

    def _take(self, req):
        """An idle solver of the request's kind, reset on the device for it."""
        sol = self.pool[Admission.kind(req)].pop()
        sol.reset(self._cfg(req))
        return sol

    def _evict(self):
        for key in self.adm.evicted:
            self.pool[key].pop().close()
        self.adm.evicted.clear()

    def run(self, requests, time_scale=1.0):
        """Serve `requests` (arrival times in seconds, compressed by
        `time_scale`); returns the completions in request order."""
        for r in sorted(requests, key=lambda r: r.arrival):
            self.adm.submit(r)
        live = {}          # rid -> (req, solver, admitted_at, steps_done)
        building = {}      # rid -> (req, future of its solver, admitted_at)
        t0 = time.perf_counter()
        main = torch.cuda.current_stream(self.device)
        total = len(requests)
        # Solvers are built on a worker thread: their host-side set-up
        # (allocations, graph capture and instantiation) would otherwise
        # hold up the next step of every case already resident.
        pool = concurrent.futures.ThreadPoolExecutor(max_workers=1)
        try:
            while len(self.results) < total:
                now = (time.perf_counter() - t0) / time_scale
                admitted = self.adm.admit(now)
                self._evict()
                for req in admitted:
                    if req.rid in self.adm.reused:
                        live[req.rid] = [req, self._take(req), now, 0]
                    else:
                        building[req.rid] = (req, pool.submit(self._build_on_worker, req), now)
                for rid in [r for r, (_, fut, _) in building.items() if fut.done()]:
                    req, fut, adm_t = building.pop(rid)
                    live[rid] = [req, fut.result(), adm_t, 0]
                if not live:
                    if building:
                        concurrent.futures.wait([fut for _, fut, _ in building.values()],
                                                return_when=concurrent.futures.FIRST_COMPLETED)
                    else:
                        nxt = self.adm.queue[0].arrival if self.adm.queue else now
                        time.sleep(max(0.0, (nxt - now) * time_scale))
                    continue
                self._step_batch(live, main, t0, time_scale)
        finally:
            pool.shutdown(wait=True)
        self.wall = time.perf_counter() - t0
        return [self.results[r.rid] for r in requests]

    def _build_on_worker(self, req):
        torch.cuda.set_device(self.device)   # the worker thread's current device
        sol = self._build(req)
        # the set-up kernels ran on this thread's current stream; finish them
        # here so that a step on any stream sees initialised fields
        torch.cuda.current_stream(self.device).synchronize()
        return sol

    def _step_batch(self, live, main, t0, time_scale):
        """One step of every live case, then their scalar blocks in one copy;
        finished cases leave."""
        rids = list(live)
        start = torch.cuda.Event()
        start.record(main)
        used = set()
        for slot, rid in enumerate(rids):
            s = self.streams[slot % len(self.streams)]
            used.add(s)
            s.wait_event(start)
            with torch.cuda.stream(s):
                live[rid][1].launch_step()
        for s in used:
            main.wait_stream(s)
        blob = torch.cat([live[rid][1]._sc for rid in rids])
        if blob.numel() > self._host.numel():
            self._host = torch.empty(blob.numel(), dtype=torch.uint8, pin_memory=True)
        host = self._host[:blob.numel()]
        host.copy_(blob, non_blocking=True)
        main.synchronize()
        self.step_batches += 1
        done_t = (time.perf_counter() - t0) / time_scale
        for k, rid in enumerate(rids):
            req, sol, adm_t, nst = live[rid]
            view = _abi.WfScalars.from_address(host.data_ptr() + k * self._nsc)
            err = ""
            try:
                info = sol.apply_scalars(view)
            except RuntimeError as e:
                info, err = {}, str(e)
            nst += 1
            live[rid][3] = nst
            self.cell_steps += req.n ** 3
            if nst >= req.n_steps or err:
                self.results[rid] = Completion(rid, req.arrival, adm_t, done_t, nst,
                                               req.n ** 3, info, err)
                if self.keep_fields:
                    self.fields[rid] = {k2: sol.f[k2].numpy() for k2 in ("u", "v", "w", "p")}
                del live[rid]
                if err:      # a failed case's solver is not reused
                    sol.close()
                    self.adm.release(rid)
                else:        # the solver stays resident for the next request of its kind
                    kind = Admission.kind(req)
                    self.pool.setdefault(kind, []).append(sol)
                    self.adm.release(rid, keep=kind)

    def summary(self):
        lat = np.array([c.latency for c in self.results.values()])
        return {"requests": len(lat),
                "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "mcell_steps_per_s": self.cell_steps / self.wall / 1e6 if self.wall else None,
                "wall_s": self.wall, "step_batches": self.step_batches,
                "peak_resident_bytes": self.adm.peak, "solvers_built": self.built,
                "solver_reuses": len(self.adm.reused)}

    def close(self):
        """Free the idle solvers kept for reuse."""
        for sols in self.pool.values():
            for sol in sols:
                sol.close()
        self.pool.clear()
        self.adm.idle.clear()
