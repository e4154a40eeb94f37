"""Benchmark: lid-driven cavity LES steps on B200 (warpflow B200 build).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 80] [--precision fp64|mixed]

Workload (N=1): the 80^3 cavity of cases/cavity_serial.yaml -- Re 400,
WALE, seeded 1 % noise, variable dt (x1.1 from 3e-4, capped at 0.8 dtmax),
3-level RBGS multigrid 6/6/300, 4 V-cycles, div_tolerance 1e-6.  One step
is one FlowSolver.step().  Under torchrun each rank advances its own
independent replica of the case on its GPU (the case does not shard;
weak scaling), timing is the max over ranks.

Prints one JSON line (rank 0).  ``value`` is Mcell-steps/s from CUDA
events around each step's graph launch with the state resident in HBM;
the L2 (126 MB) is flushed between timed steps by writing a 512 MB buffer
(the 80^3 working set, ~70 MB, would otherwise stay L2-resident).
``e2e`` is the same metric through the public API with the state coming
from and going back to pinned host buffers every step.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "warpflow-les_b200"))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def case_raw(n, levels, precision, seed_noise=0.01):
    return {
        "case": "cavity_serial_%d" % n,
        "domain": {"lx": 1.0, "ly": 1.0, "lz": 1.0},
        "grid": {"nx": n, "ny": n, "nz": n},
        "physics": {"reynolds": 400, "sgs": {"enabled": True, "model": "wale", "cw": 0.46}},
        "initial": {"type": "rest", "noise": seed_noise},
        "boundaries": {"west": "wall", "east": "wall", "south": "slip", "north": "slip",
                       "bottom": "wall", "top": "moving_lid", "lid_velocity": 1.0},
        "numerics": {"mg_levels": levels, "max_outer_iters": 30, "div_tolerance": 1.0e-6,
                     "mg_precision": precision},
        "time": {"n_steps": 1000, "variable_dt": True, "dt_init": 3.0e-4,
                 "safety_factor": 0.8, "dt_growth": 1.1},
        "mpi": {"domains": [1, 1, 1]},
    }


# ---------------------------------------------------------------------------
# algorithmic byte model of one step (reference passes, one read of each
# distinct input and one write of each output per pass over the N^3 cells)
# ---------------------------------------------------------------------------
def vcycle_words(levels, n_pre=6, n_post=6, n_coarse=300):
    """Words per fine cell of one V-cycle: RBGS sweeps (phi, rhs -> phi),
    restriction (+ coarse phi zeroing) and prolongation."""
    L = levels
    w = 0.0
    for l in range(L):
        sweeps = (n_pre + n_post) if l < L - 1 else n_coarse
        w += sweeps * 3.0 / 8 ** l
    for l in range(1, L):
        w += 2.0 / 8 ** (l - 1) + 2.0 / 8 ** l      # restrict l-1 -> l
        w += 1.0 / 8 ** l + 2.0 / 8 ** (l - 1)      # prolong l -> l-1
    return w


def step_bytes(n, iters, nmg, levels, mg_word=8):
    """Bytes per step: fixed 89 words (dt reduce 7, copies 6, WALE 4, two RK
    stages 54, two calvels 18), 4 per divergence pass, and per multigrid
    solve the solve (6 + 4 V-cycles) plus p += pp (3) and calvel (9)."""
    v = vcycle_words(levels)
    fixed = 89 + 4 * iters + 12 * nmg
    mg = nmg * (6 + 4 * v)
    return n ** 3 * (8.0 * fixed + mg_word * mg)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = list(csv.reader(io.StringIO(open(self.path).read())))
        os.unlink(self.path)
        sm, mx, pw, reasons = [], None, [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                pw.append(float(r[3]))
            except ValueError:
                continue
            for nm, val in zip(names, r[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "power_w_max": max(pw) if pw else None, "samples": len(sm),
                "reasons": sorted(reasons)}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return PEAKS_FALLBACK["hbm_gbs"], "fallback"


# DRAM bytes per launch of the dominant kernels, from the ncu captures
# summarised under profiles/ (dram__bytes_read.sum + dram__bytes_write.sum)
NCU_TRAFFIC = {("k_rbgs_split", 256): (189163264, "profiles/rbgs_split_256_full.md"),
               ("k_rbgs_split", 80): (5156864, "profiles/rbgs_split_80_full.md"),
               ("coarse", 20): (172032, "profiles/coarse_p2p_20_full.md")}


def kernel_roofline(sol, args, peak, peak_kind):
    """The dominant kernel of the step (largest share of the step's launch
    list), timed live with CUDA events after the timed region, as replays of
    a CUDA graph of its launches (the form the step runs them in: host
    launch overhead is not counted).  Level 0 of 80^3 and larger (FP64): the split half-sweep
    -- relax(6) and relax(12) differ by exactly 12 half-sweep launches, so
    their difference isolates the kernel; its algorithmic bytes are 1.5 words
    per cell (read the other colour, read the own colour's rhs, write the own
    colour).  Smaller cases: the coarse-level relax.  Where the coarse level
    runs through its operator and is not the dominant kernel, it is reported
    beside it as ``roofline_coarse``."""
    import torch
    if args.precision != "fp64":
        return {"bound": "hbm", "kernel": None, "achieved": None, "peak": peak,
                "unit": "GB/s", "frac": None, "traffic": None,
                "note": "mixed precision relaxes FP32 levels outside the FP64 harness; "
                        "see roofline_step"}, None
    mg = sol.mg
    n = args.n
    if n >= 80:
        main = _split_roofline(mg, n, peak, peak_kind)
        extra = _coarse_roofline(mg, args, peak, peak_kind) if mg._cop_part is not None \
            else None
        return main, extra
    return _coarse_roofline(mg, args, peak, peak_kind), None


def _timed_graph(fn, reps):
    """Seconds per call of `fn` (kernel launches on the current stream),
    timed as replays of a CUDA graph that captured one call -- the form the
    step runs its kernels in, so host launch overhead is not counted; falls
    back to timing direct calls if the capture is refused."""
    import torch
    fn()
    torch.cuda.synchronize()
    try:
        s = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s, capture_error_mode="thread_local"):
                fn()
        g.replay()
        torch.cuda.synchronize()
        run = g.replay
    except Exception:
        run = fn
    a, b = _events()
    a.record()
    for _ in range(reps):
        run()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps / 1e3


def _timed_relax(mg, l, sweeps, reps):
    return _timed_graph(lambda: mg._relax(l, sweeps), reps)   # s per relax


def _roof(name, key, alg, t, peak, peak_kind):
    traffic, src = NCU_TRAFFIC.get(key, (None, None))
    ach = alg / t / 1e9
    return {"bound": "hbm", "kernel": name, "achieved": round(ach, 2), "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": round(ach / peak, 5),
            "traffic": traffic, "traffic_source": src, "alg_bytes_per_launch": round(alg),
            "us_per_launch": round(t * 1e6, 2)}


def _split_roofline(mg, n, peak, peak_kind):
    import numpy as np
    lev0 = mg.levels[0]
    lev0.rhs.assign(np.random.default_rng(7).standard_normal(lev0.shape))
    t = (_timed_relax(mg, 0, 12, 20) - _timed_relax(mg, 0, 6, 20)) / 12
    return _roof("k_rbgs_split (level-0 half-sweep, FP64)", ("k_rbgs_split", n),
                 1.5 * n ** 3 * 8, t, peak, peak_kind)


def _coarse_roofline(mg, args, peak, peak_kind):
    import numpy as np
    import torch
    lc = args.levels - 1
    nc = args.n >> lc
    lv = mg.levels[lc]
    lv.rhs.assign(np.random.default_rng(8).standard_normal(lv.shape))
    if mg._cop_part is None:
        t = _timed_relax(mg, lc, 300, 5)
        return _roof("coarse relax %d^3, 300 sweeps in one launch (latency-bound)" % nc,
                     ("coarse", nc), 3 * (nc + 2) ** 3 * 8, t, peak, peak_kind)
    # the coarse solve through the precomputed symmetric operator, against
    # the bytes of the work it replaces: n_coarse sweeps of the level
    # (read phi and rhs, write phi: 3 words per cell per sweep)
    t = _timed_graph(mg._coarse_solve, 10)
    N = nc ** 3
    out = _roof("coarse %d^3 relax via the symmetric operator (k_cop_vg + k_cop_gemm + "
                "k_cop_out + 2 k_rbgs)" % nc, ("cop", nc), 300 * 3 * N * 8, t, peak, peak_kind)
    out["note"] = ("alg_bytes = the reference's 300 sweeps of the level (3 words per cell "
                   "per sweep); the operator form moves far fewer, so frac is the sweeps' "
                   "equivalent bandwidth, timed through the harness (k_zero + the kernels) as "
                   "CUDA-graph replays")
    return out


# ---------------------------------------------------------------------------
def run_oracle(n, levels, steps, warmup):
    """The reference algorithm on the host cores (NumPy FP64 oracle port;
    the reference's Warp CPU path cannot run here: warp-lang is not
    installed)."""
    from oracle import wf_oracle as O
    from warpflow.config import case_from_dict
    cfg = case_from_dict(case_raw(n, levels, "fp64"))
    sol = O.OracleSolver(cfg)
    for _ in range(warmup):
        sol.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        sol.step()
    dt = time.perf_counter() - t0
    return n ** 3 * steps / dt / 1e6, dt


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def ensemble_compare(ncases, steps, warmup, streams=32, single_graph=True, seed=0):
    """The seeded cavity ensemble (N in {32..96}, Re in [100, 1000], lid in
    [0.5, 1.5]) advanced together with mixed-precision multigrid (one graph
    launch per batch step), and the plain FP64 per-case loop on the same
    cases (every case's own step graph launched one after another on one
    stream), each timed over the same number of batch steps; every batch
    step ends with one gather of all cases' scalar blocks."""
    import torch
    from warpflow.ensemble import Ensemble, cavity_case, random_ensemble
    specs = random_ensemble(ncases, seed=seed)

    def run(precision, concurrent):
        cfgs = [cavity_case(sp.n, sp.re, sp.ulid, precision=precision) for sp in specs]
        if concurrent:
            ens = Ensemble(cfgs, nstreams=streams, single_graph=single_graph)
        else:
            ens = Ensemble(cfgs, nstreams=1, single_graph=False)
        for _ in range(warmup):
            ens.step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            ens.step()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        cells = ens.cells(range(len(ens)))
        iters = sum(s.outer_iters for s in ens.solvers) / len(ens)
        ens.close()
        del ens
        torch.cuda.empty_cache()
        return cells * steps / dt / 1e6, dt, iters

    val, dt, iters = run("mixed", True)
    plain, pdt, piters = run("fp64", False)
    return {"cases": ncases, "steps": steps, "warmup": warmup, "seed": seed,
            "sizes": sorted({sp.n for sp in specs}),
            "mixed_batched_Mcell_steps_per_s": round(val, 2),
            "ms_per_batch_step": round(1e3 * dt / steps, 3), "iters_mean": round(iters, 2),
            "plain_fp64_per_case_loop_Mcell_steps_per_s": round(plain, 2),
            "plain_ms_per_batch_step": round(1e3 * pdt / steps, 3),
            "plain_iters_mean": round(piters, 2),
            "speedup_vs_plain": round(val / plain, 3),
            "timing": "wall clock around the timed batch steps, synced on both sides"}


def bench_ensemble(args):
    """Ensemble mode: ensemble_compare on --cases cases for --steps steps."""
    out = ensemble_compare(args.cases, args.steps, max(3, args.warmup),
                           streams=args.streams or 32, single_graph=bool(args.single_graph))
    out.update({"mode": "ensemble", "metric": "Mcell-steps/s (cavity ensemble, mixed MG)",
                "value": out["mixed_batched_Mcell_steps_per_s"], "unit": "Mcell-steps/s"})
    print(json.dumps(out), flush=True)


def step256_extra(peak, peak_kind, steps=10, warmup=3):
    """The 256^3 cavity with 5 multigrid levels (FP64), device-timed like the
    main line (CUDA events around each step's graph launch, L2 flushed
    between steps)."""
    import torch
    from warpflow import FlowSolver, build_topology
    from warpflow.config import case_from_dict
    n, levels = 256, 5
    cfg = case_from_dict(case_raw(n, levels, "fp64"))
    sol = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
    for _ in range(warmup):
        sol.step()
    torch.cuda.synchronize()
    ms, its, nmgs = [], [], []
    for _ in range(steps):
        flush.zero_()
        a, b = _events()
        a.record()
        sol.launch_step()
        b.record()
        sol.finish_step()
        ms.append(a.elapsed_time(b))
        its.append(sol.outer_iters)
        nmgs.append(sol.last_nmg)
    sol.close()
    del sol, flush
    torch.cuda.empty_cache()
    tot = sum(ms) / 1e3
    byts = sum(step_bytes(n, it, m, levels, 8) for it, m in zip(its, nmgs))
    ach = byts / tot / 1e9
    return {"workload": "lid-driven cavity 256^3, Re 400, WALE, variable dt, 5-level RBGS "
                        "multigrid 6/6/300 x4, FP64", "steps": steps, "warmup": warmup,
            "ms_per_step": round(sum(ms) / steps, 4),
            "value": round(n ** 3 * steps / tot / 1e6, 2), "unit": "Mcell-steps/s",
            "iters_mean": round(sum(its) / steps, 3),
            "roofline_step": {"bound": "hbm", "achieved": round(ach, 1), "peak": peak,
                              "peak_kind": peak_kind, "unit": "GB/s",
                              "frac": round(ach / peak, 4)}}


def bench_serve(args):
    """Serving: seeded Poisson request streams (20 req/s, N in {32..128},
    Re in [100, 1000], steps in [100, 2000] scaled by --step-scale: a
    reduced form of the served-stream configuration) served with continuous
    batching under a 150 GB budget, one stream per seed; then the first
    seed's requests all at once (the saturation throughput)."""
    import numpy as np
    import torch
    from warpflow.serve import CavityServer, poisson_stream
    runs = []
    for seed in range(args.seeds):
        reqs = poisson_stream(count=args.requests, rate=20.0, seed=seed,
                              step_scale=args.step_scale)
        srv = CavityServer(budget_bytes=150 * 10 ** 9, nstreams=args.streams or 16)
        srv.warmup(reqs)
        srv.run(reqs)
        s = srv.summary()
        srv.close()
        span = max(r.arrival for r in reqs) - min(r.arrival for r in reqs)
        offered = sum(r.n ** 3 * r.n_steps for r in reqs) / span / 1e6
        runs.append({"seed": seed, "p50_s": round(s["p50_s"], 4), "p99_s": round(s["p99_s"], 4),
                     "Mcell_steps_per_s": round(s["mcell_steps_per_s"], 2),
                     "offered_Mcell_steps_per_s": round(offered, 2),
                     "wall_s": round(s["wall_s"], 2), "step_batches": s["step_batches"],
                     "solvers_built": s["solvers_built"], "solver_reuses": s["solver_reuses"],
                     "peak_resident_GB": round(s["peak_resident_bytes"] / 1e9, 3)})
        del srv
        torch.cuda.empty_cache()
    reqs = poisson_stream(count=args.requests, rate=20.0, seed=0, step_scale=args.step_scale)
    srv = CavityServer(budget_bytes=150 * 10 ** 9, nstreams=args.streams or 16)
    srv.warmup(reqs)
    srv.run(reqs, time_scale=1e-9)    # every request arrives at once
    sat = srv.summary()
    srv.close()
    p50s = [r["p50_s"] for r in runs]
    print(json.dumps({
        "mode": "serve", "metric": "served cavity stream: p50/p99 latency, Mcell-steps/s",
        "p50_s_median": round(float(np.median(p50s)), 4),
        "p50_s_spread": round(max(p50s) / min(p50s), 3),
        "p99_s_median": round(float(np.median([r["p99_s"] for r in runs])), 4),
        "value": round(float(np.median([r["Mcell_steps_per_s"] for r in runs])), 2),
        "unit": "Mcell-steps/s",
        "saturation_Mcell_steps_per_s": round(sat["mcell_steps_per_s"], 2),
        "runs": runs,
        "config": {"requests": args.requests, "rate_per_s": 20.0, "seeds": args.seeds,
                   "step_scale": args.step_scale, "budget_GB": 150,
                   "streams": args.streams or 16,
                   "reduced": "step counts x %g and %d requests per stream (the full "
                              "configuration: x1, 256)" % (args.step_scale, args.requests),
                   "latency": "arrival to end of last step, wall clock",
                   "startup": "one solver per kind built and stepped before the stream "
                              "starts, kept resident for reuse"}}), flush=True)


def bench_poisson(args):
    """Standalone Poisson solve on 256^3 with 5 levels, RHS
    N(0,1) on the 258^3 level-0 array with the ring zeroed and the mean
    removed (the reference harness tests/test_mg.py), solved to a relative
    max-norm residual of 1e-10 with FP64 V-cycles and with FP32 V-cycles in
    FP64 defect correction."""
    import numpy as np
    import torch
    from oracle.wf_oracle import make_mg_rhs
    from warpflow import Multigrid, build_topology
    from warpflow.config import case_from_dict
    n, L = args.n if args.n != 80 else 256, 5
    rhs = make_mg_rhs(n, seed=0)
    out = {"mode": "poisson", "metric": "standalone Poisson to rel. residual 1e-10",
           "config": {"n": n, "levels": L, "rhs": "default_rng(0).standard_normal, ring 0, "
                                                 "mean removed", "tol": 1e-10}}
    sols = {}
    for prec in ("fp64", "mixed"):
        cfg = case_from_dict({"grid": {"nx": n, "ny": n, "nz": n},
                              "numerics": {"mg_levels": L, "mg_precision": prec}})
        mg = Multigrid(cfg, build_topology(cfg), "cuda:0", 1.0 / n, 1.0 / n, 1.0 / n)
        lev0 = mg.levels[0]
        lev0.rhs.assign(rhs)
        lev0.phi.zero_()
        mg._refill(lev0)
        r0 = mg.residual_max(0)
        cyc, ms = 0, 0.0
        hist = []
        while cyc < 60:
            a, b = _events()
            a.record()
            mg._vcycle()
            b.record()
            r = mg.residual_max(0)
            ms += a.elapsed_time(b)
            cyc += 1
            hist.append(r / r0)
            if r <= 1e-10 * r0:
                break
        s = slice(1, n + 1)
        phi = lev0.phi.t[s, s, s]
        res_l2 = None
        sols[prec] = phi.double().clone()
        # bytes per fine cell per cycle: FP64 V-cycle + residual check, or the
        # FP32 V-cycle + FP64 residual (read phi, rhs, write r32) + FP64 correction
        cell_b = (8 * vcycle_words(L) + 16) if prec == "fp64" else (4 * vcycle_words(L) + 40)
        out[prec] = {"cycles": cyc, "ms": round(ms, 3), "ms_per_cycle": round(ms / cyc, 3),
                     "rel_residual": hist[-1], "residual_history": [float("%.3e" % h) for h in hist],
                     "alg_GBps": round(n ** 3 * cell_b * cyc / (ms / 1e3) / 1e9, 1)}
        del mg
        torch.cuda.empty_cache()
    d = sols["mixed"] - sols["fp64"]
    d = d - d.mean()
    out["mixed_vs_fp64_max_abs"] = float(d.abs().max())
    out["fp64_solution_max_abs"] = float((sols["fp64"] - sols["fp64"].mean()).abs().max())
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=80)
    ap.add_argument("--levels", type=int, default=3)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mode", default="step", choices=["step", "ensemble", "serve", "poisson"])
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--streams", type=int, default=None,
                    help="stream pool (default: 32 for --mode ensemble, 16 for --mode serve)")
    ap.add_argument("--single-graph", type=int, default=1,
                    help="ensemble: all cases in one CUDA graph (1) or a stream pool (0)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the 256^3 step and the ensemble comparison added to the line")
    ap.add_argument("--ens-steps", type=int, default=50)
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--seeds", type=int, default=5)
    ap.add_argument("--step-scale", type=float, default=0.05)
    args = ap.parse_args()
    if args.mode != "step":
        import torch
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        {"ensemble": bench_ensemble, "serve": bench_serve, "poisson": bench_poisson}[
            args.mode](args)
        return
    K, W = args.steps, max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    metric = "Mcell-steps/s (%d^3 cavity step, %s, div<=1e-6)" % (
        args.n, "FP64" if args.precision == "fp64" else "mixed-precision MG")
    cfg_desc = {"workload": "lid-driven cavity %d^3, Re 400, WALE, variable dt, "
                            "%d-level RBGS multigrid 6/6/300 x4 V-cycles" % (args.n, args.levels),
                "n": args.n, "mg_levels": args.levels, "mg_precision": args.precision,
                "replicas": world, "l2": "flushed between timed steps (512 MB write)"}

    if args.impl == "reference":
        if rank != 0:
            return
        ks = min(K, 6)
        val, dt = run_oracle(args.n, args.levels, ks, 1)
        line = {"impl": "reference", "metric": metric, "value": round(val, 4),
                "unit": "Mcell-steps/s", "n_gpus": args.gpus, "steps": ks, "warmup": 1,
                "ms_per_step": round(1e3 * dt / ks, 2), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded hash noise, reference init_noise)",
                "config": cfg_desc,
                "cpu_baseline": {"value": round(val, 4), "unit": "Mcell-steps/s", "cores": 1,
                                 "kind": "port",
                                 "sample": "%d steps of the %d^3 cavity after 1 warm-up step "
                                           "(NumPy FP64 oracle; the reference's Warp CPU path "
                                           "is unavailable: warp-lang not installed)"
                                           % (ks, args.n)},
                "e2e": {"value": round(val, 4), "unit": "Mcell-steps/s",
                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from warpflow import FlowSolver, build_topology
    from warpflow.config import case_from_dict

    cfg = case_from_dict(case_raw(args.n, args.levels, args.precision))
    sol = FlowSolver(cfg, build_topology(cfg), dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # ---- warm-up ----------------------------------------------------------
    for _ in range(W):
        sol.step()
    torch.cuda.synchronize()
    counts = sol.launch_counts()   # filled by graph capture, or by a host-loop step

    # ---- timed region -----------------------------------------------------
    sampler = ClockSampler(local)
    sampler.start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    iters, nmgs = [], []
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(K):
        flush.zero_()
        starts[k].record()
        sol.launch_step()
        ends[k].record()
        sol.finish_step()
        iters.append(sol.outer_iters)
        nmgs.append(sol.last_nmg)
    torch.cuda.synchronize()
    barrier()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    dev_s = sum(step_ms) / 1e3
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([dev_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s = float(t.item())
    value = world * args.n ** 3 * K / dev_s / 1e6
    launches = sum(counts[0] + counts[3] + it * counts[1] + m * counts[2]
                   for it, m in zip(iters, nmgs))

    # ---- roofline (algorithmic bytes of the measured iterations) ------------
    mg_word = 4 if args.precision == "mixed" else 8
    bytes_tot = sum(step_bytes(args.n, it, m, args.levels, mg_word)
                    for it, m in zip(iters, nmgs))
    peak, peak_kind = load_peaks()
    achieved = bytes_tot / (sum(step_ms) / 1e3) / 1e9
    roofline_step = {"bound": "hbm", "kernel": "whole step (one CUDA graph launch)",
                     "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "alg_bytes_per_step": round(bytes_tot / K),
                     "note": "algorithmic bytes of the reference passes (measured iters per "
                             "step) / device step time; frac of the measured copy peak"}
    roofline, roofline_coarse = kernel_roofline(sol, args, peak, peak_kind)

    # ---- end to end through the public API with host buffers ---------------
    e2e = None
    if not args.no_e2e:
        # the step's state: the velocities, the accumulated pressure and the
        # eddy viscosity (the next step's dt reads the previous step's vis)
        state_in = ("u", "v", "w", "p", "vis")
        state_out = state_in
        host = {k: torch.empty(sol.f[k].shape, dtype=torch.float64, pin_memory=True)
                for k in state_in}
        for k in state_in:
            host[k].copy_(sol.f[k].t)
        outs = {k: torch.empty(sol.f[k].shape, dtype=torch.float64, pin_memory=True)
                for k in state_out}
        ke = max(10, K // 3)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            for k in state_in:
                sol.f[k].t.copy_(host[k], non_blocking=True)
            sol.step()
            for k in state_out:
                outs[k].copy_(sol.f[k].t, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            for k in state_in:
                if k in outs:
                    host[k], outs[k] = outs[k], host[k]
        torch.cuda.synchronize()
        barrier()
        te = time.perf_counter() - t0
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([te], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te = float(t.item())
        nb = sol.f["u"].t.numel() * 8
        e2e = {"value": round(world * args.n ** 3 * ke / te / 1e6, 2),
               "unit": "Mcell-steps/s", "steps": ke,
               "h2d_bytes_per_step": nb * len(state_in),
               "d2h_bytes_per_step": nb * len(state_out) + sol._sc.numel(),
               "api": "FlowSolver.step() with u,v,w,p,vis uploaded from and downloaded "
                      "to pinned host memory every step (each step starts from the previous "
                      "step's downloaded state); wall clock"}

    # ---- CPU baseline (oracle port on the host cores) -----------------------
    cpu = None
    if rank == 0 and not args.no_cpu:
        cval, cdt = run_oracle(args.n, args.levels, 2, 0)
        cpu = {"value": round(cval, 4), "unit": "Mcell-steps/s", "cores": 1, "kind": "port",
               "sample": "first 2 steps of the %d^3 cavity (NumPy FP64 oracle, %.1f s); the "
                         "reference's Warp CPU path is unavailable here" % (args.n, cdt)}

    extras = {}
    if world == 1 and not args.no_extras and args.n == 80:
        extras["extra_step256_L5_fp64"] = step256_extra(peak, peak_kind)
        extras["extra_ensemble64_mixed_vs_plain"] = ensemble_compare(64, args.ens_steps, 3)

    if rank == 0:
        line = {"metric": metric, "value": round(value, 2), "unit": "Mcell-steps/s",
                "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": round(sum(step_ms) / K, 4), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded hash noise, reference init_noise)",
                "config": cfg_desc, "iters_mean": round(sum(iters) / K, 3),
                "wall_s": round(wall, 3), "gpu_launches": int(launches),
                "launches_per_step": round(launches / K, 1),
                "clocks": clocks, "roofline": roofline, "roofline_step": roofline_step,
                "roofline_coarse": roofline_coarse,
                "cpu_baseline": cpu, "e2e": e2e}
        line.update(extras)
        print(json.dumps(line), flush=True)
    sol.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
