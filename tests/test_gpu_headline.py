"""Whole-step parity at the benchmark configurations, on the production path.

The 80^3 cavity of the benchmark (variable dt from 3e-4, Re 400, WALE,
3-level multigrid 6/6/300 x 4) runs as the bench runs it: one CUDA graph
launch per step, level 0 relaxed on its row-parity-split copy, the 20^3
coarse level through its precomputed operator, each diffusion inside its
convection pass.  The 32^3 fixed-dt cavity runs its full 200 steps.  Both
are compared with the FP64 CPU oracle:

* FP64: every field, ghosts included, within 1e-10 max abs after the first
  step; identical outer-iteration counts every step, the divergence trace
  of every outer iteration within 1e-5 relative, dt within 1e-12 relative;
  u, v, w within 1e-8 rms at the end (the solver's 100-step tolerance,
  here after 6 and 200 steps).
* Mixed-precision multigrid: every step's divergence below div_tolerance
  (1e-6) and u, v, w within 1e-7 rms of the FP64 oracle at the end.
* Ensemble and served cases (mixed): the same check per case.
"""
import numpy as np
import pytest

from helpers import make_cfg
from oracle import wf_oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p", "ustar", "vstar", "wstar", "uoo", "voo", "woo", "vis",
          "su", "pp")
VEL = ("u", "v", "w")


def _oracle_run(cfg, nsteps):
    """Per-step (info, rmax trace) of the FP64 oracle, the fields after the
    first step and after the last."""
    ora = O.OracleSolver(cfg)
    steps, first = [], None
    for s in range(nsteps):
        q = ora.step()
        steps.append((q, list(ora.rmax_trace)))
        if s == 0:
            first = {k: ora.f[k].copy() for k in FIELDS}
    last = {k: ora.f[k].copy() for k in FIELDS}
    return steps, first, last


@pytest.fixture(scope="module")
def cavity80():
    cfg = make_cfg(n=80, levels=3, vdt=True)
    return cfg, _oracle_run(cfg, 6)


@pytest.fixture(scope="module")
def cavity32():
    cfg = make_cfg(n=32, levels=3, vdt=False)
    return cfg, _oracle_run(cfg, 200)


def _solver(cfg):
    from warpflow import FlowSolver, build_topology
    sol = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    assert sol.step_mode == "graph"
    return sol


def _rms(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)))


def _run_fp64(cfg, ref):
    steps, first, last = ref
    sol = _solver(cfg)
    worst1 = {}
    for s, (q, trace) in enumerate(steps, 1):
        r = sol.step()
        assert r["iters"] == q["iters"], (s, r, q)
        assert r["dt"] == pytest.approx(q["dt"], rel=1e-12)
        assert r["ctime"] == pytest.approx(q["ctime"], rel=1e-12)
        np.testing.assert_allclose(sol.rmax_trace, trace, rtol=1e-5, atol=1e-16)
        if s == 1:
            for k in FIELDS:
                worst1[k] = float(np.abs(sol.f[k].numpy() - first[k]).max())
                assert worst1[k] <= 1e-10, (k, worst1[k])
    rms = {k: _rms(sol.f[k].numpy(), last[k]) for k in VEL}
    for k in VEL:
        assert rms[k] <= 1e-8, (k, rms[k])
    print("fp64 n=%d: first-step max abs %.2e, final rms u/v/w %s"
          % (sol.n, max(worst1.values()), ["%.2e" % rms[k] for k in VEL]))
    return sol


def _run_mixed(cfg, ref):
    steps, _, last = ref
    sol = _solver(cfg)
    assert sol.mixed
    for s, (q, _) in enumerate(steps, 1):
        r = sol.step()
        assert r["rmax"] < cfg.numerics.div_tolerance, (s, r)
    rms = {k: _rms(sol.f[k].numpy(), last[k]) for k in VEL}
    for k in VEL:
        assert rms[k] <= 1e-7, (k, rms[k])
    print("mixed n=%d: final rms u/v/w vs FP64 oracle %s"
          % (sol.n, ["%.2e" % rms[k] for k in VEL]))
    return sol


def test_cavity80_fp64_production_path(cavity80):
    cfg, ref = cavity80
    sol = _run_fp64(cfg, ref)
    # the production kernels were in use: split level 0, coarse operator
    assert sol.mg._cop_part is not None
    assert sol.mg._tmp64 is not None


def test_cavity80_mixed(cavity80):
    _, ref = cavity80
    _run_mixed(make_cfg(n=80, levels=3, vdt=True, precision="mixed"), ref)


def test_cavity32_fixed_dt_200_steps_fp64(cavity32):
    cfg, ref = cavity32
    _run_fp64(cfg, ref)


def test_cavity32_fixed_dt_200_steps_mixed(cavity32):
    _, ref = cavity32
    _run_mixed(make_cfg(n=32, levels=3, vdt=False, precision="mixed"), ref)


def _oracle_final(cfg, nsteps):
    ora = O.OracleSolver(cfg)
    for _ in range(nsteps):
        ora.step()
    return {k: ora.f[k] for k in VEL}


def test_ensemble_cases_match_fp64_oracle():
    """Two cases of different size, Re and lid velocity stepped as one
    ensemble (one graph launch per step, mixed multigrid)."""
    from warpflow.ensemble import Ensemble, cavity_case
    specs = [(16, 250.0, 0.8), (24, 700.0, 1.3)]
    nsteps = 20
    ens = Ensemble([cavity_case(n, re, ul, precision="mixed") for n, re, ul in specs])
    for _ in range(nsteps):
        for info in ens.step():
            assert not isinstance(info, Exception), info
            assert info["rmax"] < 1e-6
    for sol, (n, re, ul) in zip(ens.solvers, specs):
        ref = _oracle_final(cavity_case(n, re, ul, precision="fp64"), nsteps)
        for k in VEL:
            rms = _rms(sol.f[k].numpy(), ref[k])
            assert rms <= 1e-7, (n, k, rms)
    ens.close()


def test_served_case_matches_fp64_oracle():
    """A request served in a mix with another (continuous batching, mixed
    multigrid) ends within 1e-7 rms of the FP64 oracle."""
    from warpflow.ensemble import cavity_case
    from warpflow.serve import CavityServer, Request, levels_for
    reqs = [Request(rid=0, n=24, re=300.0, ulid=1.0, n_steps=15, arrival=0.0,
                    levels=levels_for(24)),
            Request(rid=1, n=16, re=900.0, ulid=0.7, n_steps=25, arrival=0.0,
                    levels=levels_for(16)),
            Request(rid=2, n=24, re=600.0, ulid=1.3, n_steps=10, arrival=0.05,
                    levels=levels_for(24))]
    srv = CavityServer(nstreams=2, keep_fields=True)
    srv.warmup(reqs)
    done = srv.run(reqs)
    # the start-up solvers and finished ones were reset and reused
    assert srv.summary()["solver_reuses"] >= 2
    srv.close()
    for req, c in zip(reqs, done):
        assert not c.error, c.error
        assert c.info["rmax"] < 1e-6
        ref = _oracle_final(cavity_case(req.n, req.re, req.ulid, levels=req.levels,
                                        precision="fp64"), req.n_steps)
        for k in VEL:
            rms = _rms(srv.fields[req.rid][k], ref[k])
            assert rms <= 1e-7, (req.rid, k, rms)
