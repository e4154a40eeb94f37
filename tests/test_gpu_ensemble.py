"""Batched ensemble and continuous-batching server (GPU): a case's result
is the same alone and inside the mix (bit for bit: same kernels, same
arithmetic, no cross-case coupling), and the served stream respects its
memory budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPECS = [(16, 150.0, 0.8), (24, 900.0, 1.3), (32, 400.0, 1.0), (16, 600.0, 0.6)]


def _alone(n, re, ulid, steps, precision):
    from warpflow import FlowSolver, build_topology
    from warpflow.ensemble import cavity_case
    cfg = cavity_case(n, re, ulid, precision=precision)
    sol = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    infos = [sol.step() for _ in range(steps)]
    return infos, {k: sol.f[k].numpy() for k in ("u", "v", "w", "p", "vis")}


@pytest.mark.parametrize("single_graph", [True, False], ids=["one_graph", "streams"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ensemble_matches_alone(precision, single_graph):
    from warpflow.ensemble import Ensemble, cavity_case
    cfgs = [cavity_case(n, re, u, precision=precision) for n, re, u in SPECS]
    ens = Ensemble(cfgs, nstreams=3, single_graph=single_graph)
    assert (ens._graph is not None) == single_graph
    steps = 4
    for _ in range(steps):
        infos = ens.step()
        assert all(isinstance(i, dict) for i in infos)
    for k, (n, re, u) in enumerate(SPECS):
        ref_infos, ref = _alone(n, re, u, steps, precision)
        sol = ens.solvers[k]
        assert sol.outer_iters == ref_infos[-1]["iters"]
        assert sol.dt == ref_infos[-1]["dt"]
        for name, arr in ref.items():
            np.testing.assert_array_equal(sol.f[name].numpy(), arr)


@pytest.mark.parametrize("serial", [False, True])
def test_reset_matches_fresh_solver(serial):
    """A solver reset on the device for a new case (Re, lid velocity) steps
    exactly like a solver built for that case (the server's reuse)."""
    from warpflow import FlowSolver, build_topology
    from warpflow.ensemble import cavity_case
    a_cfg = cavity_case(24, 300.0, 0.8, precision="mixed")
    b_cfg = cavity_case(24, 700.0, 1.2, precision="mixed")
    a = FlowSolver(a_cfg, build_topology(a_cfg), "cuda:0", serial=serial)
    for _ in range(3):
        a.step()
    a.reset(b_cfg)
    b = FlowSolver(b_cfg, build_topology(b_cfg), "cuda:0", serial=serial)
    for _ in range(5):
        assert a.step() == b.step()
    for name in ("u", "v", "w", "p", "vis", "su", "pp", "uoo"):
        np.testing.assert_array_equal(a.f[name].numpy(), b.f[name].numpy(), err_msg=name)
    assert (a.itime, a.rey, a.ulid) == (b.itime, b.rey, b.ulid)
    with pytest.raises(ValueError):
        a.reset(cavity_case(32, 700.0, 1.2, precision="mixed"))


def test_case_bytes_matches_allocation():
    from warpflow import FlowSolver, build_topology
    from warpflow.ensemble import cavity_case
    from warpflow.serve import case_bytes
    for n, prec in ((32, "mixed"), (48, "fp64")):
        cfg = cavity_case(n, precision=prec)
        sol = FlowSolver(cfg, build_topology(cfg), "cuda:0")
        assert sol.device_bytes() == case_bytes(n, 3, prec)


def test_server_stream_matches_alone_and_budget():
    from warpflow.serve import CavityServer, Request, case_bytes, operator_bytes
    reqs = [Request(0, 16, 300.0, 1.0, 6, arrival=0.00),
            Request(1, 32, 700.0, 0.7, 3, arrival=0.01),
            Request(2, 16, 900.0, 1.2, 5, arrival=0.02),
            Request(3, 24, 200.0, 1.0, 4, arrival=0.03),
            Request(4, 16, 500.0, 0.9, 2, arrival=0.50)]
    # forces queueing; the shared coarse operators are charged once each
    budget = case_bytes(32) + case_bytes(16) + operator_bytes(32) + operator_bytes(16) + 4096
    srv = CavityServer(budget_bytes=budget, nstreams=4, keep_fields=True)
    srv.warmup(reqs)          # start-up cases leave no trace in the served ones
    done = srv.run(reqs)
    assert [c.rid for c in done] == [0, 1, 2, 3, 4]
    assert all(c.steps == r.n_steps and not c.error for c, r in zip(done, reqs))
    assert srv.adm.peak <= budget
    assert all(c.finished >= c.admitted >= 0 for c in done)
    s = srv.summary()
    assert s["p99_s"] >= s["p50_s"] > 0
    for r in reqs:
        _, ref = _alone(r.n, r.re, r.ulid, r.n_steps, r.precision)
        for name in ("u", "v", "w", "p"):
            np.testing.assert_array_equal(srv.fields[r.rid][name], ref[name])
