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
    ens = Ensemble(cfgs, nstreams=3, single_graph=single_graph, buckets=False)
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


BUCKET_SPECS = [(16, 150.0, 0.8, 0.01), (24, 900.0, 1.3, 0.01), (16, 600.0, 0.6, 0.05),
                (24, 300.0, 1.0, 0.002), (16, 950.0, 1.4, 0.02), (32, 400.0, 1.0, 0.01)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bucketed_ensemble_matches_alone(precision):
    """Cases of the same size share every launch of their bucket; each case
    still computes exactly what it computes alone, step by step, including
    when cases of one bucket need different numbers of outer iterations."""
    from warpflow import FlowSolver, build_topology
    from warpflow.ensemble import Ensemble, cavity_case
    cfgs = [cavity_case(n, re, u, precision=precision, noise=nz) for n, re, u, nz in BUCKET_SPECS]
    mixed = Ensemble(cfgs[:2], nstreams=1)      # two sizes: a branch per case by default
    assert not mixed.buckets and mixed.layout()[0] == [0, 1]
    mixed.close()
    ens = Ensemble(cfgs, nstreams=2, buckets=True)
    bucket, counts = ens.layout()
    assert len(counts) == 3 and bucket[0] == bucket[2] == bucket[4] != bucket[1]
    alone = [FlowSolver(c, build_topology(c), "cuda:0") for c in cfgs]
    differing = 0
    for _ in range(5):
        infos = ens.step()
        refs = [s.step() for s in alone]
        assert infos == refs
        its = [i["iters"] for i, b in zip(infos, bucket) if b == bucket[0]]
        differing += len(set(its)) > 1
    for sol, ref in zip(ens.solvers, alone):
        for name in ("u", "v", "w", "p", "vis", "su", "pp"):
            np.testing.assert_array_equal(sol.f[name].numpy(), ref.f[name].numpy(),
                                          err_msg=name)
    assert differing >= 1, "no step had cases of one bucket at different iteration counts"
    # the same step with a branch per case launches every kernel per case
    per_case = 0
    for s in ens.solvers:
        c0, c1, c2, c3 = s.launch_counts()
        per_case += c0 + c3 + s.outer_iters * c1 + s.last_nmg * c2
    assert ens.launches_per_step() < per_case
    ens.close()


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


def test_bucket_with_cluster_coarse_sweeps():
    """A bucket whose coarsest level relaxes by sweeps at a size where a
    lone case would use a thread-block-cluster kernel (24^3: cluster
    kernels cannot serve a bucket's case table) falls back to the one-CTA
    kernel: the bucket is built and each case agrees with its lone run to
    rounding (a different sweep kernel, the same sweeps)."""
    from warpflow import FlowSolver, build_topology
    from warpflow.ensemble import Ensemble, cavity_case
    cfgs = []
    for re in (200.0, 500.0, 800.0):
        c = cavity_case(48, re, 1.0, levels=2, precision="fp64")
        c.numerics.mg_coarse = "sweeps"
        cfgs.append(c)
    ens = Ensemble(cfgs, nstreams=1)          # one size: bucketed by default
    assert ens.buckets
    bucket, counts = ens.layout()
    assert len(counts) == 1 and bucket == [0, 0, 0]
    alone = [FlowSolver(c, build_topology(c), "cuda:0") for c in cfgs]
    for _ in range(2):
        infos = ens.step()
        refs = [s.step() for s in alone]
        assert [i["iters"] for i in infos] == [r["iters"] for r in refs]
    for sol, ref in zip(ens.solvers, alone):
        for name in ("u", "v", "w", "p"):
            a, b = sol.f[name].numpy(), ref.f[name].numpy()
            assert np.abs(a - b).max() <= 1e-10 * max(1.0, np.abs(b).max()), name
    ens.close()
