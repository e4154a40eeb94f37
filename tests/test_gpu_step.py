"""Whole-step parity of FlowSolver (GPU) against the reference.

* golden vectors from the reference's own source: every field, ghosts
  included, within 1e-10 max abs after each recorded step, with identical
  outer-iteration counts, dt and ctime;
* the CPU oracle over longer runs: 1e-10 max abs after 1 step, the same
  divergence trajectory and iteration counts, and 1e-8 rms after 100 steps;
* the reference's own regression invariants (tests/test_cavity.py:68-111).
"""
import numpy as np
import pytest

from helpers import GOLDEN_CAVITY, golden, golden_cfg, make_cfg
from oracle import wf_oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p", "ustar", "vstar", "wstar", "uoo", "voo", "woo", "vis",
          "su", "pp")


def _solver(cfg, mode=None):
    from warpflow import FlowSolver, build_topology
    return FlowSolver(cfg, build_topology(cfg), "cuda:0", step_mode=mode)


@pytest.mark.parametrize("mode", ["graph", "host"])
@pytest.mark.parametrize("tag", GOLDEN_CAVITY)
def test_step_matches_reference_golden(tag, mode):
    g = golden(tag)
    sol = _solver(golden_cfg(g), mode)
    for name in ("u", "v", "w", "p", "vis"):
        np.testing.assert_array_equal(sol.f[name].numpy(), g["init_" + name])
    info = g["info"]
    for s in range(1, len(info) + 1):
        r = sol.step()
        ref = info[s - 1]
        assert r["iters"] == int(ref[3]), (s, r, ref)
        assert r["dt"] == pytest.approx(ref[1], rel=1e-13)
        assert r["ctime"] == pytest.approx(ref[0], rel=1e-13)
        assert r["rmax"] == pytest.approx(ref[2], rel=1e-6)
        assert r["cfl"] == pytest.approx(ref[4], rel=1e-10)
        for key in g.files:
            if key.startswith("s%d_" % s):
                name = key.split("_", 1)[1]
                d = float(np.abs(sol.f[name].numpy() - g[key]).max())
                assert d <= 1e-10, (tag, s, name, d)


def test_serial_stepper_bit_identical():
    """A stepper built without programmatic dependent launch (the default)
    and one built with it compute exactly the same step."""
    from warpflow import FlowSolver, build_topology
    cfg = make_cfg(24, levels=3)
    a = FlowSolver(cfg, build_topology(cfg), "cuda:0", serial=False)
    b = FlowSolver(cfg, build_topology(cfg), "cuda:0", serial=True)
    for _ in range(3):
        ra, rb = a.step(), b.step()
        assert ra == rb
    for name in FIELDS:
        np.testing.assert_array_equal(a.f[name].numpy(), b.f[name].numpy())


def test_old_velocities_are_the_whole_pre_step_fields():
    """uoo/voo/woo hold u/v/w as they were when the step began, ghost layers
    included (solver.py:223-225; the step copies them in its dt pass)."""
    sol = _solver(make_cfg(20, levels=2))
    sol.step()
    before = {k: sol.f[k].numpy() for k in ("u", "v", "w")}
    sol.step()
    for k in ("u", "v", "w"):
        np.testing.assert_array_equal(sol.f[k + "oo"].numpy(), before[k])


def _compare_run(cfg, nsteps, check_every=1):
    sol = _solver(cfg)
    ora = O.OracleSolver(cfg)
    worst = 0.0
    for s in range(1, nsteps + 1):
        r = sol.step()
        q = ora.step()
        assert r["iters"] == q["iters"], (s, r, q)
        assert r["dt"] == pytest.approx(q["dt"], rel=1e-12)
        np.testing.assert_allclose(sol.rmax_trace, ora.rmax_trace, rtol=1e-5, atol=1e-16)
        if s % check_every == 0 or s == nsteps:
            for name in ("u", "v", "w", "p", "vis"):
                a, b = sol.f[name].numpy(), ora.f[name]
                if name == "p":  # p is defined up to the solver's own constant drift
                    pass
                worst = max(worst, float(np.abs(a - b).max()))
    return sol, ora, worst


def test_one_step_1e10_at_32():
    """The 32^3 fixed-dt cavity, first step: every field within 1e-10."""
    cfg = make_cfg(n=32, levels=3, vdt=False)
    sol = _solver(cfg)
    ora = O.OracleSolver(cfg)
    sol.step()
    ora.step()
    for name in FIELDS:
        d = float(np.abs(sol.f[name].numpy() - ora.f[name]).max())
        assert d <= 1e-10, (name, d)


@pytest.mark.slow
def test_100_steps_rms_1e8_at_16():
    """100 steps (variable dt): rms difference of u, v, w <= 1e-8 and the
    same outer-iteration count on every step."""
    cfg = make_cfg(n=16, levels=3, vdt=True)
    sol, ora, _ = _compare_run(cfg, 100, check_every=25)
    for name in ("u", "v", "w"):
        a, b = sol.f[name].numpy(), ora.f[name]
        rms = float(np.sqrt(np.mean((a - b) ** 2)))
        assert rms <= 1e-8, (name, rms)


@pytest.fixture(scope="module")
def cavity24():
    """The reference regression case: 24^3, 3 levels, 30 steps."""
    cfg = make_cfg(n=24, levels=3)
    sol = _solver(cfg)
    infos = [sol.step() for _ in range(30)]
    return sol, infos


def test_projection_converges(cavity24):
    _, infos = cavity24
    for info in infos:
        assert info["rmax"] < 1.0e-6
        assert info["iters"] <= 6


def test_fields_finite(cavity24):
    sol, _ = cavity24
    for name in ("u", "v", "w", "p", "vis"):
        assert np.isfinite(sol.f[name].numpy()).all(), name


def test_boundary_ghosts(cavity24):
    sol, _ = cavity24
    n, P = sol.ncells[0], 3
    s = slice(P, P + n)
    u, v, w, p = (sol.f[k].numpy() for k in ("u", "v", "w", "p"))
    assert np.allclose(u[P:P + n, P:P + n, P + n], sol.ulid)
    assert np.allclose(u[P - 1, s, s], 0.0) and np.allclose(u[P + n, s, s], 0.0)
    assert np.allclose(v[s, P - 1, s], 0.0) and np.allclose(v[s, P + n, s], 0.0)
    assert np.allclose(w[s, s, P - 1], 0.0) and np.allclose(w[s, s, P + n], 0.0)
    assert np.allclose(p[P - 1, s, s], p[P, s, s])
    assert np.allclose(p[P + n, s, s], p[P + n - 1, s, s])
    assert np.allclose(p[s, P - 1, s], p[s, P, s])
    assert np.allclose(p[s, P + n, s], p[s, P + n - 1, s])
    assert np.allclose(p[s, s, P - 1], p[s, s, P])
    assert np.allclose(p[s, s, P + n], p[s, s, P + n - 1])


def test_divergence_error_raised():
    """A blown-up state raises the reference's message (solver.py:190-193);
    the failure is made on the host by planting a huge velocity."""
    cfg = make_cfg(n=16, levels=3)
    sol = _solver(cfg)
    u = sol.f["u"].numpy()
    u[8, 8, 8] = 1.0e9
    sol.f["u"].assign(u)
    with pytest.raises(RuntimeError, match="projection diverged|time step collapsed"):
        sol.step()


def test_dt_collapse_raised():
    cfg = make_cfg(n=16, levels=3)
    sol = _solver(cfg)
    vis = sol.f["vis"].numpy()
    vis[:] = -1.0e30  # negative viscosity -> dtmax <= 0 (solver.py:143-144)
    sol.f["vis"].assign(vis)
    with pytest.raises(RuntimeError, match="time step collapsed"):
        sol.step()
