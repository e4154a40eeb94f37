"""Mixed-precision multigrid (FP32 V-cycles inside an FP64 defect
correction) against the FP64 oracle.  Tolerances: the solve within 1e-5
relative of the FP64 4-cycle result; a cavity run keeps every step's
divergence below div_tolerance with the FP64 iteration counts and stays
within 1e-7 rms (velocity) of the FP64 oracle."""
import numpy as np
import pytest

from helpers import make_cfg
from oracle import wf_oracle as O

pytestmark = pytest.mark.gpu


def _mg(n, levels, precision):
    from warpflow import Multigrid, build_topology
    cfg = make_cfg(n=n, levels=levels, precision=precision)
    h = 1.0 / n
    return Multigrid(cfg, build_topology(cfg), "cuda:0", h, h, h)


@pytest.mark.parametrize("n,levels", [(32, 3), (64, 3), (64, 5)])
def test_mixed_solve_close_to_fp64(n, levels):
    from warpflow.fields import DeviceField
    mg = _mg(n, levels, "mixed")
    shape = (n + 6,) * 3
    rhs = np.random.default_rng(3).standard_normal(shape)
    su = DeviceField.zeros(shape, "cuda:0")
    pp = DeviceField.zeros(shape, "cuda:0")
    su.assign(rhs)
    mg.solve(su, pp, 3)
    ref = np.zeros(shape)
    h = 1.0 / n
    O.Multigrid(n, levels, h, h, h).solve(rhs, ref, n)
    rel = np.abs(pp.numpy() - ref).max() / np.abs(ref).max()
    assert rel <= 1e-5, rel


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_defect_correction_reaches_1e10(precision):
    """Standalone Poisson (tests/test_mg.py harness): cycles until the max
    residual drops by 1e10; the mixed form needs at most two more cycles
    than the FP64 form and reaches the same FP64 accuracy."""
    n, levels = 32, 4
    mg = _mg(n, levels, precision)
    lev0 = mg.levels[0]
    rhs = O.make_mg_rhs(n, 0)
    lev0.rhs.assign(rhs)
    lev0.phi.zero_()
    mg._refill(lev0)
    r0 = mg.residual_max(0)
    cycles = 0
    while mg.residual_max(0) > 1e-10 * r0 and cycles < 40:
        mg._vcycle()
        cycles += 1
    assert mg.residual_max(0) <= 1e-10 * r0
    assert cycles <= 14, cycles
    # the FP64 oracle run of the same number of FP64 cycles
    omg = O.Multigrid(n, levels, 1.0 / n, 1.0 / n, 1.0 / n)
    omg.levels[0].rhs[...] = rhs
    for _ in range(cycles):
        omg.vcycle()
    ref = omg.levels[0].phi
    got = lev0.phi.numpy()
    s = slice(1, n + 1)
    # solutions of the singular Neumann problem agree up to round-off level
    d = got[s, s, s] - ref[s, s, s]
    assert np.abs(d - d.mean()).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.slow
def test_mixed_cavity_run_within_tolerance():
    cfg_m = make_cfg(n=32, levels=3, vdt=True, precision="mixed")
    cfg_d = make_cfg(n=32, levels=3, vdt=True, precision="fp64")
    from warpflow import FlowSolver, build_topology
    sol = FlowSolver(cfg_m, build_topology(cfg_m), "cuda:0")
    ora = O.OracleSolver(cfg_d)
    for s in range(40):
        r = sol.step()
        q = ora.step()
        assert r["rmax"] < 1e-6
        assert r["iters"] == q["iters"], (s, r, q)
    for name in ("u", "v", "w"):
        a, b = sol.f[name].numpy(), ora.f[name]
        rms = float(np.sqrt(np.mean((a - b) ** 2)))
        assert rms <= 1e-7, (name, rms)
