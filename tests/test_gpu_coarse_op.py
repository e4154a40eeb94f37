"""The coarsest-level relax applied through its precomputed symmetric
operator (representative columns) against the same relax run as sweeps: multigrid solves agree to rounding at every
supported coarse size, both match the FP64 oracle, the FP32 operator serves
the mixed form, applications are deterministic, and whole steps reproduce the
sweeping solver."""
import numpy as np
import pytest

from helpers import make_cfg
from oracle import wf_oracle as O

pytestmark = pytest.mark.gpu


def _solve(n, L, prec, coarse, seed=3, hs=(1.0, 1.0, 1.0)):
    from warpflow import Multigrid, build_topology
    from warpflow.config import case_from_dict
    from warpflow.fields import DeviceField
    cfg = case_from_dict({"grid": {"nx": n, "ny": n, "nz": n},
                          "numerics": {"mg_levels": L, "mg_precision": prec,
                                       "mg_coarse": coarse}})
    h = 1.0 / n
    mg = Multigrid(cfg, build_topology(cfg), "cuda:0", h * hs[0], h * hs[1], h * hs[2])
    shape = (n + 6,) * 3
    rhs = np.random.default_rng(seed).standard_normal(shape)
    su = DeviceField.zeros(shape, "cuda:0")
    pp = DeviceField.zeros(shape, "cuda:0")
    su.assign(rhs)
    mg.solve(su, pp, 3)
    return rhs, pp.numpy(), mg


@pytest.mark.parametrize("n", [16, 32, 48, 64, 80, 96])   # coarsest 4, 8, ..., 24
def test_operator_matches_sweeps_and_oracle(n):
    rhs, a, mg = _solve(n, 3, "fp64", "operator")
    assert mg._cop_part is not None          # the operator path was taken
    _, b, _ = _solve(n, 3, "fp64", "sweeps")
    scale = np.abs(b).max()
    assert np.abs(a - b).max() <= 1e-12 * scale
    if n <= 48:
        h = 1.0 / n
        ref = np.zeros_like(rhs)
        O.Multigrid(n, 3, h, h, h).solve(rhs, ref, n)
        assert np.abs(a - ref).max() <= 1e-11 * np.abs(ref).max()


@pytest.mark.parametrize("hs", [(1.0, 1.3, 1.0), (1.0, 1.3, 0.7)], ids=["two_equal", "none_equal"])
def test_operator_with_unequal_spacing(hs):
    """Fewer symmetries (8 or 4 maps instead of 24): more stored columns, the
    same product."""
    _, a, mg = _solve(80, 3, "fp64", "operator", hs=hs)
    assert mg._cop_part is not None
    _, b, _ = _solve(80, 3, "fp64", "sweeps", hs=hs)
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_operator_mixed_precision():
    _, a, mg = _solve(80, 3, "mixed", "operator")
    assert mg._cop_part is not None
    _, b, _ = _solve(80, 3, "mixed", "sweeps")
    _, c, _ = _solve(80, 3, "fp64", "sweeps")
    assert np.abs(a - b).max() <= 1e-5 * np.abs(c).max()
    assert np.abs(a - c).max() <= 1e-5 * np.abs(c).max()


def test_operator_deterministic():
    _, a, _ = _solve(64, 3, "fp64", "operator", seed=5)
    _, b, _ = _solve(64, 3, "fp64", "operator", seed=5)
    np.testing.assert_array_equal(a, b)


def test_unsupported_size_falls_back_to_sweeps():
    _, a, mg = _solve(72, 3, "fp64", "operator")   # coarsest 18
    assert mg._cop_part is None


def test_steps_match_sweeping_solver():
    from warpflow import FlowSolver, build_topology
    out = []
    for coarse in ("operator", "sweeps"):
        cfg = make_cfg(40, levels=3)
        cfg.numerics.mg_coarse = coarse
        sol = FlowSolver(cfg, build_topology(cfg), "cuda:0")
        infos = [sol.step() for _ in range(5)]
        out.append((infos, {k: sol.f[k].numpy() for k in ("u", "v", "w", "p")}))
    (ia, fa), (ib, fb) = out
    assert [r["iters"] for r in ia] == [r["iters"] for r in ib]
    for k in fa:
        assert np.abs(fa[k] - fb[k]).max() <= 1e-12, k
