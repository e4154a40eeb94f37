"""The reference's own tests, run unchanged against this package.

``WF_REFERENCE_TESTS`` names a directory that holds the reference
checkout's ``tests/test_cavity.py`` and ``tests/test_mg.py`` and its
``cases/cavity_serial.yaml`` (the checkout itself, or a copy of those
files); the tests skip when it is unset.

* ``tests/test_cavity.py`` runs under pytest as it is: its 24^3, 30-step
  cavity and the invariants it checks (projection convergence, finite
  fields, exact boundary ghosts).
* ``tests/test_mg.py`` is the reference's multigrid harness: its
  ``make_rhs`` and ``residual`` -- which reads the levels' coefficient
  arrays ``aw ... ap`` -- run on this package's GPU ``Multigrid`` for the
  80^3 benchmark case, and its ``main()`` runs as a script would.
"""
import importlib.util
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PLUGIN_DIR = os.path.join(HERE, "refsuite")
PKG = os.path.join(ROOT, "warpflow-les_b200")


def _ref():
    d = os.environ.get("WF_REFERENCE_TESTS")
    if not d:
        pytest.skip("WF_REFERENCE_TESTS is not set")
    return d


def test_reference_test_cavity_unchanged():
    ref = _ref()
    path = os.path.join(ref, "tests", "test_cavity.py")
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([PLUGIN_DIR, PKG, env.get("PYTHONPATH", "")])
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider",
                        "-p", "wf_refsuite_plugin", path],
                       cwd=ref, env=env, capture_output=True, text=True, timeout=900)
    print(r.stdout[-2000:], r.stderr[-2000:])
    assert r.returncode == 0
    assert "3 passed" in r.stdout


def test_reference_mg_harness_unchanged():
    ref = _ref()
    if PLUGIN_DIR not in sys.path:
        sys.path.insert(0, PLUGIN_DIR)
    import wf_refsuite_plugin  # noqa: F401  (this package's warpflow, the warp stand-in)
    spec = importlib.util.spec_from_file_location(
        "ref_test_mg", os.path.join(ref, "tests", "test_mg.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)

    from warpflow import Multigrid, build_topology, load_case
    cfg = load_case(os.path.join(ref, "cases", "cavity_serial.yaml"))
    topo = build_topology(cfg)
    mg = Multigrid(cfg, topo, "cuda:0", 1.0 / cfg.grid.nx, 1.0 / cfg.grid.ny,
                   1.0 / cfg.grid.nz)
    lev0 = mg.levels[0]
    mod.make_rhs(lev0)
    lev0.phi.zero_()
    mg._refill(lev0)
    r_prev = mod.residual(lev0)
    assert r_prev > 0
    for it in range(6):
        mg._vcycle()
        r = mod.residual(lev0)
        # the reference harness's residual (coefficient views) and the
        # library's residual kernel agree
        assert r == pytest.approx(mg.residual_max(0), rel=1e-9)
        # "a healthy geometric MG drops the residual by 1-2 orders per cycle"
        assert r < 0.2 * r_prev, (it, r, r_prev)
        r_prev = r
    # the harness as a script (prints one residual line per cycle)
    old = sys.argv
    cwd = os.getcwd()
    try:
        os.chdir(ref)
        sys.argv = ["test_mg.py", "cases/cavity_serial.yaml", "3"]
        mod.main()
    finally:
        sys.argv = old
        os.chdir(cwd)
