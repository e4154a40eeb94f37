"""The convection passes specialised on the grid size (k_conv with the padded
extent as a compile-time constant: 86 for 80^3, 262 for 256^3, diffusion
fused in as the step runs it) against the generic form with runtime strides
(WF_CONV_PC=0), which the oracle tests pin at 16^3, 40^3 and 72^3.  The
switch is read once per process, so each form steps in its own process;
SHA-1 of u, v, w, p and pp after the steps must be equal."""
import os
import subprocess
import sys

import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu


def child(n, levels, steps):
    import hashlib

    from helpers import make_cfg
    from warpflow import FlowSolver, build_topology
    cfg = make_cfg(n, levels=levels)
    sol = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    for _ in range(steps):
        sol.step()
    h = hashlib.sha1()
    for name in ("u", "v", "w", "p", "pp"):
        h.update(sol.f[name].numpy().tobytes())
    print("sha1", sol.step_mode, h.hexdigest())


def _run(n, levels, steps, generic):
    env = dict(os.environ)
    env.pop("WF_CONV_PC", None)
    env.pop("WF_STEP_MODE", None)
    if generic:
        env["WF_CONV_PC"] = "0"
    code = ("import sys; sys.path[:0] = %r; import test_gpu_conv_specialised as t; "
            "t.child(%d, %d, %d)" % ([os.path.join(ROOT, "tests"), PKG, ROOT], n, levels, steps))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("sha1 ")][-1]
    return line.split()[1:]


@pytest.mark.parametrize("n,levels,steps", [(80, 3, 2), (256, 5, 1)])
def test_specialised_convection_equals_generic(n, levels, steps):
    mode_s, spec = _run(n, levels, steps, generic=False)
    mode_g, gen = _run(n, levels, steps, generic=True)
    assert mode_s == mode_g == "graph"
    assert spec == gen
