"""One-launch red-black sweeps (used by default for levels >= 128) forced
on at small sizes in a child process: multigrid solves must match the FP64
oracle, and the mixed form must stay within its tolerance."""
import json
import os
import subprocess
import sys

import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import json, sys
sys.path[:0] = [%r, %r]
import numpy as np
from oracle import wf_oracle as O
from warpflow import Multigrid, build_topology
from warpflow.config import case_from_dict
from warpflow.fields import DeviceField
out = {}
for n, L, prec in ((20, 2, "fp64"), (24, 3, "fp64"), (40, 3, "fp64"), (40, 3, "mixed"), (70, 2, "fp64")):
    cfg = case_from_dict({"grid": {"nx": n, "ny": n, "nz": n},
                          "numerics": {"mg_levels": L, "mg_precision": prec}})
    h = 1.0 / n
    mg = Multigrid(cfg, build_topology(cfg), "cuda:0", h, h, h)
    shape = (n + 6,) * 3
    rhs = np.random.default_rng(n).standard_normal(shape)
    su = DeviceField.zeros(shape, "cuda:0"); pp = DeviceField.zeros(shape, "cuda:0")
    su.assign(rhs)
    mg.solve(su, pp, 3)
    ref = np.zeros(shape)
    O.Multigrid(n, L, h, h, h).solve(rhs, ref, n)
    out["%%d_%%d_%%s" %% (n, L, prec)] = float(np.abs(pp.numpy() - ref).max() / np.abs(ref).max())
    # harness relax with an odd sweep count on level 0 (fp64 only)
    if prec == "fp64":
        lev = mg.levels[0]
        lev.rhs.assign(np.random.default_rng(1).standard_normal(lev.shape))
        lev.phi.zero_()
        mg._relax(0, 5)
        ol = O.Level(n, h, h, h)
        ol.rhs[...] = lev.rhs.numpy()
        for _ in range(5):
            O.rbgs(ol, 0); O.rbgs(ol, 1); O.mg_refill(ol.phi, n)
        out["relax_%%d" %% n] = float(np.abs(lev.phi.numpy() - ol.phi).max() / np.abs(ol.phi).max())
print(json.dumps(out))
""" % (ROOT, PKG)


def test_one_launch_sweeps_match_oracle():
    env = dict(os.environ, WF_SWEEP2_MIN="8")
    r = subprocess.run([sys.executable, "-c", SCRIPT], capture_output=True, text=True,
                       env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    for key, rel in res.items():
        tol = 1e-5 if key.endswith("mixed") else 1e-11
        assert rel <= tol, (key, rel)
