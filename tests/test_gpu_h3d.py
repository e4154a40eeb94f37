"""Hydro3D restart round trip through a solver: export a stepped cavity's
state and import it into a fresh solver of the same case.  The real cells
of u, v, w and p come back bit for bit; the ghost layers are rebuilt as a
fresh solver's are (zero, then the initial fills), and the imported solver
steps on."""
import ctypes

import numpy as np
import pytest

from helpers import make_cfg

pytestmark = pytest.mark.gpu


def test_export_import_round_trip(tmp_path):
    from warpflow import FlowSolver, _abi, build_topology, h3d
    cfg = make_cfg(n=16, levels=3)
    a = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    for _ in range(3):
        a.step()
    path = h3d.export(a, str(tmp_path))
    assert open(str(tmp_path / "final_ctime.dat")).read().startswith("       0")
    b = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    h3d.import_restart(b, path)
    n, P = 16, 3
    core = slice(P, P + n)
    for name in ("u", "v", "w", "p"):
        np.testing.assert_array_equal(b.f[name].numpy()[core, core, core],
                                      a.f[name].numpy()[core, core, core], err_msg=name)
    # the ghosts: the initial fills applied to zero ghosts around these cells
    c = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    for name in ("u", "v", "w", "p"):
        z = np.zeros(c.f[name].shape)
        z[core, core, core] = a.f[name].numpy()[core, core, core]
        c.f[name].assign(z)
    _abi.call("wf_fill_initial", ctypes.byref(c.case), c._stream())
    for name in ("u", "v", "w", "p"):
        np.testing.assert_array_equal(b.f[name].numpy(), c.f[name].numpy(), err_msg=name)
    vis = b.f["vis"].numpy()
    assert np.all(vis[core, core, core] == b.rey)
    b.set_time_state(a.dt, a.ctime, a.itime)
    info = b.step()
    assert info["rmax"] < 1e-6 and np.isfinite(b.f["u"].numpy()).all()
