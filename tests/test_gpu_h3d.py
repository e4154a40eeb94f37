"""Hydro3D restart round trip through a solver: export a stepped cavity's
state, import it into a fresh solver of the same case, and the real cells
and this package's ghost layers of u, v, w, p are identical; the imported
solver then steps exactly like the original (vis = 1/Re everywhere in the
exported file, as the reference writes it, so both start from that)."""
import numpy as np
import pytest

from helpers import make_cfg

pytestmark = pytest.mark.gpu


def test_export_import_round_trip(tmp_path):
    from warpflow import FlowSolver, build_topology, h3d
    cfg = make_cfg(n=16, levels=3)
    a = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    for _ in range(3):
        a.step()
    path = h3d.export(a, str(tmp_path))
    assert open(str(tmp_path / "final_ctime.dat")).read().startswith("       0")
    b = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    h3d.import_restart(b, path)
    for name in ("u", "v", "w", "p"):
        np.testing.assert_array_equal(b.f[name].numpy(), a.f[name].numpy(), err_msg=name)
    # the same state in both: vis from the file (1/Re) and the same time
    a.f["vis"].assign(b.f["vis"].numpy())
    b.set_time_state(a.dt, a.ctime, a.itime)
    for _ in range(2):
        assert a.step() == b.step()
    for name in ("u", "v", "w", "p", "vis"):
        np.testing.assert_array_equal(b.f[name].numpy(), a.f[name].numpy(), err_msg=name)
