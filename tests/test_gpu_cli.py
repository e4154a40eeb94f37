"""CLI and snapshot resume (GPU): the reference's log format, snapshot
layout, and an exact resume (3 + 3 steps == 6 steps, bit for bit)."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest
import yaml

from conftest import PKG
from helpers import CASE_TMPL

pytestmark = pytest.mark.gpu


def _case(tmp_path, n=16, steps=6, n_out=3):
    raw = yaml.safe_load(yaml.safe_dump(CASE_TMPL))
    raw["grid"] = {"nx": n, "ny": n, "nz": n}
    raw["time"]["n_steps"] = steps
    raw["output"] = {"n_out": n_out, "log_interval": 1, "outdir": str(tmp_path / "out")}
    p = tmp_path / "case.yaml"
    p.write_text(yaml.safe_dump(raw))
    return p


def test_cli_log_and_snapshots(tmp_path):
    case = _case(tmp_path)
    r = subprocess.run([sys.executable, os.path.join(PKG, "run.py"), "--case", str(case)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[0].startswith("warpflow-les 0.1.0: case=cavity_test grid=16x16x16")
    pat = re.compile(r"^it +\d+  ctime \d\.\d{6}  dt \d\.\d{3}e[+-]\d\d  rmax \d\.\d{3}e[+-]\d\d"
                     r"  outer +\d+  cfl \d+\.\d\d$")
    its = [l for l in lines if l.startswith("it ")]
    assert len(its) == 6 and all(pat.match(l) for l in its), its
    assert lines[-1].startswith("done: itime=6 ctime=")
    snaps = sorted(os.listdir(tmp_path / "out"))
    assert snaps == ["snap_000003_r000.npz", "snap_000006_r000.npz"]
    z = np.load(tmp_path / "out" / snaps[-1])
    for k in ("u", "v", "w", "p", "ctime", "dt", "offsets", "ncells", "gshape"):
        assert k in z.files
    assert z["u"].shape == (22, 22, 22)


def test_resume_is_exact(tmp_path):
    from warpflow import FlowSolver, build_topology, load_case
    from warpflow.io import read_snapshot, restore, write_snapshot
    cfg = load_case(_case(tmp_path))
    a = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    for _ in range(6):
        a.step()
    b = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    for _ in range(3):
        b.step()
    path = write_snapshot(b, 3)
    c = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    restore(c, read_snapshot(path))
    assert c.itime == 3 and c.dt == b.dt
    for _ in range(3):
        info = c.step()
    assert c.itime == 6 and info["ctime"] == a.ctime
    for k in ("u", "v", "w", "p", "vis"):
        np.testing.assert_array_equal(c.f[k].numpy(), a.f[k].numpy())


def test_async_snapshot_matches_sync(tmp_path):
    """A snapshot taken by SnapshotWriter while the solver keeps stepping is
    the same file content as write_snapshot at that step."""
    from warpflow import FlowSolver, build_topology, load_case
    from warpflow.io import SnapshotWriter, read_snapshot, write_snapshot
    cfg = load_case(_case(tmp_path))
    cfg.output.outdir = str(tmp_path / "async")
    a = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    w = SnapshotWriter(a)
    for _ in range(3):
        a.step()
    w.write(3)
    for _ in range(2):        # later steps overwrite the fields meanwhile
        a.step()
    path = w.wait()
    w.close()
    cfg2 = load_case(_case(tmp_path))
    cfg2.output.outdir = str(tmp_path / "sync")
    b = FlowSolver(cfg2, build_topology(cfg2), "cuda:0")
    for _ in range(3):
        b.step()
    ref = read_snapshot(write_snapshot(b, 3))
    got = read_snapshot(path)
    assert sorted(got) == sorted(ref)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
