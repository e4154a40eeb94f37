"""Sub-domain decomposition on the GPU: the product's FlowSolver at 2 and 8
ranks (one process per rank, all on cuda:0, halos through gloo; the ranks'
kernels never wait on one another) against the goldens made by running the
reference's own source decomposed the same way.  Every field of every rank
after every step within 1e-10, the same outer-iteration counts, dt within
1e-12 relative."""
import os

import numpy as np
import pytest
import yaml

from conftest import GOLDEN
from ranks_util import run_ranks

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "p", "ustar", "vstar", "wstar", "uoo", "voo", "woo", "vis", "su",
          "pp")


def gpu_rank(rank, nranks, tag):
    from warpflow import FlowSolver, build_topology
    from warpflow.config import case_from_dict
    g = np.load(os.path.join(GOLDEN, "golden_%s.npz" % tag))
    cfg = case_from_dict(yaml.safe_load(str(g["case_yaml"])))
    sol = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    out = {}
    for name in ("u", "v", "w", "p", "vis"):
        out["init_" + name] = sol.f[name].numpy().copy()
    infos = []
    for s in range(1, cfg.time.n_steps + 1):
        info = sol.step()
        infos.append([info["ctime"], info["dt"], info["rmax"], info["iters"], info["cfl"]])
        for name in FIELDS:
            out["s%d_%s" % (s, name)] = sol.f[name].numpy().copy()
    out["info"] = np.array(infos)
    out["mode"] = np.array(sol.step_mode)
    return out


@pytest.mark.parametrize("tag", ["r2x_16x8x8_l3", "r8_16_l2"])
def test_decomposed_solver_matches_reference(tag):
    g = np.load(os.path.join(GOLDEN, "golden_%s.npz" % tag))
    nr = int(g["nranks"])
    res = run_ranks("test_gpu_ranks", "gpu_rank", nr, (tag,), timeout=900)
    worst = 0.0
    for r, out in enumerate(res):
        assert str(out["mode"]) == "ranks"
        ref_info = g["r%d_info" % r]
        np.testing.assert_array_equal(out["info"][:, 3], ref_info[:, 3])
        np.testing.assert_allclose(out["info"][:, 1], ref_info[:, 1], rtol=1e-12, atol=0)
        np.testing.assert_allclose(out["info"][:, 2], ref_info[:, 2], rtol=1e-6, atol=1e-14)
        for key in out:
            if key in ("info", "mode"):
                continue
            d = float(np.abs(out[key] - g["r%d_%s" % (r, key)]).max())
            worst = max(worst, d)
            assert d <= 1e-10, (tag, r, key, d)
    print("%s: %d ranks, max |gpu - reference| = %.3e" % (tag, nr, worst))


def test_cli_decomposed_under_torchrun(tmp_path):
    """run.py under torchrun at 2 ranks (halos through gloo, both ranks on
    cuda:0): the reference's log lines from rank 0, one snapshot per rank,
    and each rank's final fields equal to the reference's decomposed run."""
    import socket
    import subprocess
    import sys

    from conftest import PKG
    g = np.load(os.path.join(GOLDEN, "golden_r2x_16x8x8_l3.npz"))
    raw = yaml.safe_load(str(g["case_yaml"]))
    raw["output"]["outdir"] = str(tmp_path / "out")
    case = tmp_path / "case.yaml"
    case.write_text(yaml.safe_dump(raw))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, WF_DIST_BACKEND="gloo")
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                        "--master-port", str(port), os.path.join(PKG, "run.py"),
                        "--case", str(case)],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    its = [l for l in r.stdout.splitlines() if l.startswith("it ")]
    assert len(its) == 2, r.stdout
    assert "domains=[2, 1, 1]" in r.stdout
    for rank in range(2):
        z = np.load(tmp_path / "out" / ("snap_000002_r%03d.npz" % rank))
        for name in ("u", "v", "w", "p"):
            d = float(np.abs(z[name] - g["r%d_s2_%s" % (rank, name)]).max())
            assert d <= 1e-10, (rank, name, d)
        assert tuple(z["offsets"]) == (8 * rank, 0, 0)
