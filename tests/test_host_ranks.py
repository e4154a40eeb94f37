"""Sub-domain decomposition on the CPU (gloo, one process per rank): the
oracle's decomposed form against goldens made by running the reference's
own source at 2 and 8 ranks (tests/golden/make_golden.py ranks), and the
product's topology against the same runs."""
import os

import numpy as np
import pytest
import yaml

from conftest import GOLDEN
from ranks_util import run_ranks

CASES = ["r2x_16x8x8_l3", "r8_16_l2"]
FIELDS = ("u", "v", "w", "p", "ustar", "vstar", "wstar", "uoo", "voo", "woo", "vis", "su",
          "pp")


def _golden(tag):
    return np.load(os.path.join(GOLDEN, "golden_%s.npz" % tag))


def _cfg(g):
    from warpflow.config import case_from_dict
    return case_from_dict(yaml.safe_load(str(g["case_yaml"])))


def oracle_rank(rank, nranks, tag):
    """One rank of the decomposed oracle run of golden `tag`."""
    from oracle import wf_oracle as O
    g = _golden(tag)
    cfg = _cfg(g)
    sd = tuple(int(m) for m in cfg.mpi.domains)
    sol = O.OracleSolver(cfg, O.RankComm(O.cart_neighbors(rank, sd)))
    out = {}
    for name in ("u", "v", "w", "p", "vis"):
        out["init_" + name] = sol.f[name].copy()
    infos = []
    for s in range(1, cfg.time.n_steps + 1):
        info = sol.step()
        infos.append([info["ctime"], info["dt"], info["rmax"], info["iters"], info["cfl"]])
        for name in FIELDS:
            out["s%d_%s" % (s, name)] = sol.f[name].copy()
    out["info"] = np.array(infos)
    return out


def topo_rank(rank, nranks, tag):
    """The product's build_topology at one rank of the run of golden `tag`."""
    from warpflow import build_topology
    topo = build_topology(_cfg(_golden(tag)))
    nb = np.array([topo.neighbors[a] for a in "xyz"])
    return {"coords": np.array(topo.coords), "local": np.array(topo.local_ncells),
            "neighbors": nb, "rank": np.array(topo.rank), "nranks": np.array(topo.nranks),
            "offsets": np.array(topo.global_offsets),
            "ar": np.array(topo.comm.allreduce(float(rank), op="max"))}


@pytest.mark.parametrize("tag", CASES)
def test_cart_neighbors_follow_mpi_row_major(tag):
    from oracle import wf_oracle as O
    g = _golden(tag)
    sd = tuple(int(m) for m in _cfg(g).mpi.domains)
    for r in range(int(g["nranks"])):
        want = g["r%d_neighbors" % r]
        got = O.cart_neighbors(r, sd)
        for a, name in enumerate("xyz"):
            assert [x if x >= 0 else -1 for x in want[a]] == list(got[name]), (r, name)


@pytest.mark.parametrize("tag", CASES)
def test_decomposed_oracle_matches_reference(tag):
    g = _golden(tag)
    nr = int(g["nranks"])
    res = run_ranks("test_host_ranks", "oracle_rank", nr, (tag,))
    for r, out in enumerate(res):
        np.testing.assert_array_equal(out["info"][:, 3], g["r%d_info" % r][:, 3])
        np.testing.assert_allclose(out["info"], g["r%d_info" % r], rtol=1e-12, atol=0)
        for key in out:
            if key == "info":
                continue
            ref = g["r%d_%s" % (r, key)]
            d = float(np.abs(out[key] - ref).max())
            assert d <= 1e-12, (tag, r, key, d)


@pytest.mark.parametrize("tag", CASES)
def test_topology_matches_reference_ranks(tag):
    g = _golden(tag)
    nr = int(g["nranks"])
    res = run_ranks("test_host_ranks", "topo_rank", nr, (tag,))
    for r, out in enumerate(res):
        assert int(out["rank"]) == r and int(out["nranks"]) == nr
        assert tuple(out["coords"]) == tuple(g["r%d_coords" % r])
        assert tuple(out["local"]) == tuple(g["r%d_local" % r])
        nb = g["r%d_neighbors" % r]
        np.testing.assert_array_equal(out["neighbors"], np.where(nb < 0, -1, nb))
        assert float(out["ar"]) == nr - 1
