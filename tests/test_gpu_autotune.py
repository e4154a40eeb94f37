"""The relax autotuner times each strategy and installs the fastest; the
installed strategy does not change results beyond FP64 rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_small_sizes(tmp_path):
    from warpflow import autotune
    table = autotune.tune(sizes=(8, 20), sweeps=60)
    assert set(table) == {8, 20}
    for n, rec in table.items():
        assert rec["best"] in (0, 1, 2, 3, 4)
        assert min(rec["us"].values()) == rec["us"][str(rec["best"])]
    p = tmp_path / "tune.json"
    autotune.save(table, p)
    back = autotune.load_and_apply(p)
    assert back["coarse"]["20"]["best"] == table[20]["best"]


def test_tune_buckets_installs_faster_form(tmp_path):
    """The ensemble tuner times a bucket against a branch per case, keeps
    the faster one per size, and its cache re-installs the same caps."""
    from warpflow import autotune
    try:
        table = autotune.tune_buckets(sizes=(16, 24), ncases=3, reps=2)
        assert set(table) == {16, 24}
        for n, rec in table.items():
            t = rec["ms"]
            assert rec["cap"] == (3 if t["bucket"] < t["branches"] else 1)
            assert autotune.bucket_cap(n) == rec["cap"]
        p = tmp_path / "tune.json"
        autotune.save({}, p, buckets=table)
        for n in table:
            autotune.set_bucket_cap(n, 0)
        autotune.load_and_apply(p)
        assert all(autotune.bucket_cap(n) == rec["cap"] for n, rec in table.items())
    finally:
        for n in (16, 24):
            autotune.set_bucket_cap(n, 0)


def test_tune_shapes_and_bit_identical_step():
    """The shape tuner times k_conv and k_rbgs_split shapes at 80^3 (each
    checked bit-identical to the default), installs the fastest, and a
    solver built with non-default shapes (several planes per thread) steps
    exactly like one built with the defaults, alone and in a bucket."""
    from warpflow import FlowSolver, autotune, build_topology
    from warpflow.ensemble import cavity_case
    try:
        table = autotune.tune_shapes(sizes=(80,), conv=((32, 8, 1), (16, 16, 3), (64, 4, 8)),
                                     split=((2, 8, 1), (1, 4, 1), (4, 2, 1)), reps=3)
        for kind in ("conv", "split"):
            rec = table[kind][80]
            assert tuple(autotune.shape(kind, 80)) == tuple(rec["best"])
            assert min(rec["us"].values()) == rec["us"]["%dx%dx%d" % tuple(rec["best"])]
        cfg = cavity_case(80, precision="fp64")
        autotune.set_shape("conv", 80, 16, 16, 3)
        autotune.set_shape("split", 80, 4, 2)
        a = FlowSolver(cfg, build_topology(cfg), "cuda:0")
        autotune.set_shape("conv", 80, 0, 0, 0)
        autotune.set_shape("split", 80, 0, 0, 0)
        b = FlowSolver(cfg, build_topology(cfg), "cuda:0")
        for _ in range(2):
            assert a.step() == b.step()
        for name in ("u", "v", "w", "p", "pp", "ustar"):
            np.testing.assert_array_equal(a.f[name].numpy(), b.f[name].numpy(), err_msg=name)
        a.close()
        b.close()
    finally:
        autotune.set_shape("conv", 80, 0, 0, 0)
        autotune.set_shape("split", 80, 0, 0, 0)


def test_conv_planes_in_a_bucket():
    """Several planes per thread in a bucket launch (grid z = cases x plane
    groups, the last group short): each case as alone."""
    from warpflow import FlowSolver, autotune, build_topology
    from warpflow.ensemble import Ensemble, cavity_case
    cfgs = [cavity_case(24, re, 1.0, precision="fp64") for re in (200.0, 700.0)]
    try:
        autotune.set_shape("conv", 24, 32, 4, 5)
        ens = Ensemble(cfgs, nstreams=1)
        assert ens.layout()[0] == [0, 0]
        autotune.set_shape("conv", 24, 0, 0, 0)
        alone = [FlowSolver(c, build_topology(c), "cuda:0") for c in cfgs]
        for _ in range(2):
            assert ens.step() == [s.step() for s in alone]
        for sol, ref in zip(ens.solvers, alone):
            for name in ("u", "v", "w", "p"):
                np.testing.assert_array_equal(sol.f[name].numpy(), ref.f[name].numpy())
        ens.close()
    finally:
        autotune.set_shape("conv", 24, 0, 0, 0)


@pytest.mark.parametrize("n", [8, 12, 16, 20, 24])
@pytest.mark.parametrize("sweeps", [40, 41, 300])
def test_strategies_agree(n, sweeps):
    """All three coarse implementations give the same relax result."""
    from helpers import make_cfg
    from warpflow import Multigrid, autotune, build_topology
    cfg = make_cfg(n=n, levels=1)
    mg = Multigrid(cfg, build_topology(cfg), "cuda:0", 1 / n, 1 / n, 1 / n)
    lev = mg.levels[0]
    rhs = np.random.default_rng(1).standard_normal(lev.shape)
    outs = []
    for s in (0, 1, 2, 3, 4):
        if s == 4 and n == 8:
            continue
        autotune.set_strategy(n, s)
        lev.rhs.assign(rhs)
        lev.phi.zero_()
        mg._relax(0, sweeps)
        outs.append(lev.phi.numpy())
    autotune.set_strategy(n, 0 if n <= 16 else (2 if n == 20 else 4))
    for o in outs[1:]:
        assert np.abs(o - outs[0]).max() <= 1e-12 * np.abs(outs[0]).max()
