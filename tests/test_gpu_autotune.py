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
    assert back["20"]["best"] == table[20]["best"]


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
