"""Per-kernel parity of libwfb200 against the CPU oracle on seeded random
inputs (GPU).  Byte-moving kernels (fills, copies, init noise) must match
bit for bit; FP64 arithmetic kernels within 1e-13 relative (FMA
contraction and division rounding are the only differences)."""
import ctypes

import numpy as np
import pytest
import torch

from helpers import make_cfg
from oracle import wf_oracle as O

pytestmark = pytest.mark.gpu


def _solver(n=16, levels=3, **kw):
    from warpflow import FlowSolver, build_topology
    cfg = make_cfg(n=n, levels=levels, **kw)
    return FlowSolver(cfg, build_topology(cfg), "cuda:0")


def _rand(shape, seed):
    return np.random.default_rng(seed).standard_normal(shape)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _call(name, *args):
    from warpflow import _abi
    _abi.call(name, *args)
    torch.cuda.synchronize()


def _close(a, b, rel=1e-13):
    scale = max(1.0, float(np.abs(b).max()))
    d = float(np.abs(a - b).max())
    assert d <= rel * scale, d


@pytest.mark.parametrize("kind", ["u", "v", "w", "vis", "pbound", "p_mirror"])
def test_fills_bit_exact(kind):
    sol = _solver(n=12)
    n = 12
    shp = sol.f["u"].shape
    a = _rand(shp, 1)
    fld = sol.f["u"]
    fld.assign(a)
    ref = a.copy()
    s = _stream()
    if kind == "u":
        _call("wf_fill_u", fld.ptr, n, 0.75, s)
        O.apply_u(ref, n, 0.75)
    elif kind == "v":
        _call("wf_fill_v", fld.ptr, n, s)
        O.apply_v(ref, n)
    elif kind == "w":
        _call("wf_fill_w", fld.ptr, n, s)
        O.apply_w(ref, n)
    elif kind == "vis":
        _call("wf_fill_vis", fld.ptr, n, 0.0025, s)
        O.apply_vis(ref, n, 0.0025)
    elif kind == "pbound":
        _call("wf_fill_pbound", fld.ptr, n, s)
        O.apply_pbound(ref, n)
    else:
        _call("wf_fill_p_mirror", fld.ptr, n, s)
        O.apply_p_mirror(ref, n)
    np.testing.assert_array_equal(fld.numpy(), ref)


def test_init_noise_bit_exact():
    n = 16
    sol = _solver(n=n, noise=0.0)
    for k in ("u", "v", "w"):
        sol.f[k].zero_()
    _call("wf_init_noise", sol.f["u"].ptr, sol.f["v"].ptr, sol.f["w"].ptr, n, 0.01, 1,
          _stream())
    u = np.zeros(sol.f["u"].shape)
    v = np.zeros_like(u)
    w = np.zeros_like(u)
    O.init_noise(u, v, w, 0.01, 1, n)
    np.testing.assert_array_equal(sol.f["u"].numpy(), u)
    np.testing.assert_array_equal(sol.f["v"].numpy(), v)
    np.testing.assert_array_equal(sol.f["w"].numpy(), w)


def _randomise(sol, names, seed, scale=1.0):
    out = {}
    for i, k in enumerate(names):
        a = scale * _rand(sol.f[k].shape, seed + i)
        sol.f[k].assign(a)
        out[k] = a
    return out


@pytest.mark.parametrize("comp", [0, 1, 2])
@pytest.mark.parametrize("alpha", [0.5, 1.0])
@pytest.mark.parametrize("n", [16, 40, 72])   # whole and partial 32-cell runs along k
def test_conv_diff(comp, alpha, n):
    sol = _solver(n=n)
    sol.dt = 3.3e-4
    f = _randomise(sol, ["u", "v", "w", "uoo", "voo", "woo", "vis", "ustar", "vstar",
                         "wstar"], 10)
    c = "uvw"[comp]
    star = c + "star"
    dtp = sol._sc.data_ptr()  # wf_scalars.dt is the first member
    _call("wf_conv", ctypes.byref(sol.case), comp, alpha, dtp, _stream())
    O.conv4th(c, f["u"], f["v"], f["w"], f[c + "oo"], f[star], sol.dx, sol.dy, sol.dz,
              3.3e-4, alpha, n)
    _close(sol.f[star].numpy(), f[star])
    _call("wf_diff", ctypes.byref(sol.case), comp, alpha, dtp, _stream())
    O.diff4th(c, f[c], f["vis"], f[star], sol.dx, sol.dy, sol.dz, 3.3e-4, alpha, n)
    _close(sol.f[star].numpy(), f[star])


def test_calvel_calmas():
    n = 16
    sol = _solver(n=n)
    sol.dt = 2.5e-4
    f = _randomise(sol, ["ustar", "vstar", "wstar", "p", "u", "v", "w", "su"], 20)
    _call("wf_calvel", ctypes.byref(sol.case), 0.5, sol._sc.data_ptr(), _stream())
    for comp, d in (("u", sol.dx), ("v", sol.dy), ("w", sol.dz)):
        O.calvel(comp, f[comp + "star"], f["p"], f[comp], d, 2.5e-4, 0.5, n)
    for k in ("u", "v", "w"):
        _close(sol.f[k].numpy(), f[k])
    _call("wf_calmas", ctypes.byref(sol.case), _stream())
    rmax = O.calmas(f["u"], f["v"], f["w"], f["su"], sol.dx, sol.dy, sol.dz, 2.5e-4, n)
    _close(sol.f["su"].numpy(), f["su"])
    sc = sol._pull_scalars()
    assert sc.rmax == pytest.approx(rmax, rel=1e-13)
    assert sc.iters == 1


def test_wale_and_checkdt():
    n = 16
    sol = _solver(n=n)
    f = _randomise(sol, ["u", "v", "w"], 30, scale=0.1)
    vis = np.full(sol.f["vis"].shape, sol.rey)
    sol.f["vis"].assign(vis)
    _call("wf_wale_vis", ctypes.byref(sol.case), _stream())
    O.wale(f["u"], f["v"], f["w"], vis, sol.dx, sol.dy, sol.dz, sol.rey, 0.46, n)
    O.apply_vis(vis, n, sol.rey)
    _close(sol.f["vis"].numpy(), vis, rel=1e-12)
    sol.dt = 3.0e-4
    _call("wf_checkdt", ctypes.byref(sol.case), _stream())
    sc = sol._pull_scalars()
    assert sc.umax == O.maxabs(f["u"], n)
    assert sc.vmax == O.maxabs(f["v"], n)
    assert sc.wmax == O.maxabs(f["w"], n)
    dtv = O.dtvisc(f["u"], f["v"], f["w"], sol.f["vis"].numpy(), sol.dx, sol.dy, sol.dz, n)
    assert sc.dtvisc == pytest.approx(dtv, rel=1e-14)
    dtcfl = min(sol.dx / sc.umax, sol.dy / sc.vmax, sol.dz / sc.wmax)
    dtmax = min(dtv, dtcfl)
    assert sc.cfl == pytest.approx(3.0e-4 / dtmax, rel=1e-13)
    assert sc.dt == pytest.approx(min(3.0e-4 * 1.1, 0.8 * dtmax), rel=1e-13)
    assert sc.itime == 1


def test_add_ring():
    n = 12
    sol = _solver(n=n)
    f = _randomise(sol, ["p", "pp"], 40)
    _call("wf_add_ring", sol.f["p"].ptr, sol.f["pp"].ptr, n, _stream())
    O.add_ring(f["p"], f["pp"], n)
    np.testing.assert_array_equal(sol.f["p"].numpy(), f["p"])


def test_mg_harness_matches_golden():
    """Two V-cycles of the standalone harness (tests/test_mg.py) against the
    golden vectors of the reference run: level 0, 1, 2 phi incl. rings."""
    from helpers import golden
    from warpflow import Multigrid, build_topology
    g = golden("mg16_l3")
    cfg = make_cfg(n=16, levels=3)
    mg = Multigrid(cfg, build_topology(cfg), "cuda:0", 1 / 16, 1 / 16, 1 / 16)
    lev0 = mg.levels[0]
    lev0.rhs.assign(g["rhs"])
    lev0.phi.zero_()
    mg._refill(lev0)
    for c in range(2):
        mg._vcycle()
        for l, key in ((0, "phi_c%d"), (1, "phi1_c%d"), (2, "phi2_c%d")):
            ref = g[key % c]
            got = mg.levels[l].phi.numpy()
            assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), (c, l)
    r = mg.residual_max(0)
    ref = float(np.abs(O.Level(16, 1 / 16, 1 / 16, 1 / 16).residual(
        g["phi_c1"], g["rhs"])).max())
    assert r == pytest.approx(ref, rel=1e-9)


@pytest.mark.parametrize("n,levels", [(16, 3), (32, 3), (48, 3), (32, 5)])
def test_mg_solve_matches_oracle(n, levels):
    from warpflow import Multigrid, build_topology
    cfg = make_cfg(n=n, levels=levels)
    h = 1.0 / n
    mg = Multigrid(cfg, build_topology(cfg), "cuda:0", h, h, h)
    sol_shape = (n + 6,) * 3
    from warpflow.fields import DeviceField
    su = DeviceField.zeros(sol_shape, "cuda:0")
    pp = DeviceField.zeros(sol_shape, "cuda:0")
    rhs = _rand(sol_shape, 50)
    su.assign(rhs)
    pp.assign(_rand(sol_shape, 51))  # solve must zero it first
    mg.solve(su, pp, 3)
    omg = O.Multigrid(n, levels, h, h, h)
    ref = np.zeros(sol_shape)
    omg.solve(rhs, ref, n)
    got = pp.numpy()
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()
