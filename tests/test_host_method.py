"""Host-side checks of two reformulations the device step relies on, made on
the oracle (CPU, no GPU):

* the coarsest-level relax through the half operator: n_coarse red-black
  sweeps from phi = 0 equal the first sweep's even-parity numerators, a
  fixed (N/2) x (N/2) map on them (n_coarse - 1 sweeps of the even half),
  and one closing sweep;
* that map is symmetric and commutes with the level's colour-preserving
  symmetries, so its columns at one representative cell per orbit give the
  whole product (the device's stored form of it);
* the diffusion of each velocity component computed right after its
  convection (before the fills of the other components and its own second
  fill) gives the reference's step bit for bit.
"""
import itertools

import numpy as np
import pytest

from helpers import make_cfg
from oracle import wf_oracle as O


def _sweeps(lev, rhs, nsweeps):
    s = lev.s
    lev.phi[...] = 0.0
    lev.rhs[...] = 0.0
    lev.rhs[s, s, s] = rhs
    for _ in range(nsweeps):
        O.rbgs(lev, 0)
        O.rbgs(lev, 1)
    return lev.phi[s, s, s].copy()


def _half_operator(n, n_coarse, hx, hy, hz):
    """S[b] = the even-parity (B) half after n_coarse - 1 sweeps from zero with
    rhs = unit at the b-th B cell (the device builds these rows)."""
    lev = O.Level(n, hx, hy, hz)
    idx = np.arange(n)
    par = (idx[:, None, None] + idx[None, :, None] + idx[None, None, :]) % 2
    even = par == 0
    bcells = np.argwhere(even)
    S = np.zeros((len(bcells), len(bcells)))
    for b, (i, j, k) in enumerate(bcells):
        e = np.zeros((n,) * 3)
        e[i, j, k] = 1.0
        S[b] = _sweeps(lev, e, n_coarse - 1)[even]
    return S, bcells


def _symmetries(n, coef):
    """Axis permutations between axes of equal coefficient, each with the
    reflections of an even number of axes: c'_d = sgn * c[src] + off."""
    out = []
    for pm in itertools.permutations(range(3)):
        if any(coef[pm[d]] != coef[d] for d in range(3)):
            continue
        for mk in (0, 3, 5, 6):
            out.append([(pm[d], -1 if (mk >> d) & 1 else 1, n - 1 if (mk >> d) & 1 else 0)
                        for d in range(3)])
    return out


@pytest.mark.parametrize("h", [(0.3, 0.3, 0.3), (0.3, 0.3, 0.5), (0.2, 0.3, 0.5)])
def test_symmetric_operator_reproduces_the_half_operator(h):
    n, n_coarse = 8, 25
    S, bcells = _half_operator(n, n_coarse, *h)
    assert np.abs(S - S.T).max() <= 1e-12 * np.abs(S).max()
    coef = tuple(1.0 / (x * x) for x in h)
    G = _symmetries(n, coef)
    assert len(G) == {1: 24, 2: 8, 3: 4}[len(set(coef))]
    pos = {tuple(c): b for b, c in enumerate(bcells)}

    def image(g, b):
        c = bcells[b]
        return pos[tuple(sg * c[src] + off for src, sg, off in g)]

    M = len(bcells)
    img = np.array([[image(g, b) for b in range(M)] for g in G])   # img[g, u] = g(u)
    for g in range(len(G)):   # S[g u, g w] = S[u, w]
        np.testing.assert_allclose(S[np.ix_(img[g], img[g])], S, rtol=0, atol=1e-12 * np.abs(S).max())
    reps = sorted({int(img[:, b].min()) for b in range(M)})
    v = np.random.default_rng(5).standard_normal(M)
    x = np.full(M, np.nan)
    for r in reps:
        for g in range(len(G)):
            o = img[g, r]
            if np.isnan(x[o]):
                x[o] = S[r] @ v[img[g]]      # sum_u S[u, r] v[g u], S[u, r] = row r
    assert not np.isnan(x).any()
    ref = v @ S
    assert np.abs(x - ref).max() <= 1e-12 * np.abs(ref).max()
    assert len(reps) <= M // len(G) + n * n


def test_half_operator_equals_the_sweeps():
    n, n_coarse = 4, 25
    h = 0.3
    lev = O.Level(n, h, h, h)
    idx = np.arange(n)
    par = (idx[:, None, None] + idx[None, :, None] + idx[None, None, :]) % 2
    even = par == 0                     # colour B: updated second
    bcells = np.argwhere(even)          # (i, j, k) order = position b
    M = len(bcells)
    S = np.zeros((M, M))
    for b, (i, j, k) in enumerate(bcells):
        e = np.zeros((n,) * 3)
        e[i, j, k] = 1.0
        S[b] = _sweeps(lev, e, n_coarse - 1)[even]
    rhs = np.random.default_rng(4).standard_normal((n,) * 3)
    direct = _sweeps(lev, rhs, n_coarse)
    # first sweep from zero: x_A = rhs / ap on the odd cells, then the even
    # cells' numerators v_B = rhs - sum of neighbour terms
    s = lev.s
    lev.phi[...] = 0.0
    lev.phi[s, s, s][~even] = (rhs / lev.ap)[~even]
    v = (rhs - lev.nbsum(lev.phi))[even]
    xb = v @ S
    lev.phi[...] = 0.0
    lev.phi[s, s, s][even] = xb
    lev.rhs[s, s, s] = rhs
    O.rbgs(lev, 0)
    O.rbgs(lev, 1)
    via = lev.phi[s, s, s]
    assert np.abs(via - direct).max() <= 1e-12 * np.abs(direct).max()


class _FusedOrder(O.OracleSolver):
    """The device step's order: each component's diffusion right after its
    convection, the reference's fills kept."""

    def step(self):
        self.itime += 1
        self.compute_dt()
        self.ctime += self.dt
        f, n = self.f, self.n
        f["uoo"][...] = f["u"]
        f["voo"][...] = f["v"]
        f["woo"][...] = f["w"]
        O.wale(f["u"], f["v"], f["w"], f["vis"], self.dx, self.dy, self.dz,
               self.rey, self.cfg.physics.sgs_cw, n)
        O.apply_vis(f["vis"], n, self.rey)
        dt, d3 = self.dt, (self.dx, self.dy, self.dz)
        comps = (("u", "ustar", "uoo"), ("v", "vstar", "voo"), ("w", "wstar", "woo"))
        for stage, alpha in enumerate(O.ALFARK):
            for comp, star, oo in comps:
                self.fill_bc(comp)
                O.conv4th(comp, f["u"], f["v"], f["w"], f[oo], f[star], *d3, dt, alpha, n)
                O.diff4th(comp, f[comp], f["vis"], f[star], *d3, dt, alpha, n)
            for comp, _, _ in comps:
                self.fill_bc(comp)
            if stage + 1 < len(O.ALFARK):
                self._calvel(alpha)
        self._project()
        return {"ctime": self.ctime, "dt": self.dt, "rmax": self.rmax,
                "iters": self.outer_iters, "cfl": self.cfl}


def test_diffusion_inside_convection_is_bit_identical():
    cfg = make_cfg(8, levels=2)
    ref, fused = O.OracleSolver(cfg), _FusedOrder(cfg)
    for _ in range(4):
        assert ref.step() == fused.step()
    for name in ref.f:
        np.testing.assert_array_equal(ref.f[name], fused.f[name], err_msg=name)
