"""CPU oracle: a vectorised NumPy FP64 restatement of the warpflow-les
per-step hot path (reference v0.1.0).

TEST INFRASTRUCTURE ONLY.  It is imported by ``tests/``, by
``__graft_entry__.smoke()`` as the checker, and by ``bench.py`` for the
``cpu_baseline`` leg and the ``--impl reference`` arm.  The product path
(``warpflow`` + ``libwfb200.so``) never imports it and has no CPU fallback.

Parity pin: this restatement is checked against golden vectors produced by
running the reference's own source (warpflow/{kernels,bcs,multigrid,
solver}.py) through a CPU stand-in for NVIDIA Warp
(``tests/golden/make_golden.py``).  Each function cites the reference
file:line it follows.

Layout: every field is a C-ordered float64 array of shape (n+6)^3 indexed
[i][j][k] with k contiguous; real cells are NPL..NPL+n-1 (kernels.py:9-12).
Multigrid levels are (n_l+2)^3 with one ring layer (multigrid.py:207-220).
"""
from __future__ import annotations

import math

import numpy as np

NPL = 3                      # topology.py:15
ALFARK = (0.5, 1.0)          # solver.py:26
N_PRE, N_POST, N_COARSE, N_VCYCLES = 6, 6, 300, 4   # multigrid.py:257-260


# --------------------------------------------------------------------------
# ghost fills (bcs.py)
# --------------------------------------------------------------------------
def _sl(axis, idx, a0, na, b0, nb):
    """Index tuple for plane `idx` of `axis`, perpendicular box [a0,a0+na) x
    [b0,b0+nb) in the order of the two remaining axes (bcs.py:42-106)."""
    s = [None, None, None]
    s[axis] = idx
    other = [d for d in range(3) if d != axis]
    s[other[0]] = slice(a0, a0 + na)
    s[other[1]] = slice(b0, b0 + nb)
    return tuple(s)


def fill_lin(fld, axis, high, g0, s0, sign, a0, na, b0, nb, nlay):
    """bcs.py:42-106 ``_mk_lin``: fld[ghost(m)] = sign*fld[src(m)], layers
    m = 0..nlay-1 in order (low: g0-m <- s0+m, high: g0+m <- s0-m)."""
    for m in range(nlay):
        g = g0 + m if high else g0 - m
        s = s0 - m if high else s0 + m
        fld[_sl(axis, g, a0, na, b0, nb)] = sign * fld[_sl(axis, s, a0, na, b0, nb)]


def fill_const(fld, axis, high, g0, val, a0, na, b0, nb, nlay):
    """bcs.py:109-163 ``_mk_const``: fld[ghost(m)] = val."""
    for m in range(nlay):
        g = g0 + m if high else g0 - m
        fld[_sl(axis, g, a0, na, b0, nb)] = val


def apply_u(u, n, ulid):
    """bcs.py:201-223 (order W, E, S, N, B, T)."""
    P = NPL
    fill_const(u, 0, False, P - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3)
    fill_const(u, 0, True, P + n - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3)
    fill_lin(u, 1, False, P - 1, P, 1.0, P - 1, n + 1, P - 1, n + 2, 3)
    fill_lin(u, 1, True, P + n, P + n - 1, 1.0, P - 1, n + 1, P - 1, n + 2, 3)
    fill_lin(u, 2, False, P - 1, P, -1.0, P - 1, n + 1, P - 1, n + 2, 3)
    fill_const(u, 2, True, P + n, ulid, P - 1, n + 1, P - 1, n + 2, 3)


def apply_v(v, n):
    """bcs.py:225-244."""
    P = NPL
    fill_lin(v, 0, False, P - 1, P, -1.0, P - 1, n + 1, P - 1, n + 2, 3)
    fill_lin(v, 0, True, P + n, P + n - 1, -1.0, P - 1, n + 1, P - 1, n + 2, 3)
    fill_const(v, 1, False, P - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3)
    fill_const(v, 1, True, P + n - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3)
    fill_lin(v, 2, False, P - 1, P, -1.0, P - 1, n + 2, P - 1, n + 1, 3)
    fill_lin(v, 2, True, P + n, P + n - 1, 1.0, P - 1, n + 2, P - 1, n + 1, 3)


def apply_w(w, n):
    """bcs.py:246-265."""
    P = NPL
    fill_lin(w, 0, False, P - 1, P, -1.0, P - 1, n + 2, P - 1, n + 1, 3)
    fill_lin(w, 0, True, P + n, P + n - 1, -1.0, P - 1, n + 2, P - 1, n + 1, 3)
    fill_lin(w, 1, False, P - 1, P, 1.0, P - 1, n + 2, P - 1, n + 1, 3)
    fill_lin(w, 1, True, P + n, P + n - 1, 1.0, P - 1, n + 2, P - 1, n + 1, 3)
    fill_const(w, 2, False, P - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3)
    fill_const(w, 2, True, P + n - 1, 0.0, P - 1, n + 2, P - 1, n + 2, 3)


def apply_vis(vis, n, rrey):
    """bcs.py:267-293: wall planes forced to 1/Re, then one mirrored layer."""
    P = NPL
    fill_const(vis, 0, False, P, rrey, P - 1, n + 2, P - 1, n + 2, 1)
    fill_lin(vis, 0, False, P - 1, P, 1.0, P - 1, n + 2, P - 1, n + 2, 1)
    fill_const(vis, 0, True, P + n - 1, rrey, P - 1, n + 2, P - 1, n + 2, 1)
    fill_lin(vis, 0, True, P + n, P + n - 1, 1.0, P - 1, n + 2, P - 1, n + 2, 1)
    fill_lin(vis, 1, False, P - 1, P, 1.0, P - 1, n + 2, P - 1, n + 2, 1)
    fill_lin(vis, 1, True, P + n, P + n - 1, 1.0, P - 1, n + 2, P - 1, n + 2, 1)
    fill_const(vis, 2, False, P, rrey, P - 1, n + 2, P - 1, n + 2, 1)
    fill_lin(vis, 2, False, P - 1, P, 1.0, P - 1, n + 2, P - 1, n + 2, 1)
    fill_lin(vis, 2, True, P + n, P + n - 1, 1.0, P - 1, n + 2, P - 1, n + 2, 1)


def apply_pbound(p, n):
    """bcs.py:295-302: one Neumann layer, perpendicular range [NPL-1, NPL+n+1]."""
    P = NPL
    for axis in (0, 1, 2):
        fill_lin(p, axis, False, P - 1, P, 1.0, P - 1, n + 3, P - 1, n + 3, 1)
        fill_lin(p, axis, True, P + n, P + n - 1, 1.0, P - 1, n + 3, P - 1, n + 3, 1)


def apply_p_mirror(p, n, npl=NPL):
    """bcs.py:304-311: full-depth Neumann mirror on every side."""
    P = NPL
    for axis, high in ((0, False), (0, True), (1, False), (1, True),
                       (2, False), (2, True)):
        g0, s0 = (P - 1, P) if not high else (P + n, P + n - 1)
        fill_lin(p, axis, high, g0, s0, 1.0, 0, n + 2 * P, 0, n + 2 * P, npl)


def apply_initial(f, n, ulid):
    """bcs.py:313-323."""
    apply_u(f["u"], n, ulid)
    apply_v(f["v"], n)
    apply_w(f["w"], n)
    apply_p_mirror(f["p"], n)


ALL_PHYS = (True,) * 6


def mg_refill(phi, n, phys=ALL_PHYS):
    """bcs.py:326-360 ``_mk_neumann`` with npl=1 on the physical faces
    (multigrid.py:264-287; face interiors only, edges and corners
    untouched).  ``phys``: west, east, south, north, bottom, top."""
    s = slice(1, n + 1)
    if phys[0]:
        phi[0, s, s] = phi[1, s, s]
    if phys[1]:
        phi[n + 1, s, s] = phi[n, s, s]
    if phys[2]:
        phi[s, 0, s] = phi[s, 1, s]
    if phys[3]:
        phi[s, n + 1, s] = phi[s, n, s]
    if phys[4]:
        phi[s, s, 0] = phi[s, s, 1]
    if phys[5]:
        phi[s, s, n + 1] = phi[s, s, n]


# --------------------------------------------------------------------------
# stencil kernels (kernels.py)
# --------------------------------------------------------------------------
class _V:
    """Shifted views of a padded field over the op range: ``V(f)(di,dj,dk)``
    is f[i+di, j+dj, k+dk] for all (i, j, k) of the range."""

    def __init__(self, f, lo, dims):
        self.f, self.lo, self.dims = f, lo, dims

    def __call__(self, di, dj, dk):
        i0, j0, k0 = self.lo
        a, b, c = self.dims
        return self.f[i0 + di:i0 + di + a, j0 + dj:j0 + dj + b,
                      k0 + dk:k0 + dk + c]


def _I(F, axis, d):
    """kernels.py:31-46 ``_ix/_iy/_iz`` at offset d (a 3-tuple) along axis."""
    def at(m):
        o = list(d)
        o[axis] += m
        return F(*o)
    return (-at(1) + 9.0 * at(0) + 9.0 * at(-1) - at(-2)) / 16.0


def _op_dims(n, comp):
    """solver.py:99-110."""
    if comp == "u":
        return (n - 1, n, n)
    if comp == "v":
        return (n, n - 1, n)
    if comp == "w":
        return (n, n, n - 1)
    return (n, n, n)


def _interior(f, dims):
    a, b, c = dims
    return f[NPL:NPL + a, NPL:NPL + b, NPL:NPL + c]


def conv4th(comp, u, v, w, oo, star, dx, dy, dz, dt, alpha, n):
    """kernels.py:53-168 (conv4th_u / conv4th_v / conv4th_w)."""
    dims = _op_dims(n, comp)
    lo = (NPL, NPL, NPL)
    U, Vv, W = _V(u, lo, dims), _V(v, lo, dims), _V(w, lo, dims)

    def sq(F, ax, off):
        x = _I(F, ax, off)
        return x * x

    if comp == "u":
        sp2 = sq(U, 0, (2, 0, 0)); sp1 = sq(U, 0, (1, 0, 0))
        sn = sq(U, 0, (0, 0, 0)); sm1 = sq(U, 0, (-1, 0, 0))
        d1 = (-sp2 + 27.0 * sp1 - 27.0 * sn + sm1) / (24.0 * dx)
        sp1 = _I(U, 1, (0, 2, 0)) * _I(Vv, 0, (1, 1, 0))
        sn = _I(U, 1, (0, 1, 0)) * _I(Vv, 0, (1, 0, 0))
        sm1 = _I(U, 1, (0, 0, 0)) * _I(Vv, 0, (1, -1, 0))
        sm2 = _I(U, 1, (0, -1, 0)) * _I(Vv, 0, (1, -2, 0))
        d2 = (-sp1 + 27.0 * sn - 27.0 * sm1 + sm2) / (24.0 * dy)
        sp1 = _I(U, 2, (0, 0, 2)) * _I(W, 0, (1, 0, 1))
        sn = _I(U, 2, (0, 0, 1)) * _I(W, 0, (1, 0, 0))
        sm1 = _I(U, 2, (0, 0, 0)) * _I(W, 0, (1, 0, -1))
        sm2 = _I(U, 2, (0, 0, -1)) * _I(W, 0, (1, 0, -2))
        d3 = (-sp1 + 27.0 * sn - 27.0 * sm1 + sm2) / (24.0 * dz)
        tot = d1 + d2 + d3
    elif comp == "v":
        sp2 = sq(Vv, 1, (0, 2, 0)); sp1 = sq(Vv, 1, (0, 1, 0))
        sn = sq(Vv, 1, (0, 0, 0)); sm1 = sq(Vv, 1, (0, -1, 0))
        dv2dy = (-sp2 + 27.0 * sp1 - 27.0 * sn + sm1) / (24.0 * dy)
        sp1 = _I(Vv, 0, (2, 0, 0)) * _I(U, 1, (1, 1, 0))
        sn = _I(Vv, 0, (1, 0, 0)) * _I(U, 1, (0, 1, 0))
        sm1 = _I(Vv, 0, (0, 0, 0)) * _I(U, 1, (-1, 1, 0))
        sm2 = _I(Vv, 0, (-1, 0, 0)) * _I(U, 1, (-2, 1, 0))
        duvdx = (-sp1 + 27.0 * sn - 27.0 * sm1 + sm2) / (24.0 * dx)
        sp1 = _I(Vv, 2, (0, 0, 2)) * _I(W, 1, (0, 1, 1))
        sn = _I(Vv, 2, (0, 0, 1)) * _I(W, 1, (0, 1, 0))
        sm1 = _I(Vv, 2, (0, 0, 0)) * _I(W, 1, (0, 1, -1))
        sm2 = _I(Vv, 2, (0, 0, -1)) * _I(W, 1, (0, 1, -2))
        dvwdz = (-sp1 + 27.0 * sn - 27.0 * sm1 + sm2) / (24.0 * dz)
        tot = duvdx + dv2dy + dvwdz
    else:
        sp2 = sq(W, 2, (0, 0, 2)); sp1 = sq(W, 2, (0, 0, 1))
        sn = sq(W, 2, (0, 0, 0)); sm1 = sq(W, 2, (0, 0, -1))
        dw2dz = (-sp2 + 27.0 * sp1 - 27.0 * sn + sm1) / (24.0 * dz)
        sp1 = _I(W, 0, (2, 0, 0)) * _I(U, 2, (1, 0, 1))
        sn = _I(W, 0, (1, 0, 0)) * _I(U, 2, (0, 0, 1))
        sm1 = _I(W, 0, (0, 0, 0)) * _I(U, 2, (-1, 0, 1))
        sm2 = _I(W, 0, (-1, 0, 0)) * _I(U, 2, (-2, 0, 1))
        duwdx = (-sp1 + 27.0 * sn - 27.0 * sm1 + sm2) / (24.0 * dx)
        sp1 = _I(W, 1, (0, 2, 0)) * _I(Vv, 2, (0, 1, 1))
        sn = _I(W, 1, (0, 1, 0)) * _I(Vv, 2, (0, 0, 1))
        sm1 = _I(W, 1, (0, 0, 0)) * _I(Vv, 2, (0, -1, 1))
        sm2 = _I(W, 1, (0, -1, 0)) * _I(Vv, 2, (0, -2, 1))
        dvwdy = (-sp1 + 27.0 * sn - 27.0 * sm1 + sm2) / (24.0 * dy)
        tot = duwdx + dvwdy + dw2dz
    _interior(star, dims)[...] = _interior(oo, dims) - dt * alpha * tot


def lap4(F, dx, dy, dz):
    """kernels.py:177-186."""
    c = F(0, 0, 0)
    lx = (-F(2, 0, 0) + 16.0 * F(1, 0, 0) - 30.0 * c + 16.0 * F(-1, 0, 0)
          - F(-2, 0, 0)) / (12.0 * dx * dx)
    ly = (-F(0, 2, 0) + 16.0 * F(0, 1, 0) - 30.0 * c + 16.0 * F(0, -1, 0)
          - F(0, -2, 0)) / (12.0 * dy * dy)
    lz = (-F(0, 0, 2) + 16.0 * F(0, 0, 1) - 30.0 * c + 16.0 * F(0, 0, -1)
          - F(0, 0, -2)) / (12.0 * dz * dz)
    return lx + ly + lz


def diff4th(comp, c, vis, star, dx, dy, dz, dt, alpha, n):
    """kernels.py:189-225; vis sampled at (i,j,k) / (i,j+1,k) / (i,j,k+1)."""
    dims = _op_dims(n, comp)
    lo = (NPL, NPL, NPL)
    C = _V(c, lo, dims)
    VI = _V(vis, lo, dims)
    vs = {"u": VI(0, 0, 0), "v": VI(0, 1, 0), "w": VI(0, 0, 1)}[comp]
    diff = vs * lap4(C, dx, dy, dz)
    st = _interior(star, dims)
    st[...] = st + dt * alpha * diff


def calvel(comp, star, p, c, d, dt, alpha, n):
    """kernels.py:232-264."""
    dims = _op_dims(n, comp)
    lo = (NPL, NPL, NPL)
    Pp = _V(p, lo, dims)
    sh = {"u": (1, 0, 0), "v": (0, 1, 0), "w": (0, 0, 1)}[comp]
    _interior(c, dims)[...] = (_interior(star, dims)
                               - dt * alpha * (Pp(*sh) - Pp(0, 0, 0)) / d)


def calmas(u, v, w, su, dx, dy, dz, dt, n):
    """kernels.py:271-289; returns rmax = max|div*dx*dy*dz|."""
    dims = (n, n, n)
    lo = (NPL, NPL, NPL)
    U, Vv, W = _V(u, lo, dims), _V(v, lo, dims), _V(w, lo, dims)
    dudx = (-U(1, 0, 0) + 27.0 * U(0, 0, 0) - 27.0 * U(-1, 0, 0)
            + U(-2, 0, 0)) / (24.0 * dx)
    dvdy = (-Vv(0, 1, 0) + 27.0 * Vv(0, 0, 0) - 27.0 * Vv(0, -1, 0)
            + Vv(0, -2, 0)) / (24.0 * dy)
    dwdz = (-W(0, 0, 1) + 27.0 * W(0, 0, 0) - 27.0 * W(0, 0, -1)
            + W(0, 0, -2)) / (24.0 * dz)
    fact = dudx + dvdy + dwdz
    _interior(su, dims)[...] = fact / dt
    return float(np.abs(fact * dx * dy * dz).max())


def wale(u, v, w, vis, dx, dy, dz, rrey, cw, n):
    """kernels.py:297-367 (WALE eddy viscosity, vis = 1/Re + nu_t)."""
    dims = (n, n, n)
    lo = (NPL, NPL, NPL)
    U, Vv, W = _V(u, lo, dims), _V(v, lo, dims), _V(w, lo, dims)
    dudx = (U(0, 0, 0) - U(-1, 0, 0)) / dx
    dudy = (0.25 * (U(0, 1, 0) + U(-1, 1, 0) - U(0, -1, 0) - U(-1, -1, 0))) / dy
    dudz = (0.25 * (U(0, 0, 1) + U(-1, 0, 1) - U(0, 0, -1) - U(-1, 0, -1))) / dz
    dvdx = (0.25 * (Vv(1, 0, 0) + Vv(1, -1, 0) - Vv(-1, 0, 0) - Vv(-1, -1, 0))) / dx
    dvdy = (Vv(0, 0, 0) - Vv(0, -1, 0)) / dy
    dvdz = (0.25 * (Vv(0, 0, 1) + Vv(0, -1, 1) - Vv(0, 0, -1) - Vv(0, -1, -1))) / dz
    dwdx = (0.25 * (W(1, 0, 0) + W(1, 0, -1) - W(-1, 0, 0) - W(-1, 0, -1))) / dx
    dwdy = (0.25 * (W(0, 1, 0) + W(0, 1, -1) - W(0, -1, 0) - W(0, -1, -1))) / dy
    dwdz = (W(0, 0, 0) - W(0, 0, -1)) / dz

    g2xx = dudx * dudx + dudy * dvdx + dudz * dwdx
    g2yy = dvdx * dudy + dvdy * dvdy + dvdz * dwdy
    g2zz = dwdx * dudz + dwdy * dvdz + dwdz * dwdz
    g2xy = dudx * dudy + dudy * dvdy + dudz * dwdy
    g2yx = dvdx * dudx + dvdy * dvdx + dvdz * dwdx
    g2xz = dudx * dudz + dudy * dvdz + dudz * dwdz
    g2zx = dwdx * dudx + dwdy * dvdx + dwdz * dudz
    g2yz = dvdx * dudz + dvdy * dvdz + dvdz * dwdz
    g2zy = dwdx * dudy + dwdy * dvdy + dwdz * dudy

    tr = (g2xx + g2yy + g2zz) / 3.0
    sdxx, sdyy, sdzz = g2xx - tr, g2yy - tr, g2zz - tr
    sdxy = 0.5 * (g2xy + g2yx)
    sdxz = 0.5 * (g2xz + g2zx)
    sdyz = 0.5 * (g2yz + g2zy)
    sdsd = (sdxx * sdxx + sdyy * sdyy + sdzz * sdzz
            + 2.0 * (sdxy * sdxy + sdxz * sdxz + sdyz * sdyz))
    sxx, syy, szz = dudx, dvdy, dwdz
    sxy = 0.5 * (dudy + dvdx)
    sxz = 0.5 * (dudz + dwdx)
    syz = 0.5 * (dvdz + dwdy)
    ss = (sxx * sxx + syy * syy + szz * szz
          + 2.0 * (sxy * sxy + sxz * sxz + syz * syz))
    delta = math.pow(dx * dy * dz, 1.0 / 3.0)
    ls = cw * delta
    with np.errstate(divide="ignore", invalid="ignore"):
        sdsd15 = np.power(sdsd, 1.5)
        denom = np.power(np.abs(ss), 2.5) + np.power(sdsd, 1.25)
        nut = np.where(sdsd > 1.0e-8, ls * ls * sdsd15 / denom, 0.0)
    _interior(vis, dims)[...] = rrey + nut


def maxabs(f, n):
    """kernels.py:374-381."""
    return float(np.abs(_interior(f, (n, n, n))).max())


def dtvisc(u, v, w, vis, dx, dy, dz, n):
    """kernels.py:384-402 (min over cells, initialiser 1e10 at solver.py:127)."""
    dims = (n, n, n)
    lo = (NPL, NPL, NPL)
    U, Vv, W, VI = (_V(u, lo, dims), _V(v, lo, dims), _V(w, lo, dims),
                    _V(vis, lo, dims))
    uc = 0.5 * (U(0, 0, 0) + U(-1, 0, 0))
    vc = 0.5 * (Vv(0, 0, 0) + Vv(0, -1, 0))
    wc = 0.5 * (W(0, 0, 0) + W(0, 0, -1))
    val = 1.0 / (np.abs(uc) / dx + np.abs(vc) / dy + np.abs(wc) / dz
                 + 2.0 * VI(0, 0, 0) * (1.0 / (dx * dx) + 1.0 / (dy * dy)
                                         + 1.0 / (dz * dz)) + 1.0e-30)
    return float(min(1.0e10, val.min()))


def add_ring(dst, src, n):
    """kernels.py:405-414: dst += src over real cells plus one ghost ring."""
    s = slice(NPL - 1, NPL + n + 1)
    dst[s, s, s] += src[s, s, s]


def init_noise(u, v, w, amp, seed, n):
    """kernels.py:452-471: uint32 hash of the padded indices."""
    idx = np.arange(NPL, NPL + n, dtype=np.uint32)
    i = idx[:, None, None]
    j = idx[None, :, None]
    k = idx[None, None, :]
    with np.errstate(over="ignore"):
        h = ((i * np.uint32(73856093)) ^ (j * np.uint32(19349663))
             ^ (k * np.uint32(83492791)) ^ np.uint32(seed))
        h = h ^ (h >> np.uint32(13))
        h = h * np.uint32(1274126177)
        h = h ^ (h >> np.uint32(16))
    r = (h.astype(np.float64) / 4294967295.0) * 2.0 - 1.0
    s = slice(NPL, NPL + n)
    u[s, s, s] = amp * r
    v[s, s, s] = amp * r
    w[s, s, s] = -amp * r


# --------------------------------------------------------------------------
# multigrid (multigrid.py)
# --------------------------------------------------------------------------
class Level:
    """multigrid.py:207-220 plus the coefficient arrays of ``_mgcoeff``
    (multigrid.py:23-67): 1/d^2 faces, zeroed across physical boundaries."""

    def __init__(self, n, dxl, dyl, dzl, dtype=np.float64, phys=ALL_PHYS):
        self.n = n
        self.phys = tuple(phys)
        shp = (n + 2,) * 3
        self.phi = np.zeros(shp, dtype=dtype)
        self.rhs = np.zeros(shp, dtype=dtype)
        s = slice(1, n + 1)
        self.dx, self.dy, self.dz = dxl, dyl, dzl
        cw = np.full((n,) * 3, 1.0 / (dxl * dxl))
        ce = cw.copy()
        cs = np.full((n,) * 3, 1.0 / (dyl * dyl))
        cn = cs.copy()
        cb = np.full((n,) * 3, 1.0 / (dzl * dzl))
        ct = cb.copy()
        # multigrid.py:38-55: zeroed only across a physical face (a seam
        # between ranks keeps its coefficient)
        if phys[0]:
            cw[0, :, :] = 0.0
        if phys[1]:
            ce[n - 1, :, :] = 0.0
        if phys[2]:
            cs[:, 0, :] = 0.0
        if phys[3]:
            cn[:, n - 1, :] = 0.0
        if phys[4]:
            cb[:, :, 0] = 0.0
        if phys[5]:
            ct[:, :, n - 1] = 0.0
        self.aw, self.ae, self.as_, self.an, self.ab, self.at = (
            cw, ce, cs, cn, cb, ct)
        self.ap = -(cw + ce + cs + cn + cb + ct)
        idx = np.arange(n)
        par = (idx[:, None, None] + idx[None, :, None] + idx[None, None, :]) % 2
        # multigrid.py:80: update where (i+j+k+color) % 2 == 1
        self.mask = [par == 1, par == 0]
        self.s = s

    def nbsum(self, phi):
        n, s = self.n, self.s
        return (self.aw * phi[0:n, s, s] + self.ae * phi[2:n + 2, s, s]
                + self.as_ * phi[s, 0:n, s] + self.an * phi[s, 2:n + 2, s]
                + self.ab * phi[s, s, 0:n] + self.at * phi[s, s, 2:n + 2])

    def residual(self, phi=None, rhs=None):
        """rhs - A phi over real cells (multigrid.py:110-117)."""
        phi = self.phi if phi is None else phi
        rhs = self.rhs if rhs is None else rhs
        s = self.s
        return rhs[s, s, s] - (self.nbsum(phi) + self.ap * phi[s, s, s])


def rbgs(lev, color):
    """multigrid.py:70-90: one colour half-sweep (same-colour cells are
    independent, so the vectorised update equals the per-thread one)."""
    s = lev.s
    new = (lev.rhs[s, s, s] - lev.nbsum(lev.phi)) / lev.ap
    core = lev.phi[s, s, s]
    m = lev.mask[color]
    core[m] = new[m]


def restrict(f, c):
    """multigrid.py:93-119 (+ the coarse phi zeroing at 310-312)."""
    res = f.residual()
    nc = c.n
    acc = np.zeros((nc,) * 3)
    for di in range(2):
        for dj in range(2):
            for dk in range(2):
                acc = acc + res[di::2, dj::2, dk::2]
    c.rhs[1:nc + 1, 1:nc + 1, 1:nc + 1] = acc * 0.125
    c.phi[...] = 0.0


def prolong(c, f):
    """multigrid.py:122-146: phi_f += trilinear (1/4, 3/4) of phi_c."""
    n = f.n
    i = np.arange(n)
    c0 = np.where(i % 2 == 0, i // 2 - 1, i // 2)
    w0 = np.where(i % 2 == 0, 0.25, 0.75)
    acc = np.zeros((n,) * 3)
    for di in range(2):
        wx = w0 if di == 0 else 1.0 - w0
        ix = c0 + di + 1
        for dj in range(2):
            wy = w0 if dj == 0 else 1.0 - w0
            iy = c0 + dj + 1
            for dk in range(2):
                wz = w0 if dk == 0 else 1.0 - w0
                iz = c0 + dk + 1
                wgt = (wx[:, None, None] * wy[None, :, None]) * wz[None, None, :]
                acc = acc + wgt * c.phi[np.ix_(ix, iy, iz)]
    s = f.s
    f.phi[s, s, s] = f.phi[s, s, s] + acc


class Multigrid:
    """multigrid.py:223-337.  One rank by default (all six faces physical);
    at a sub-domain, ``phys`` marks the physical faces and ``comm`` (see
    RankComm) exchanges the one-cell rings at the seams."""

    def __init__(self, n, nlev, dx, dy, dz, phys=ALL_PHYS, comm=None):
        self.phys = tuple(phys)
        self.comm = comm
        self.levels = [Level(n >> l, dx * 2.0 ** l, dy * 2.0 ** l, dz * 2.0 ** l,
                             phys=self.phys)
                       for l in range(nlev)]
        self.n_pre, self.n_post = N_PRE, N_POST
        self.n_coarse, self.n_vcycles = N_COARSE, N_VCYCLES

    def refill(self, lev):
        """multigrid.py:264-287: mirror at the physical faces, then the halo
        exchange of the ring (NPL_MG = 1)."""
        mg_refill(lev.phi, lev.n, self.phys)
        if self.comm is not None:
            self.comm.exchange(lev.phi, 1)

    def relax(self, l, nsweeps):
        """multigrid.py:289-299: red, black, then ONE ring refill per sweep."""
        lev = self.levels[l]
        for _ in range(nsweeps):
            rbgs(lev, 0)
            rbgs(lev, 1)
            self.refill(lev)

    def vcycle(self):
        """multigrid.py:301-322."""
        L = len(self.levels)
        for l in range(L):
            if l > 0:
                restrict(self.levels[l - 1], self.levels[l])
            self.relax(l, self.n_pre if l < L - 1 else self.n_coarse)
        for l in range(L - 2, -1, -1):
            prolong(self.levels[l + 1], self.levels[l])
            self.refill(self.levels[l])
            self.relax(l, self.n_post)

    def solve(self, su, pp, n):
        """multigrid.py:324-337."""
        lev0 = self.levels[0]
        s = slice(NPL, NPL + n)
        lev0.rhs[1:n + 1, 1:n + 1, 1:n + 1] = su[s, s, s]
        pp[...] = 0.0
        lev0.phi[...] = 0.0
        for _ in range(self.n_vcycles):
            self.vcycle()
        r = slice(NPL - 1, NPL + n + 1)
        pp[r, r, r] = lev0.phi


# --------------------------------------------------------------------------
# sub-domains (topology.py, halo.py)
# --------------------------------------------------------------------------
def cart_neighbors(rank, sd):
    """topology.py:40-45: ``Create_cart(sd, periods=False, reorder=False)``
    then ``Shift(axis, 1)`` for each axis.  MPI numbers a cartesian
    communicator's ranks in row-major order of their coordinates (the last
    axis fastest), so these neighbours follow that order -- not the x-fastest
    ``_rank_to_coords`` that places the sub-domain (topology.py:56-61).
    -1 marks a physical face."""
    c = [rank // (sd[1] * sd[2]), (rank // sd[2]) % sd[1], rank % sd[2]]
    out = {}
    for axis, name in enumerate("xyz"):
        pair = []
        for step in (-1, 1):
            cc = list(c)
            cc[axis] += step
            if 0 <= cc[axis] < sd[axis]:
                pair.append((cc[0] * sd[1] + cc[1]) * sd[2] + cc[2])
            else:
                pair.append(-1)
        out[name] = tuple(pair)
    return out


def phys_faces(neighbors):
    """multigrid.py:229-231: a face is physical where it has no neighbour
    (the cavity has no periodic face).  Order west, east, south, north,
    bottom, top."""
    return tuple(neighbors["xyz"[f // 2]][f % 2] < 0 for f in range(6))


class RankComm:
    """The reference's communicator calls at one rank of a decomposed run,
    over a torch.distributed group (gloo): ``allreduce`` (solver.py:120,
    134, 150, 176) and the HaloExchanger (halo.py:81-130)."""

    def __init__(self, neighbors):
        self.neighbors = neighbors

    def allreduce(self, x, op):
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(x)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.MIN)
        return float(t.item())

    def _sendrecv(self, snd, peer, stag, rcv, rtag):
        import torch
        import torch.distributed as dist
        st = torch.from_numpy(np.ascontiguousarray(snd))
        rt = torch.empty(rcv.shape, dtype=torch.float64)
        req = dist.isend(st, dst=peer, tag=stag)
        dist.recv(rt, src=peer, tag=rtag)
        req.wait()
        rcv[...] = rt.numpy()

    def exchange(self, arr, npl, nl=None):
        """halo.py:81-130: per axis x, y, z, the ``nl`` real layers next to
        each seam go to the neighbour and its layers land in this side's
        ghosts; a slab spans the whole array in the other two axes, ghosts
        included (tags 21 / 22 paired by data flow)."""
        nl = npl if nl is None else nl
        for axis in range(3):
            lo, hi = self.neighbors["xyz"[axis]]
            if lo < 0 and hi < 0:
                continue
            n = arr.shape[axis] - 2 * npl
            send_lo, send_hi = npl, npl + n - nl
            recv_lo, recv_hi = npl - nl, npl + n
            pairs = []
            if lo >= 0:
                pairs.append((lo, send_lo, recv_lo, 21, 22))
            if hi >= 0:
                pairs.append((hi, send_hi, recv_hi, 22, 21))
            for peer, so, ro, stag, rtag in pairs:
                sl = [slice(None)] * 3
                sl[axis] = slice(so, so + nl)
                rl = [slice(None)] * 3
                rl[axis] = slice(ro, ro + nl)
                self._sendrecv(arr[tuple(sl)], peer, stag, arr[tuple(rl)], rtag)


# --------------------------------------------------------------------------
# solver (solver.py)
# --------------------------------------------------------------------------
FIELDS = ("u", "v", "w", "p", "ustar", "vstar", "wstar", "uoo", "voo", "woo",
          "vis", "su", "pp")


class OracleSolver:
    """solver.py:29-271; ``cfg`` is the reference-shaped CaseConfig
    (config.py:88-98).  One rank by default; with ``rank``/``comm`` (a
    RankComm over a gloo group of sd_x * sd_y * sd_z processes) this is one
    sub-domain of the decomposed run (topology.py:30-53)."""

    def __init__(self, cfg, comm=None):
        self.cfg = cfg
        self.comm = comm
        sd = tuple(int(m) for m in cfg.mpi.domains)
        gn = (cfg.grid.nx, cfg.grid.ny, cfg.grid.nz)
        self.ncells = tuple(g // d for g, d in zip(gn, sd))
        n = self.ncells[0]
        self.n = n
        self.dx = cfg.domain.lx / cfg.grid.nx
        self.dy = cfg.domain.ly / cfg.grid.ny
        self.dz = cfg.domain.lz / cfg.grid.nz
        self.rey = 1.0 / cfg.physics.reynolds
        shp = (n + 2 * NPL,) * 3
        self.f = {k: np.zeros(shp) for k in FIELDS}
        self.ulid = cfg.boundaries.lid_velocity
        phys = phys_faces(comm.neighbors) if comm is not None else ALL_PHYS
        self.mg = Multigrid(n, cfg.numerics.mg_levels, self.dx, self.dy, self.dz,
                            phys=phys, comm=comm)
        self.dt = cfg.time.dt_init
        self.ctime = 0.0
        self.itime = 0
        self.rmax = 0.0
        self.cfl = 0.0
        self.outer_iters = 0
        amp = cfg.initial.noise if cfg.initial.type == "rest" else 0.0
        if amp > 0.0:
            init_noise(self.f["u"], self.f["v"], self.f["w"], amp, 1, n)
        self.f["vis"][...] = self.rey
        apply_initial(self.f, n, self.ulid)

    def _exchange(self, name):
        if self.comm is not None:
            self.comm.exchange(self.f[name], NPL)

    def _allreduce(self, x, op):
        return x if self.comm is None else self.comm.allreduce(x, op)

    def fill_bc(self, name):
        """solver.py:88-97: halo exchange, then the ghost fills (which the
        reference applies on all six faces at every rank)."""
        self._exchange(name)
        if name == "u":
            apply_u(self.f["u"], self.n, self.ulid)
        elif name == "v":
            apply_v(self.f["v"], self.n)
        else:
            apply_w(self.f["w"], self.n)

    def compute_dt(self):
        """solver.py:122-150."""
        f, n = self.f, self.n
        umax = self._allreduce(maxabs(f["u"], n), "max")
        vmax = self._allreduce(maxabs(f["v"], n), "max")
        wmax = self._allreduce(maxabs(f["w"], n), "max")
        dtv = self._allreduce(
            dtvisc(f["u"], f["v"], f["w"], f["vis"], self.dx, self.dy, self.dz, n), "min")
        big = 1.0e10
        dtcfl = big
        for d, um in zip((self.dx, self.dy, self.dz), (umax, vmax, wmax)):
            if um > 0.0:
                dtcfl = min(dtcfl, d / um)
        dtmax = min(dtv, dtcfl)
        if dtmax <= 0.0 or not (dtmax < big):
            raise RuntimeError("time step collapsed (dtmax = %.3e)" % dtmax)
        self.cfl = self.dt / dtmax
        if self.cfg.time.variable_dt:
            self.dt = self._allreduce(min(self.dt * self.cfg.time.dt_growth,
                                          self.cfg.time.safety_factor * dtmax), "min")

    def _calvel(self, alpha):
        """solver.py:155-166 (the halo exchange of u, v, w closes it)."""
        f = self.f
        for comp, star, d in (("u", "ustar", self.dx), ("v", "vstar", self.dy),
                              ("w", "wstar", self.dz)):
            calvel(comp, f[star], f["p"], f[comp], d, self.dt, alpha, self.n)
        for name in ("u", "v", "w"):
            self._exchange(name)

    def _calmas(self):
        f = self.f
        self.rmax = self._allreduce(calmas(f["u"], f["v"], f["w"], f["su"], self.dx,
                                           self.dy, self.dz, self.dt, self.n), "max")

    def _project(self):
        """solver.py:178-212."""
        f = self.f
        eps = self.cfg.numerics.div_tolerance
        maxcy = self.cfg.numerics.max_outer_iters
        self._calvel(1.0)
        iters = 0
        self.rmax_trace = []
        for it in range(1, maxcy + 1):
            iters = it
            self._calmas()
            self.rmax_trace.append(self.rmax)
            if self.rmax < eps and it > 1:
                break
            if self.rmax > 10.0:
                raise RuntimeError("projection diverged: rmax = %.6e at itime %d"
                                   % (self.rmax, self.itime))
            self.mg.solve(f["su"], f["pp"], self.n)
            add_ring(f["p"], f["pp"], self.n)
            self._exchange("p")
            apply_pbound(f["p"], self.n)
            self._calvel(1.0)
        self.outer_iters = iters
        for name in ("u", "v", "w"):
            self.fill_bc(name)

    def step(self):
        """solver.py:217-271."""
        self.itime += 1
        self.compute_dt()
        self.ctime += self.dt
        f, n = self.f, self.n
        f["uoo"][...] = f["u"]
        f["voo"][...] = f["v"]
        f["woo"][...] = f["w"]
        if self.cfg.physics.sgs_enabled:
            wale(f["u"], f["v"], f["w"], f["vis"], self.dx, self.dy, self.dz,
                 self.rey, self.cfg.physics.sgs_cw, n)
            apply_vis(f["vis"], n, self.rey)
        else:
            s = slice(NPL, NPL + n)
            f["vis"][s, s, s] = self.rey
        dt = self.dt
        d3 = (self.dx, self.dy, self.dz)
        comps = (("u", "ustar", "uoo"), ("v", "vstar", "voo"), ("w", "wstar", "woo"))
        for stage, alpha in enumerate(ALFARK):
            for comp, star, oo in comps:
                self.fill_bc(comp)
                conv4th(comp, f["u"], f["v"], f["w"], f[oo], f[star], *d3, dt,
                        alpha, n)
            for comp, star, oo in comps:
                self.fill_bc(comp)
                diff4th(comp, f[comp], f["vis"], f[star], *d3, dt, alpha, n)
            if stage + 1 < len(ALFARK):
                self._calvel(alpha)
        self._project()
        return {"ctime": self.ctime, "dt": self.dt, "rmax": self.rmax,
                "iters": self.outer_iters, "cfl": self.cfl}


def make_mg_rhs(n, seed=0):
    """tests/test_mg.py:35-45: N(0,1) on the level-0 array, ring zeroed,
    interior mean removed."""
    rng = np.random.default_rng(seed)
    h = rng.standard_normal((n + 2,) * 3)
    h[0, :, :] = 0.0
    h[-1, :, :] = 0.0
    h[:, 0, :] = 0.0
    h[:, -1, :] = 0.0
    h[:, :, 0] = 0.0
    h[:, :, -1] = 0.0
    h[1:-1, 1:-1, 1:-1] -= h[1:-1, 1:-1, 1:-1].mean()
    return h


def mg_max_residual(lev):
    """tests/test_mg.py:16-32."""
    return float(np.abs(lev.residual()).max())
