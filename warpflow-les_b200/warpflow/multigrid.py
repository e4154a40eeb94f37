"""Geometric multigrid Poisson solver (reference warpflow/multigrid.py),
run by libwfb200's multigrid kernels.

Interface kept from the reference (multigrid.py:207-337): ``levels`` with
``phi``, ``rhs``, ``n3``, ``shape`` and the coefficient arrays ``aw ... ap``
(exposed as read-only host views; the device kernels need none),
``_vcycle()``, ``_relax(l, n)``, ``_refill(lev)``, ``solve(su, pp, npl)`` and
the tunables ``n_pre``, ``n_post``, ``n_coarse``, ``n_vcycles``.

``solve`` works in place: level 0 of the V-cycle is the one-ring core of
``pp`` with ``su`` as its right-hand side, so nothing is copied in or out.
The level-0 ``phi``/``rhs`` arrays serve the standalone harness form
(``_vcycle`` / ``_relax(0, n)``), as in tests/test_mg.py.

``precision="mixed"`` (config ``numerics.mg_precision``) runs every V-cycle
in FP32 as a correction of an FP64 defect correction: the residual, the
accumulation of the solution and everything outside the multigrid stay FP64.

At a sub-domain of a decomposed case (``topo.nranks`` > 1) the solve runs
the reference's own sequence (multigrid.py:264-337) from the host, one
device pass at a time (``wf_rk_mg_op``): face coefficients kept across the
seams between ranks, the Neumann mirror on the physical faces only, and a
halo exchange of the one-cell ring after every full sweep and every
prolongation; FP64, coarsest level by sweeps.

``coarse="operator"`` (config ``numerics.mg_coarse``, the default) runs
the coarsest level's n_coarse sweeps from zero -- a fixed linear map of its
rhs -- through one precomputed dense operator on the even-parity half of
the cells (``wf_mg_build_coarse_op``) and a closing sweep, built once per
(size, spacing, n_coarse, precision) and shared by every Multigrid of the
process; each instance keeps its own partial-sum scratch.  Where the
coarsest edge is not 4..24 in steps of 4, n_coarse < 2, or the operator
would exceed ``COARSE_OP_MAX_BYTES``, the sweeps run as before.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _abi
from .fields import DeviceField, cuda_device

NPL_MG = 1  # one ring layer per level (reference multigrid.py:20)
COARSE_OP_MAX_BYTES = 2 * 1024 ** 3

_COARSE_OPS = {}  # (device, n, nlev, h, n_coarse, dtype) -> built operator tensor


class _CoeffView:
    """Host view of one constant coefficient array of a level
    (reference multigrid.py:23-67: 1/d^2 on real cells, zero across
    physical faces, ap = -sum; zero on the ring)."""

    def __init__(self, lev, which):
        self.lev, self.which = lev, which

    @property
    def shape(self):
        return self.lev.shape

    def numpy(self):
        n = self.lev.n3[0]
        a = np.zeros(self.lev.shape)
        cx, cy, cz = (1.0 / (d * d) for d in self.lev.h)
        core = {}
        for name, c in (("aw", cx), ("ae", cx), ("as_", cy), ("an", cy),
                        ("ab", cz), ("at", cz)):
            core[name] = np.full((n, n, n), c)
        phys = getattr(self.lev, "phys", (True,) * 6)
        if phys[0]:
            core["aw"][0] = 0.0
        if phys[1]:
            core["ae"][n - 1] = 0.0
        if phys[2]:
            core["as_"][:, 0] = 0.0
        if phys[3]:
            core["an"][:, n - 1] = 0.0
        if phys[4]:
            core["ab"][:, :, 0] = 0.0
        if phys[5]:
            core["at"][:, :, n - 1] = 0.0
        if self.which == "ap":
            val = -(core["aw"] + core["ae"] + core["as_"] + core["an"]
                    + core["ab"] + core["at"])
        else:
            val = core[self.which]
        a[1:n + 1, 1:n + 1, 1:n + 1] = val
        return a


class _Level:
    def __init__(self, n3, h, device, dtype=torch.float64, phys=(True,) * 6):
        self.phys = tuple(phys)
        self.n3 = tuple(n3)
        self.shape = tuple(x + 2 for x in n3)
        self.h = tuple(h)
        self.phi = DeviceField.zeros(self.shape, device, dtype)
        self.rhs = DeviceField.zeros(self.shape, device, dtype)
        for name in ("aw", "ae", "as_", "an", "ab", "at", "ap"):
            setattr(self, name, _CoeffView(self, name))


class Multigrid:
    def __init__(self, cfg, topo, device, dx, dy, dz, precision=None, coarse=None):
        self.cfg = cfg
        self.precision = precision or getattr(cfg.numerics, "mg_precision", "fp64")
        if self.precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.coarse = coarse or getattr(cfg.numerics, "mg_coarse", "operator")
        if self.coarse not in ("operator", "sweeps"):
            raise ValueError("coarse must be 'operator' or 'sweeps'")
        # a sub-domain: physical faces are those without a neighbour rank
        # (multigrid.py:229-231); its solve is the reference's sequence
        self.ranks = topo.nranks > 1
        self.phys = tuple(topo.neighbors["xyz"[f // 2]][f % 2] < 0 for f in range(6))
        self.phys_mask = sum(1 << f for f in range(6) if self.phys[f])
        self.halo = None
        if self.ranks:
            if self.precision != "fp64":
                raise ValueError("mg_precision 'mixed' runs at one rank per case")
            self.coarse = "sweeps"
        self._cop_part = None
        self.topo = topo
        self.device = cuda_device(device)
        nb = topo.local_ncells
        if len(set(nb)) != 1:
            raise ValueError("only cubic grids are supported (got %s)" % (nb,))
        self.dx, self.dy, self.dz = dx, dy, dz
        self.levels = []
        for l in range(cfg.numerics.mg_levels):
            s = 2.0 ** l
            self.levels.append(_Level(tuple(x >> l for x in nb),
                                      (dx * s, dy * s, dz * s), self.device, phys=self.phys))
        self._f32 = []
        if self.precision == "mixed":
            for lev in self.levels:
                self._f32.append((DeviceField.zeros(lev.shape, self.device, torch.float32),
                                  DeviceField.zeros(lev.shape, self.device, torch.float32)))
        # scratch of two level arrays per level: the row-parity-split copies
        # of phi and rhs that large levels relax on
        dt = torch.float32 if self.precision == "mixed" else torch.float64
        self._tmp = [DeviceField.zeros((2 * lev.shape[0],) + lev.shape[1:], self.device, dt)
                     for lev in self.levels]
        self._tmp64 = self._tmp if dt == torch.float64 else None
        self.n_pre = 6       # multigrid.py:257-260
        self.n_post = 6
        self.n_coarse = 300
        self.n_vcycles = 4
        self._sc = torch.zeros(ctypes.sizeof(_abi.WfScalars), dtype=torch.uint8,
                               device=self.device)
        self._out = torch.zeros(1, dtype=torch.float64, device=self.device)
        _abi.call("wf_scalars_init", self._sc.data_ptr(), 0.0, 0.0, 0.0, self._stream())
        self.case()   # builds (or finds) the coarse operator now, not in a timed call

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _coarse_op(self, c):
        """(operator, scratch) tensors for case `c` of the full hierarchy, or
        None when the coarse sweeps run as sweeps."""
        if self.coarse != "operator" or c.nlev < 2 or c.n_coarse < 2:
            return None
        op_e, sc_e = ctypes.c_int64(), ctypes.c_int64()
        if _abi.load().wf_mg_coarse_op_elems(ctypes.byref(c), ctypes.byref(op_e),
                                            ctypes.byref(sc_e)) != 0:
            return None
        dt = torch.float32 if c.mg_fp32 else torch.float64
        if op_e.value * (4 if c.mg_fp32 else 8) > COARSE_OP_MAX_BYTES:
            return None
        key = (self.device.index, c.n, c.nlev, c.dx, c.dy, c.dz, c.n_coarse, str(dt))
        op = _COARSE_OPS.get(key)
        if op is None:
            op = torch.empty(op_e.value, dtype=dt, device=self.device)
            c.mg_cop = op.data_ptr()
            _abi.call("wf_mg_build_coarse_op", ctypes.byref(c), self._stream())
            torch.cuda.current_stream(self.device).synchronize()
            _COARSE_OPS[key] = op
        if self._cop_part is None or self._cop_part.numel() != sc_e.value \
                or self._cop_part.dtype != dt:
            self._cop_part = torch.empty(sc_e.value, dtype=dt, device=self.device)
        return op, self._cop_part

    def case(self, su=None, pp=None, levels=None) -> _abi.WfCase:
        """The wf_case the multigrid entry points read (levels >= 1 buffers,
        sweep counts, spacing); ``su``/``pp`` are set for ``solve``."""
        levels = self.levels if levels is None else levels
        c = _abi.WfCase()
        c.n = levels[0].n3[0]
        c.nlev = len(levels)
        c.maxcy = 1
        c.n_pre, c.n_post = self.n_pre, self.n_post
        c.n_coarse, c.n_vcycles = self.n_coarse, self.n_vcycles
        c.dx, c.dy, c.dz = levels[0].h
        if self._f32 and levels is self.levels:
            c.mg_fp32 = 1
            for l, (phi32, rhs32) in enumerate(self._f32):
                c.mg_phi[l] = phi32.ptr
                c.mg_rhs[l] = rhs32.ptr
                c.mg_tmp[l] = self._tmp[l].ptr
        else:
            for l in range(1, len(levels)):
                c.mg_phi[l] = levels[l].phi.ptr
                c.mg_rhs[l] = levels[l].rhs.ptr
            if self._tmp64 is not None:
                for l, lev in enumerate(levels):
                    if lev in self.levels:
                        c.mg_tmp[l] = self._tmp64[self.levels.index(lev)].ptr
        if levels is self.levels:
            cop = self._coarse_op(c)
            if cop is not None:
                c.mg_cop, c.mg_cop_part = cop[0].data_ptr(), cop[1].data_ptr()
        if su is not None:
            c.fld[_abi.FIELD_NAMES.index("su")] = su.ptr
        if pp is not None:
            c.fld[_abi.FIELD_NAMES.index("pp")] = pp.ptr
        c.sc = self._sc.data_ptr()
        return c

    def _refill(self, lev):
        c = self.case(levels=[lev])
        _abi.call("wf_mg_refill", ctypes.byref(c), lev.phi.ptr, self._stream())

    def _relax(self, l, nsweeps):
        lev = self.levels[l]
        c = self.case(levels=[lev])
        _abi.call("wf_mg_relax", ctypes.byref(c), lev.phi.ptr, lev.rhs.ptr,
                  int(nsweeps), self._stream())

    def _coarse_solve(self):
        """The V-cycle's coarsest-level solve on the harness arrays of the
        coarsest level: phi from zero, by the coarse operator when this
        Multigrid uses one, else n_coarse sweeps."""
        lev = self.levels[-1]
        c = self.case()
        if c.mg_fp32:   # the FP32 operator serves FP32 levels only
            c.mg_cop = c.mg_cop_part = None
        _abi.call("wf_mg_coarse_solve", ctypes.byref(c), lev.phi.ptr, lev.rhs.ptr,
                  self._stream())

    def _vcycle(self):
        """One V-cycle on level 0 (multigrid.py:301-322); in mixed precision
        one FP64 defect-correction cycle around an FP32 V-cycle."""
        lev0 = self.levels[0]
        c = self.case()
        name = "wf_mg_dc_cycle" if c.mg_fp32 else "wf_mg_vcycle"
        _abi.call(name, ctypes.byref(c), lev0.phi.ptr, lev0.rhs.ptr, self._stream())

    def residual_max(self, l=0):
        """max |rhs - A phi| of a level (reference tests/test_mg.py:16-32)."""
        lev = self.levels[l]
        c = self.case(levels=[lev])
        _abi.call("wf_mg_residual_max", ctypes.byref(c), lev.phi.ptr, lev.rhs.ptr,
                  self._out.data_ptr(), self._stream())
        return float(self._out.item())

    def solve(self, su3, pp3, npl):
        """A pp = su with 4 V-cycles from zero (reference multigrid.py:324-337)."""
        if npl != 3:
            raise ValueError("solve expects 3-ghost fields")
        c = self.case(su=su3, pp=pp3)
        for i, name in enumerate(_abi.FIELD_NAMES):
            if not c.fld[i]:
                c.fld[i] = su3.ptr  # unused slots must be non-null for validation
        if self.ranks:
            self._solve_ranks(c)
            return
        _abi.call("wf_mg_solve", ctypes.byref(c), self._stream())

    # -- sub-domain form: the reference's sequence, one pass at a time -- #
    def _rk(self, c, op, level, color=0):
        _abi.call("wf_rk_mg_op", ctypes.byref(c), op, level, self.phys_mask, color,
                  self._stream())

    def _rk_refill(self, c, views, l):
        """multigrid.py:264-287: mirror at the physical faces, then the halo
        exchange of the ring."""
        self._rk(c, 1, l)
        ptr, sI, sJ, m = views[l]
        self.halo.exchange_view(ptr, sI, sJ, (m, m, m))

    def _rk_relax(self, c, views, l, nsweeps):
        """multigrid.py:289-299: red, black, one refill per sweep."""
        for _ in range(nsweeps):
            self._rk(c, 0, l, 0)
            self._rk(c, 0, l, 1)
            self._rk_refill(c, views, l)

    def _solve_ranks(self, c):
        """multigrid.py:301-337 at a sub-domain: pp zeroed, n_vcycles
        V-cycles on level 0 = the core of pp (phi) and su (rhs)."""
        if self.halo is None:
            from .halo import HaloExchanger
            self.halo = HaloExchanger(self.topo, self.device, NPL_MG)
        L = c.nlev
        views = []
        for l in range(L):
            ptr, sI, sJ, m = ctypes.c_void_p(), ctypes.c_int64(), ctypes.c_int64(), \
                ctypes.c_int32()
            _abi.call("wf_rk_level_view", ctypes.byref(c), l, ctypes.byref(ptr),
                      ctypes.byref(sI), ctypes.byref(sJ), ctypes.byref(m))
            views.append((ptr.value, sI.value, sJ.value, m.value))
        self._rk(c, 4, 0)
        for _ in range(self.n_vcycles):
            for l in range(L):
                if l > 0:
                    self._rk(c, 2, l)
                self._rk_relax(c, views, l, self.n_pre if l < L - 1 else self.n_coarse)
            for l in range(L - 2, -1, -1):
                self._rk(c, 3, l)
                self._rk_refill(c, views, l)
                self._rk_relax(c, views, l, self.n_post)
