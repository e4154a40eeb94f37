"""Time-marching flow solver (reference warpflow/solver.py), B200 build.

``FlowSolver.step()`` is one launch of a CUDA graph built once per solver
by libwfb200 (``wf_stepper_*``): dt control, WALE, both Heun RK2 stages,
and the projection loop all run on the device, and the loop's
data-dependent exit is a conditional graph node set by the divergence
kernel.  The host reads one small scalar block per step (the reference
makes five or more blocking readbacks, solver.py:119,133,175).

Public interface as the reference (solver.py:29-271): constructor
``FlowSolver(cfg, topo, device)``, ``step() -> {ctime, dt, rmax, iters,
cfl}``, the field dict ``f`` (13 names), ``ncells``, ``dx/dy/dz``, ``rey``,
``dt``, ``ctime``, ``itime``, ``rmax``, ``cfl``, ``outer_iters``, ``bnd``,
``ulid``, ``mg``, ``cfg``, ``topo``; same exception messages.

At a sub-domain of a decomposed case (``topo.nranks`` > 1, one process per
GPU) ``step()`` runs the reference's own sequence from the host instead of
the graph: each device pass through its C-ABI entry, the halo exchange
before every ghost fill and after every velocity correction, and the
reference's allreduces of the dt reductions and of the divergence maximum
(solver.py:88-212).
"""
from __future__ import annotations

import ctypes
import os

import torch

from . import _abi
from .bcs import BoundaryKernels
from .fields import DeviceField, cuda_device
from .multigrid import Multigrid
from .topology import MAX, MIN, NPL

ALFARK = (0.5, 1.0)  # Heun RK2 stage coefficients (reference solver.py:26)

STEP_MODES = {"graph": 0, "host": 1}
STEP_SERIAL = 2   # WF_STEP_SERIAL: no programmatic dependent launch


class FlowSolver:
    def __init__(self, cfg, topo, device, step_mode=None, serial=True):
        """`serial` (the default) builds the step without programmatic
        dependent launch: each kernel's CTAs become resident only after the
        previous kernel finished.  Measured on B200 the single-case step
        graph is about 1.3 % faster that way at 80^3 (1.008 against 1.024 ms
        and 1.019 against 1.031 ms in two runs; 256^3 and 512^3 unchanged),
        and many solvers stepping concurrently need it (waiting CTAs would
        hold SMs other streams could use).  `serial=False` launches the
        step's kernels with programmatic dependent launch; the results are
        the same bits."""
        self.cfg = cfg
        self.topo = topo
        dev = cuda_device(device)
        self.device = dev
        ni, nj, nk = topo.local_ncells
        if not (ni == nj == nk):
            raise ValueError("only cubic grids are supported (got %s)" % ((ni, nj, nk),))
        self.ncells = (ni, nj, nk)
        self.n = ni
        self.dx = cfg.domain.lx / cfg.grid.nx
        self.dy = cfg.domain.ly / cfg.grid.ny
        self.dz = cfg.domain.lz / cfg.grid.nz
        self.rey = 1.0 / cfg.physics.reynolds

        shape = (ni + 2 * NPL,) * 3
        self.f = {name: DeviceField.zeros(shape, dev) for name in _abi.FIELD_NAMES}

        b = cfg.boundaries
        self.bnd = {"west": b.west, "east": b.east, "south": b.south,
                    "north": b.north, "bottom": b.bottom, "top": b.top}
        self.bcs = BoundaryKernels(self.bnd, dev)
        self.ulid = b.lid_velocity
        self.mg = Multigrid(cfg, topo, dev, self.dx, self.dy, self.dz)
        self.mixed = self.mg.precision == "mixed"

        nsc = ctypes.sizeof(_abi.WfScalars)
        self._sc = torch.zeros(nsc, dtype=torch.uint8, device=dev)
        self._sc_host = torch.zeros(nsc, dtype=torch.uint8, pin_memory=True)
        self._sc_view = _abi.WfScalars.from_address(self._sc_host.data_ptr())

        self._dt = cfg.time.dt_init
        self._ctime = 0.0
        self.itime = 0
        self.rmax = 0.0
        self.cfl = 0.0
        self.outer_iters = 0
        self.rmax_trace = []

        self.case = self._make_case()
        self._init_state()

        self.ranks = topo.nranks > 1
        self._stepper = None
        self.serial = bool(serial)
        if self.ranks:
            from .halo import HaloExchanger
            self.halo = HaloExchanger(topo, dev, NPL)
            self.step_mode = "ranks"
            return
        mode = step_mode or os.environ.get("WF_STEP_MODE", "graph")
        if mode not in STEP_MODES:
            raise ValueError("step_mode must be one of %s" % sorted(STEP_MODES))
        self.step_mode = mode
        self._stepper = ctypes.c_void_p()
        _abi.call("wf_stepper_create", ctypes.byref(self.case),
                  STEP_MODES[mode] | (STEP_SERIAL if serial else 0),
                  ctypes.byref(self._stepper))

    def _init_state(self):
        """solver.py:30-83 initial state on the device: scalars (with 1/Re and
        the lid velocity the step reads), hash noise, vis = 1/Re, initial
        ghost fills."""
        cfg, ni = self.cfg, self.n
        s = self._stream()
        _abi.call("wf_scalars_init", self._sc.data_ptr(), float(self._dt), float(self.rey),
                  float(self.ulid), s)
        amp = cfg.initial.noise if cfg.initial.type == "rest" else 0.0
        if amp > 0.0:
            _abi.call("wf_init_noise", self.f["u"].ptr, self.f["v"].ptr, self.f["w"].ptr,
                      ni, float(amp), 1, s)
        self.f["vis"].fill_(self.rey)
        _abi.call("wf_fill_initial", ctypes.byref(self.case), s)

    def reset(self, cfg):
        """Start over as the case `cfg`, which may differ from this solver's
        only in its Reynolds number, lid velocity, initial dt and step count:
        every field is zeroed and re-initialised on the device, and the
        built step is reused (it reads 1/Re and the lid velocity from the
        scalar block).  No allocation, no graph capture.  Used by the server
        to serve a new request from a resident solver of the same size."""
        same = (cfg.grid, cfg.domain, cfg.numerics, cfg.initial, cfg.physics.sgs_enabled,
                cfg.physics.sgs_cw, cfg.time.variable_dt, cfg.time.dt_growth,
                cfg.time.safety_factor)
        old = (self.cfg.grid, self.cfg.domain, self.cfg.numerics, self.cfg.initial,
               self.cfg.physics.sgs_enabled, self.cfg.physics.sgs_cw, self.cfg.time.variable_dt,
               self.cfg.time.dt_growth, self.cfg.time.safety_factor)
        b, ob = cfg.boundaries, self.cfg.boundaries
        if same != old or (b.west, b.east, b.south, b.north, b.bottom, b.top) != \
                (ob.west, ob.east, ob.south, ob.north, ob.bottom, ob.top):
            raise ValueError("reset: the new case must match this solver's grid, "
                             "boundaries and numerics")
        self.cfg = cfg
        self.rey = 1.0 / cfg.physics.reynolds
        self.ulid = b.lid_velocity
        self._dt = cfg.time.dt_init
        self._ctime = 0.0
        self.itime = 0
        self.rmax = 0.0
        self.cfl = 0.0
        self.outer_iters = 0
        self.rmax_trace = []
        self.case.rrey = self.rey
        self.case.ulid = float(self.ulid)
        for f in self.f.values():
            f.zero_()
        self._init_state()

    # ------------------------------------------------------------------ #
    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _make_case(self) -> _abi.WfCase:
        cfg = self.cfg
        c = self.mg.case()
        c.sgs = 1 if cfg.physics.sgs_enabled else 0
        c.variable_dt = 1 if cfg.time.variable_dt else 0
        c.maxcy = int(cfg.numerics.max_outer_iters)
        c.dx, c.dy, c.dz = self.dx, self.dy, self.dz
        c.rrey = self.rey
        c.cw = float(cfg.physics.sgs_cw)
        c.ulid = float(self.ulid)
        c.dt_growth = float(cfg.time.dt_growth)
        c.safety = float(cfg.time.safety_factor)
        c.eps = float(cfg.numerics.div_tolerance)
        for i, name in enumerate(_abi.FIELD_NAMES):
            c.fld[i] = self.f[name].ptr
        c.sc = self._sc.data_ptr()
        return c

    def _pull_scalars(self):
        self._sc_host.copy_(self._sc, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return self._sc_view

    def _push_scalar(self, name, value):
        sc = self._pull_scalars()
        setattr(sc, name, value)
        self._sc.copy_(self._sc_host, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()

    @property
    def dt(self):
        return self._dt

    @dt.setter
    def dt(self, value):
        self._dt = float(value)
        self._push_scalar("dt", self._dt)

    @property
    def ctime(self):
        return self._ctime

    @ctime.setter
    def ctime(self, value):
        self._ctime = float(value)
        self._push_scalar("ctime", self._ctime)

    def set_time_state(self, dt, ctime, itime):
        """Set dt, ctime and itime on the device and the host (resume)."""
        sc = self._pull_scalars()
        sc.dt, sc.ctime, sc.itime = float(dt), float(ctime), int(itime)
        self._sc.copy_(self._sc_host, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        self._dt, self._ctime, self.itime = float(dt), float(ctime), int(itime)

    # ------------------------------------------------------------------ #
    def fill_bc(self, name, alfabc=0):
        """One boundu/boundv/boundw call (reference solver.py:88-97)."""
        n = self.n
        if name == "u":
            self.bcs.apply_u(self.f["u"], n, self.ulid, alfabc)
        elif name == "v":
            self.bcs.apply_v(self.f["v"], n, alfabc)
        elif name == "w":
            self.bcs.apply_w(self.f["w"], n, alfabc)

    def step(self):
        """One time step (reference solver.py:217-271)."""
        if self.ranks:
            return self._step_ranks()
        self.launch_step()
        return self.finish_step()

    # -- sub-domain form (solver.py:88-271 at one of several ranks) ------ #
    def _fill_bc_ranks(self, name):
        """solver.py:88-97: halo exchange, then the ghost fills (the
        reference fills all six faces at every rank)."""
        self.halo.exchange(self.f[name])
        self.fill_bc(name)

    def _calvel_ranks(self, alpha):
        """solver.py:155-166: the correction, then the halo exchange of u,
        v, w (no ghost fill)."""
        _abi.call("wf_calvel", ctypes.byref(self.case), float(alpha), self._dt_dev,
                  self._stream())
        for name in ("u", "v", "w"):
            self.halo.exchange(self.f[name])

    def _step_ranks(self):
        c, s, comm = ctypes.byref(self.case), self._stream(), self.topo.comm
        cfg = self.cfg
        self._dt_dev = ctypes.c_void_p(self._sc.data_ptr() + _abi.WfScalars.dt.offset)
        self.itime += 1
        # solver.py:122-150: this rank's reductions on the device, the
        # global ones and the dt update on the host
        _abi.call("wf_checkdt", c, s)
        sc = self._pull_scalars()
        umax = comm.allreduce(float(sc.umax), op=MAX)
        vmax = comm.allreduce(float(sc.vmax), op=MAX)
        wmax = comm.allreduce(float(sc.wmax), op=MAX)
        dtvisc = comm.allreduce(float(sc.dtvisc), op=MIN)
        big = 1.0e10
        dtcfl = big
        for d, um in zip((self.dx, self.dy, self.dz), (umax, vmax, wmax)):
            if um > 0.0:
                dtcfl = min(dtcfl, d / um)
        dtmax = min(dtvisc, dtcfl)
        if dtmax <= 0.0 or not (dtmax < big):
            raise RuntimeError("time step collapsed (dtmax = %.3e)" % dtmax)
        self.cfl = self._dt / dtmax
        if cfg.time.variable_dt:
            self._dt = comm.allreduce(min(self._dt * cfg.time.dt_growth,
                                          cfg.time.safety_factor * dtmax), op=MIN)
        self._ctime += self._dt
        sc.dt, sc.ctime, sc.itime, sc.cfl, sc.dtmax = (self._dt, self._ctime, self.itime,
                                                       self.cfl, dtmax)
        sc.status = _abi.ST_OK
        self._sc.copy_(self._sc_host, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()

        _abi.call("wf_copy_oo", c, s)
        _abi.call("wf_wale_vis", c, s)
        for stage, alpha in enumerate(ALFARK):
            for comp in range(3):
                self._fill_bc_ranks("uvw"[comp])
                _abi.call("wf_conv", c, comp, float(alpha), self._dt_dev, s)
            for comp in range(3):
                self._fill_bc_ranks("uvw"[comp])
                _abi.call("wf_diff", c, comp, float(alpha), self._dt_dev, s)
            if stage + 1 < len(ALFARK):
                self._calvel_ranks(alpha)

        # solver.py:178-212
        eps = cfg.numerics.div_tolerance
        maxcy = cfg.numerics.max_outer_iters
        self._calvel_ranks(1.0)
        iters = 0
        self.rmax_trace = []
        for it in range(1, maxcy + 1):
            iters = it
            _abi.call("wf_calmas", c, s)
            self.rmax = comm.allreduce(float(self._pull_scalars().rmax), op=MAX)
            self.rmax_trace.append(self.rmax)
            if self.rmax < eps and it > 1:
                break
            if self.rmax > 10.0:
                raise RuntimeError("projection diverged: rmax = %.6e at itime %d"
                                   % (self.rmax, self.itime))
            self.mg.solve(self.f["su"], self.f["pp"], NPL)
            _abi.call("wf_add_ring", self.f["p"].ptr, self.f["pp"].ptr, self.n, s)
            self.halo.exchange(self.f["p"])
            self.bcs.apply_pbound(self.f["p"], self.n)
            self._calvel_ranks(1.0)
        else:
            if self.topo.rank == 0:
                print("warning: projection did not converge, rmax = %.6e after %d "
                      "iterations" % (self.rmax, maxcy), flush=True)
        self.outer_iters = iters
        for name in ("u", "v", "w"):
            self._fill_bc_ranks(name)
        sc = self._pull_scalars()
        sc.rmax, sc.iters, sc.status = self.rmax, iters, _abi.ST_OK
        self._sc.copy_(self._sc_host, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return {"ctime": self._ctime, "dt": self._dt, "rmax": self.rmax,
                "iters": self.outer_iters, "cfl": self.cfl}

    def launch_step(self):
        """Enqueue one step on the current stream without waiting."""
        if self.ranks:
            raise RuntimeError("a sub-domain steps through step() (its halo exchanges "
                               "and allreduces need the host)")
        _abi.call("wf_stepper_step", self._stepper, self._stream())

    def launch_counts(self):
        """Kernel launches of (prologue, calmas pass, multigrid part,
        epilogue) of this solver's step."""
        arr = (ctypes.c_int32 * 4)()
        _abi.call("wf_stepper_launch_counts", self._stepper, arr)
        return tuple(arr)

    def finish_step(self):
        """Wait for the enqueued step, update the host-side scalars and raise
        the reference's errors."""
        return self.apply_scalars(self._pull_scalars())

    def apply_scalars(self, sc):
        """Take the device scalar block of a finished step (a WfScalars view)
        into the host attributes; raise the reference's errors."""
        self.last_nmg = int(sc.nmg)
        self.itime = int(sc.itime)
        self._dt = float(sc.dt)
        self._ctime = float(sc.ctime)
        self.rmax = float(sc.rmax)
        self.cfl = float(sc.cfl)
        self.outer_iters = int(sc.iters)
        self.rmax_trace = [float(sc.rmax_trace[i])
                           for i in range(min(self.outer_iters, 32))]
        st = int(sc.status)
        if st == _abi.ST_DT_COLLAPSE:
            raise RuntimeError("time step collapsed (dtmax = %.3e)" % sc.dtmax)
        if st == _abi.ST_DIVERGED:
            raise RuntimeError("projection diverged: rmax = %.6e at itime %d"
                               % (self.rmax, self.itime))
        if st == _abi.ST_WAIT_TIMEOUT:
            raise RuntimeError("device-side wait timed out in the multigrid coarse solve "
                               "(itime %d); results of this step are invalid" % self.itime)
        if st == _abi.ST_NOT_CONVERGED:
            if self.topo.rank == 0:
                print("warning: projection did not converge, rmax = %.6e after %d "
                      "iterations" % (self.rmax, self.cfg.numerics.max_outer_iters),
                      flush=True)
            self._push_scalar("status", _abi.ST_OK)
        return {"ctime": self._ctime, "dt": self._dt, "rmax": self.rmax,
                "iters": self.outer_iters, "cfl": self.cfl}

    def device_bytes(self):
        """Device memory held by this solver's fields, multigrid hierarchy,
        scratch and scalar block (a coarse-level operator is shared by all
        solvers of its size and not counted here)."""
        ts = [f.t for f in self.f.values()] + [self._sc]
        for lev in self.mg.levels:
            ts += [lev.phi.t, lev.rhs.t]
        for a, b in self.mg._f32:
            ts += [a.t, b.t]
        ts += [t.t for t in self.mg._tmp]
        ts += [self.mg._sc, self.mg._out]
        if self.mg._cop_part is not None:   # the coarse operator itself is shared
            ts.append(self.mg._cop_part)
        return int(sum(t.numel() * t.element_size() for t in ts))

    def close(self):
        if getattr(self, "_stepper", None):
            _abi.load().wf_stepper_destroy(self._stepper)
            self._stepper = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
