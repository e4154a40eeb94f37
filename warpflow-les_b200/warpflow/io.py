"""Snapshots (reference warpflow/io.py:9-27): one compressed .npz per rank
with the full u, v, w, p blocks (ghosts included) and the metadata keys
ctime, dt, offsets, ncells, gshape -- the reference's file layout.

Two keys are added so that a run can resume from a snapshot, which the
reference cannot: ``vis`` (the next dt depends on the previous step's
viscosity) and ``itime``.  Readers of the reference format ignore them."""
import concurrent.futures
from pathlib import Path

import numpy as np
import torch

SNAP_FIELDS = ("u", "v", "w", "p", "vis")


def _snap_path(sol, itime):
    outdir = Path(sol.cfg.output.outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    return outdir / ("snap_%06d_r%03d.npz" % (itime, sol.topo.rank))


def _save(path, data, meta):
    np.savez_compressed(path, **data, **meta)
    return path


def _meta(sol):
    return dict(ctime=np.float64(sol.ctime), dt=np.float64(sol.dt),
                itime=np.int64(sol.itime),
                offsets=np.array(sol.topo.global_offsets, dtype=np.int64),
                ncells=np.array(sol.ncells, dtype=np.int64),
                gshape=np.array((sol.cfg.grid.nx, sol.cfg.grid.ny, sol.cfg.grid.nz),
                                dtype=np.int64))


def write_snapshot(sol, itime):
    """Write the snapshot now (the caller waits for the device and the file)."""
    data = {name: sol.f[name].numpy() for name in SNAP_FIELDS}
    return _save(_snap_path(sol, itime), data, _meta(sol))


class SnapshotWriter:
    """Snapshots that do not stall the step stream.  ``write`` copies the
    fields device-to-device into a staging set on the solver's stream (a
    few microseconds at 80^3), then a side stream moves them into pinned
    host buffers while later steps run, and a worker thread compresses and
    writes the file once that copy has landed.  One snapshot is in flight at
    a time: the next ``write`` (or ``close``) first waits for the previous
    file.  Files are identical to ``write_snapshot``'s."""

    def __init__(self, sol):
        self.sol = sol
        dev = sol.device
        self._stage = {n: torch.empty_like(sol.f[n].t) for n in SNAP_FIELDS}
        self._host = {n: torch.empty(sol.f[n].t.shape, dtype=sol.f[n].t.dtype,
                                     pin_memory=True) for n in SNAP_FIELDS}
        self._copy = torch.cuda.Stream(dev)
        self._pool = concurrent.futures.ThreadPoolExecutor(max_workers=1)
        self._pending = None

    def write(self, itime):
        self.wait()
        sol = self.sol
        main = torch.cuda.current_stream(sol.device)
        for n in SNAP_FIELDS:
            self._stage[n].copy_(sol.f[n].t, non_blocking=True)
        staged = torch.cuda.Event()
        staged.record(main)
        with torch.cuda.stream(self._copy):
            self._copy.wait_event(staged)
            for n in SNAP_FIELDS:
                self._host[n].copy_(self._stage[n], non_blocking=True)
            landed = torch.cuda.Event()
            landed.record(self._copy)
        path, meta = _snap_path(sol, itime), _meta(sol)

        def finish():
            landed.synchronize()
            return _save(path, {n: self._host[n].numpy() for n in SNAP_FIELDS}, meta)

        self._pending = self._pool.submit(finish)
        return path

    def wait(self):
        """Block until the snapshot in flight (if any) is on disk; its path."""
        if self._pending is None:
            return None
        fut, self._pending = self._pending, None
        return fut.result()

    def close(self):
        self.wait()
        self._pool.shutdown()


def read_snapshot(path):
    """Load a snapshot written by ``write_snapshot`` into a dict."""
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def restore(sol, snap):
    """Put a snapshot's state into a FlowSolver of the same case: u, v, w,
    p, vis (ghosts included), dt, ctime and itime."""
    n = tuple(int(x) for x in snap["ncells"])
    if n != tuple(sol.ncells):
        raise ValueError("snapshot grid %s does not match the solver's %s" % (n, sol.ncells))
    missing = [k for k in ("vis", "itime") if k not in snap]
    if missing:
        raise ValueError("snapshot lacks %s (written by a reference build?); "
                         "it cannot be resumed exactly" % missing)
    for name in ("u", "v", "w", "p", "vis"):
        sol.f[name].assign(snap[name])
    sol.set_time_state(dt=float(snap["dt"]), ctime=float(snap["ctime"]),
                       itime=int(snap["itime"]))
