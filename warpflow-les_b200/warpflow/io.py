"""Snapshots (reference warpflow/io.py:9-27): one compressed .npz per rank
with the full u, v, w, p blocks (ghosts included) and the metadata keys
ctime, dt, offsets, ncells, gshape -- the reference's file layout.

Two keys are added so that a run can resume from a snapshot, which the
reference cannot: ``vis`` (the next dt depends on the previous step's
viscosity) and ``itime``.  Readers of the reference format ignore them."""
from pathlib import Path

import numpy as np


def write_snapshot(sol, itime):
    outdir = Path(sol.cfg.output.outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    data = {name: sol.f[name].numpy() for name in ("u", "v", "w", "p", "vis")}
    path = outdir / ("snap_%06d_r%03d.npz" % (itime, sol.topo.rank))
    np.savez_compressed(
        path, **data,
        ctime=np.float64(sol.ctime), dt=np.float64(sol.dt),
        itime=np.int64(sol.itime),
        offsets=np.array(sol.topo.global_offsets, dtype=np.int64),
        ncells=np.array(sol.ncells, dtype=np.int64),
        gshape=np.array((sol.cfg.grid.nx, sol.cfg.grid.ny, sol.cfg.grid.nz),
                        dtype=np.int64))
    return path


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
