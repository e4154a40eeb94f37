"""Snapshot output (reference warpflow/io.py:9-27): one compressed .npz per
rank with the full u, v, w, p blocks (ghosts included) and the metadata
keys ctime, dt, offsets, ncells, gshape."""
from pathlib import Path

import numpy as np


def write_snapshot(sol, itime):
    outdir = Path(sol.cfg.output.outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    data = {name: sol.f[name].numpy() for name in ("u", "v", "w", "p")}
    path = outdir / ("snap_%06d_r%03d.npz" % (itime, sol.topo.rank))
    np.savez_compressed(
        path, **data,
        ctime=np.float64(sol.ctime), dt=np.float64(sol.dt),
        offsets=np.array(sol.topo.global_offsets, dtype=np.int64),
        ncells=np.array(sol.ncells, dtype=np.int64),
        gshape=np.array((sol.cfg.grid.nx, sol.cfg.grid.ny, sol.cfg.grid.nz),
                        dtype=np.int64))
    return path
