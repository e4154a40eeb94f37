"""Hydro3D restart exchange and Ghia centreline post-processing.

* ``export`` writes a Hydro3D restart (``final_ctime.dat`` and
  ``tecbin0000.bin``) from a solver's current fields, with the ghost layers
  rebuilt to Hydro3D's depth (reference tests/h3d_bridge.py:59-99).
* ``read_tecbin`` reads a Hydro3D ``tecbin`` dump (h3d_bridge.py:102-128);
  ``import_restart`` loads one into a ``FlowSolver`` (real cells, then this
  package's own ghost fills on the device).
* ``compare`` pairs Hydro3D dumps with warpflow snapshots field by field
  (h3d_bridge.py:131-165).
* ``centreline_profiles`` / ``ghia_rms`` / ``write_centreline_csv``: the
  cavity centreline profiles against Ghia et al. (1982) (reference
  scripts/plot_ghia.py:36-50, 95-110).

The tecbin file is Fortran unformatted sequential: three header records --
(tti, ttj, ttk), the ghost depth pl, (-1, -1, -1) -- then one record of 23
doubles per point, i fastest, then j, then k: x, y, z at columns 0-2, p at
3, vis at 6, u at 8, v at 11, w at 14, the rest zero.  Every record is
framed by its byte length as a little-endian int32 before and after.  The
whole body is read and written as one structured array, not record by
record.

    python -m warpflow.h3d export <outdir> [--case X.yaml]
    python -m warpflow.h3d compare <h3d-dir> <snapshot-dir> [--n 80]
    python -m warpflow.h3d ghia <snapshot.npz> --ghia-dir D [--out DIR]
"""
from __future__ import annotations

import argparse
import csv
import os

import numpy as np

NPL = 3                  # ghost layers of this package's fields
PL_H3D = 4               # Hydro3D ghost layers (LMR = 2, pl_ex = 2)
NCOL = 23
COL = {"p": 3, "vis": 6, "u": 8, "v": 11, "w": 14}
_NORMAL = {"west": "u", "east": "u", "south": "v", "north": "v", "bottom": "w", "top": "w"}
_AXIS = {"west": 0, "east": 0, "south": 1, "north": 1, "bottom": 2, "top": 2}

_REC = np.dtype([("head", "<i4"), ("val", "<f8", (NCOL,)), ("tail", "<i4")])


def fill_ghosts(real, name, bnd, npl, ulid):
    """The real cells of one field surrounded by `npl` ghost layers as
    Hydro3D's boundary routine fills them for the cavity (walls, slip,
    moving lid): pressure mirrored; the lid's u = ulid; the face-normal
    component 0; tangential components mirrored with sign +1 on slip and lid
    faces, -1 on walls.  The faces are filled in the order of `bnd`, layer
    by layer, so edges and corners take the value the later face writes
    (h3d_bridge.py:27-56)."""
    n = real.shape[0]
    g = np.zeros((n + 2 * npl,) * 3)
    g[npl:npl + n, npl:npl + n, npl:npl + n] = real
    for side, kind in bnd.items():
        ax = _AXIS[side]
        for m in range(npl):
            if side in ("west", "south", "bottom"):
                gi, ri = npl - 1 - m, npl + m
            else:
                gi, ri = npl + n + m, npl + n - 1 - m
            ghost = [slice(None)] * 3
            inner = [slice(None)] * 3
            ghost[ax], inner[ax] = gi, ri
            if name == "p":
                val = g[tuple(inner)]
            elif kind == "moving_lid" and name == "u":
                val = ulid
            elif name == _NORMAL[side]:
                val = 0.0
            else:
                val = (1.0 if kind in ("slip", "moving_lid") else -1.0) * g[tuple(inner)]
            g[tuple(ghost)] = val
    return g


def write_tecbin(path, fields, n, dx, pl=PL_H3D):
    """Write `fields` ({"u","v","w","p","vis"} -> arrays of (n + 2 pl)^3,
    indexed [i][j][k]) as a tecbin file; point coordinates
    (index - pl + 1/2) dx."""
    t = n + 2 * pl
    with open(path, "wb") as fh:
        np.array([12, t, t, t, 12], "<i4").tofile(fh)
        np.array([4, pl, 4], "<i4").tofile(fh)
        np.array([12, -1, -1, -1, 12], "<i4").tofile(fh)
        body = np.zeros((t, t, t), _REC)            # [k][j][i]: i fastest on disk
        body["head"] = body["tail"] = 8 * NCOL
        xs = (np.arange(t) - pl + 0.5) * dx
        val = body["val"]
        val[..., 0] = xs[None, None, :]
        val[..., 1] = xs[None, :, None]
        val[..., 2] = xs[:, None, None]
        for name, col in COL.items():
            val[..., col] = np.transpose(fields[name], (2, 1, 0))
        body.tofile(fh)


def read_tecbin(path, n, raw=False):
    """The u, v, w, p, vis arrays of a tecbin dump, indexed [i][j][k]: the
    real cells ([pl:pl+n] on every axis), or with raw=True every plane of the
    file, (n + 2 pl)^3 (file plane s at x = (s - 3) dx)."""
    with open(path, "rb") as fh:
        head = np.fromfile(fh, "<i4", 13)
        pl = int(head[6])
        if pl != PL_H3D or head[0] != 12 or head[5] != 4:
            raise ValueError("%s: not a Hydro3D tecbin dump with %d ghost layers"
                             % (path, PL_H3D))
        t = n + 2 * pl
        if tuple(head[1:4]) != (t, t, t):
            raise ValueError("%s holds %s points, expected %d^3 for n = %d"
                             % (path, tuple(head[1:4]), t, n))
        body = np.fromfile(fh, _REC, t ** 3)
    if body.size != t ** 3 or not (np.all(body["head"] == 8 * NCOL)
                                   and np.all(body["tail"] == 8 * NCOL)):
        raise ValueError("%s: truncated or corrupt record stream" % path)
    body = body.reshape(t, t, t)
    out = {}
    s = slice(None) if raw else slice(pl, pl + n)
    for name, col in COL.items():
        a = np.transpose(body["val"][..., col], (2, 1, 0))
        out[name] = np.ascontiguousarray(a[s, s, s])
    return out


def export_fields(sol):
    """A solver's u, v, w, p (and vis = 1/Re) on Hydro3D's ghost depth,
    rebuilt from the real cells (h3d_bridge.py:69-82)."""
    n = sol.ncells[0]
    core = slice(NPL, NPL + n)
    fields = {}
    for name in ("u", "v", "w", "p"):
        real = sol.f[name].numpy()[core, core, core]
        fields[name] = fill_ghosts(real, name, sol.bnd, PL_H3D, sol.ulid)
    fields["vis"] = np.full_like(fields["u"], sol.rey)
    return fields


def export(sol, outdir):
    """``final_ctime.dat`` and ``tecbin0000.bin`` for Hydro3D from `sol`'s
    current state (h3d_bridge.py:59-99); returns the tecbin path."""
    os.makedirs(outdir, exist_ok=True)
    with open(os.path.join(outdir, "final_ctime.dat"), "w") as fh:
        fh.write("       0%18.12f%18.12f%18.12f\n" % (0.0, 0.0, 1.0))
    path = os.path.join(outdir, "tecbin0000.bin")
    write_tecbin(path, export_fields(sol), sol.ncells[0], sol.dx)
    return path


def import_restart(sol, path):
    """Load a tecbin dump's real cells of u, v, w, p and vis into `sol` and
    rebuild this package's ghost layers on the device as a fresh solver's
    are built: ghosts zeroed, then the initial fills of the velocities and
    pressure and the vis fill.  (The fills are ordered face sequences whose
    edge and corner values depend on what the ghosts held before, so the
    ghosts are rebuilt from zero rather than from whatever `sol` held.)"""
    import ctypes

    from . import _abi
    n = sol.ncells[0]
    got = read_tecbin(path, n)
    core = slice(NPL, NPL + n)
    for name in ("u", "v", "w", "p", "vis"):
        a = np.zeros(sol.f[name].shape)
        a[core, core, core] = got[name]
        sol.f[name].assign(a)
    s = sol._stream()
    _abi.call("wf_fill_initial", ctypes.byref(sol.case), s)
    _abi.call("wf_fill_vis", sol.f["vis"].ptr, n, float(sol.rey), s)


def compare(h3ddir, snapdir, n=80, step=25, upto=100):
    """Per field max and rms differences between Hydro3D dumps
    ``h3d_itNNN.bin`` and warpflow snapshots ``snap_NNNNNN_r000.npz`` every
    `step` steps (h3d_bridge.py:131-165).  Hydro3D's file plane s pairs with
    this package's array index s - 1 (planes 4..82 against 3..81 at n = 80);
    pressure is compared demeaned (its additive constant is not fixed).
    Returns {it: {field: (max, rms)}}; missing pairs are skipped."""
    lo, hi = 4, n + 3
    out = {}
    for it in range(step, upto + 1, step):
        hp = os.path.join(h3ddir, "h3d_it%03d.bin" % it)
        sp = os.path.join(snapdir, "snap_%06d_r000.npz" % it)
        if not (os.path.exists(hp) and os.path.exists(sp)):
            continue
        h3d = read_tecbin(hp, n, raw=True)
        z = np.load(sp)
        row = {}
        for name in ("u", "v", "w", "p"):
            mine = z[name][lo - 1:hi - 1, lo - 1:hi - 1, lo - 1:hi - 1].astype(np.float64)
            ref = h3d[name][lo:hi, lo:hi, lo:hi].copy()
            if name == "p":
                mine = mine - mine.mean()
                ref = ref - ref.mean()
            d = np.abs(mine - ref)
            row[name] = (float(d.max()), float(np.sqrt((d ** 2).mean())))
        out[it] = row
    return out


def read_ghia(path):
    """A Ghia et al. table: one header line, then (coordinate, value) rows."""
    data = np.loadtxt(path, skiprows=1)
    return data[:, 0], data[:, 1]


def centreline_profiles(u, w):
    """u(z) on the vertical centreline and w(x) on the horizontal one from
    full (n+6)^3 arrays (plot_ghia.py:36-50).  x = 0.5 is u face n/2 (full
    index n/2 + 2), the centreline cell centre n/2 has full index n/2 + 3,
    and cell centres sit at (c + 1/2) dx.  Returns (zc, u_prof, xc, w_prof)."""
    n = u.shape[0] - 2 * NPL
    if n % 2:
        raise ValueError("centreline profiles need an even n")
    h = n // 2
    zc = (np.arange(n) + 0.5) / n
    u_prof = u[h + 2, h + 3, NPL:NPL + n].copy()
    w_prof = w[NPL:NPL + n, h + 3, h + 2].copy()
    return zc, u_prof, zc.copy(), w_prof


def ghia_rms(profiles, ghia_u, ghia_w):
    """rms deviation of the profiles from the Ghia tables, interpolated at
    the tables' coordinates (plot_ghia.py:95-98): (u rms, w rms)."""
    zc, u_prof, xc, w_prof = profiles
    gz, gu = ghia_u
    gx, gw = ghia_w
    u_err = float(np.sqrt(np.mean((np.interp(gz, zc, u_prof) - gu) ** 2)))
    w_err = float(np.sqrt(np.mean((np.interp(gx, xc, w_prof) - gw) ** 2)))
    return u_err, w_err


def write_centreline_csv(path, profiles):
    """The profiles as CSV, columns z, u_centerline, x, w_centerline
    (plot_ghia.py:100-106)."""
    zc, u_prof, xc, w_prof = profiles
    with open(path, "w", newline="") as fh:
        wr = csv.writer(fh)
        wr.writerow(["z", "u_centerline", "x", "w_centerline"])
        for row in zip(zc, u_prof, xc, w_prof):
            wr.writerow(["%.6f" % row[0], "%.8f" % row[1], "%.6f" % row[2], "%.8f" % row[3]])


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m warpflow.h3d")
    sub = ap.add_subparsers(dest="cmd", required=True)
    e = sub.add_parser("export")
    e.add_argument("outdir")
    e.add_argument("--case", default="cases/cavity_serial.yaml")
    c = sub.add_parser("compare")
    c.add_argument("h3ddir")
    c.add_argument("snapdir")
    c.add_argument("--n", type=int, default=80)
    g = sub.add_parser("ghia")
    g.add_argument("snapshot")
    g.add_argument("--ghia-dir", required=True)
    g.add_argument("--out", default=".")
    args = ap.parse_args(argv)
    if args.cmd == "export":
        from . import FlowSolver, build_topology, load_case
        cfg = load_case(args.case)
        sol = FlowSolver(cfg, build_topology(cfg), "cuda:0")
        print("wrote", export(sol, args.outdir), "ttc =", sol.ncells[0] + 2 * PL_H3D)
    elif args.cmd == "compare":
        for it, row in compare(args.h3ddir, args.snapdir, n=args.n).items():
            print("it %3d" % it)
            for name, (dmax, rms) in row.items():
                print("  %s  max|d| %.3e  rms %.3e" % (name, dmax, rms))
    else:
        z = np.load(args.snapshot)
        prof = centreline_profiles(z["u"], z["w"])
        gu = read_ghia(os.path.join(args.ghia_dir, "Ghia_U.dat"))
        gw = read_ghia(os.path.join(args.ghia_dir, "Ghia_W.dat"))
        u_err, w_err = ghia_rms(prof, gu, gw)
        print("u(z) vs Ghia Re=400: rms = %.4f" % u_err)
        print("w(x) vs Ghia Re=400: rms = %.4f" % w_err)
        os.makedirs(args.out, exist_ok=True)
        write_centreline_csv(os.path.join(args.out, "centreline.csv"), prof)


if __name__ == "__main__":
    main()
