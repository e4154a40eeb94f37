"""Generate the golden vectors in this folder by running the reference
solver's own source (warpflow-les v0.1.0: warpflow/{kernels,bcs,multigrid,
solver,config,topology}.py) unmodified on the CPU through ``refshim/``, a
stand-in for NVIDIA Warp and a one-rank mpi4py.

Run once, in a container that has the reference checkout:

    python tests/golden/make_golden.py /path/to/warpflow-les [mg|tecbin|ranks]

``ranks`` runs the reference at several ranks (one process per rank, the
shim's mpi4py joined by a gloo group) on sub-domain decompositions.

Writes ``golden_*.npz`` next to this file.  Nothing at test time reads the
reference; tests only read the committed ``.npz`` files.
"""
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CASE = """
case: {name}
domain:  {{lx: 1.0, ly: 1.0, lz: 1.0}}
grid:    {{nx: {n}, ny: {n}, nz: {n}}}
physics:
  reynolds: {re}
  sgs: {{enabled: {sgs}, model: wale, cw: 0.46}}
initial: {{type: rest, noise: {noise}}}
boundaries:
  west: wall
  east: wall
  south: slip
  north: slip
  bottom: wall
  top: moving_lid
  lid_velocity: {ulid}
numerics:
  mg_levels: {levels}
  max_outer_iters: 30
  div_tolerance: 1.0e-6
time: {{n_steps: {steps}, variable_dt: {vdt}, dt_init: 3.0e-4,
       safety_factor: 0.8, dt_growth: 1.1}}
output: {{n_out: 100000, log_interval: 1, outdir: /tmp/wf_golden}}
mpi: {{domains: [1, 1, 1]}}
"""

# (tag, n, levels, steps, Re, sgs, noise, ulid, variable_dt, fields-after-step)
CAVITY_CASES = [
    ("c8_l3_vdt", 8, 3, 3, 400, "true", 0.01, 1.0, "true", (1, 3)),
    ("c12_l3_fdt_re100", 12, 3, 2, 100, "true", 0.01, 0.75, "false", (1, 2)),
    ("c8_l2_nosgs", 8, 2, 2, 400, "false", 0.01, 1.0, "true", (2,)),
    ("c16_l3_vdt", 16, 3, 1, 400, "true", 0.01, 1.0, "true", (1,)),
]

ALL_FIELDS = ("u", "v", "w", "p", "ustar", "vstar", "wstar", "uoo", "voo",
              "woo", "vis", "su", "pp")

RANK_CASE = """
case: {name}
domain:  {{lx: 1.0, ly: 1.0, lz: 1.0}}
grid:    {{nx: {nx}, ny: {ny}, nz: {nz}}}
physics:
  reynolds: 400
  sgs: {{enabled: true, model: wale, cw: 0.46}}
initial: {{type: rest, noise: 0.01}}
boundaries:
  west: wall
  east: wall
  south: slip
  north: slip
  bottom: wall
  top: moving_lid
  lid_velocity: 1.0
numerics:
  mg_levels: {levels}
  max_outer_iters: 30
  div_tolerance: 1.0e-6
time: {{n_steps: {steps}, variable_dt: true, dt_init: 3.0e-4,
       safety_factor: 0.8, dt_growth: 1.1}}
output: {{n_out: 100000, log_interval: 1, outdir: /tmp/wf_golden}}
mpi: {{domains: [{dx}, {dy}, {dz}]}}
"""

# (tag, global grid, mpi.domains, levels, steps): every rank's sub-domain is
# a cube, as the reference's ghost fills require
RANK_CASES = [
    ("r2x_16x8x8_l3", (16, 8, 8), (2, 1, 1), 3, 2),
    ("r8_16_l2", (16, 16, 16), (2, 2, 2), 2, 1),
]


def main():
    if len(sys.argv) == 5 and sys.argv[2] == "ranks-worker":
        ranks_worker(sys.argv[1], sys.argv[3], sys.argv[4])
        return
    if len(sys.argv) not in (2, 3) or not os.path.isdir(os.path.join(sys.argv[1], "warpflow")):
        sys.exit("usage: python tests/golden/make_golden.py <path of the warpflow-les "
                 "source tree, the directory holding warpflow/> [mg]\n"
                 "  mg: regenerate only the multigrid harness file\n"
                 "  tecbin: regenerate only the Hydro3D exchange file\n"
                 "  ranks: regenerate only the sub-domain decomposition files")
    ref = sys.argv[1]
    only = sys.argv[2] if len(sys.argv) == 3 else None
    if only == "ranks":
        ranks_golden(ref)
        return
    only_mg = only == "mg"
    if only == "tecbin":
        sys.path.insert(0, os.path.join(HERE, "refshim"))
        sys.path.insert(0, ref)
        tecbin_golden(ref)
        return
    sys.path.insert(0, os.path.join(HERE, "refshim"))
    sys.path.insert(0, ref)
    from warpflow.config import load_case
    from warpflow.multigrid import Multigrid
    from warpflow.solver import FlowSolver
    from warpflow.topology import build_topology

    tmp = tempfile.mkdtemp()
    for tag, n, lev, steps, re, sgs, noise, ulid, vdt, keep in (() if only_mg else CAVITY_CASES):
        path = os.path.join(tmp, tag + ".yaml")
        with open(path, "w") as fh:
            fh.write(CASE.format(name=tag, n=n, re=re, sgs=sgs, noise=noise,
                                 ulid=ulid, levels=lev, steps=steps, vdt=vdt))
        cfg = load_case(path)
        topo = build_topology(cfg)
        t0 = time.time()
        sol = FlowSolver(cfg, topo, "cpu")
        out = {"case_yaml": np.array(open(path).read())}
        for name in ("u", "v", "w", "p", "vis"):
            out["init_" + name] = sol.f[name].numpy().copy()
        infos = []
        for s in range(1, steps + 1):
            info = sol.step()
            infos.append([info["ctime"], info["dt"], info["rmax"],
                          info["iters"], info["cfl"]])
            if s in keep:
                names = ALL_FIELDS if s == keep[0] else ("u", "v", "w", "p", "vis")
                for name in names:
                    out["s%d_%s" % (s, name)] = sol.f[name].numpy().copy()
        out["info"] = np.array(infos, dtype=np.float64)
        np.savez_compressed(os.path.join(HERE, "golden_%s.npz" % tag), **out)
        print(tag, "%.1fs" % (time.time() - t0), infos[-1], flush=True)

    # standalone multigrid harness (tests/test_mg.py:35-66): 16^3, 3 levels
    path = os.path.join(tmp, "mg.yaml")
    with open(path, "w") as fh:
        fh.write(CASE.format(name="mg", n=16, re=400, sgs="true", noise=0.01,
                             ulid=1.0, levels=3, steps=1, vdt="true"))
    cfg = load_case(path)
    topo = build_topology(cfg)
    mg = Multigrid(cfg, topo, "cpu", 1.0 / 16, 1.0 / 16, 1.0 / 16)
    lev0 = mg.levels[0]
    rng = np.random.default_rng(0)
    h = rng.standard_normal(lev0.rhs.shape)
    h[0, :, :] = 0.0
    h[-1, :, :] = 0.0
    h[:, 0, :] = 0.0
    h[:, -1, :] = 0.0
    h[:, :, 0] = 0.0
    h[:, :, -1] = 0.0
    h[1:-1, 1:-1, 1:-1] -= h[1:-1, 1:-1, 1:-1].mean()
    lev0.rhs.assign(h)
    lev0.phi.zero_()
    mg._refill(lev0)
    out = {"rhs": h}
    # the coefficient arrays _mgcoeff writes (multigrid.py:23-67), at the
    # harness spacing and at three different spacings per axis
    coef = ("aw", "ae", "as_", "an", "ab", "at", "ap")
    for l, lv in enumerate(mg.levels):
        for name in coef:
            out["coef%d_%s" % (l, name)] = getattr(lv, name).numpy().copy()
    mgx = Multigrid(cfg, topo, "cpu", 0.1, 0.2, 0.3)
    for l, lv in enumerate(mgx.levels):
        for name in coef:
            out["coefx%d_%s" % (l, name)] = getattr(lv, name).numpy().copy()
    for c in range(2):
        mg._vcycle()
        out["phi_c%d" % c] = lev0.phi.numpy().copy()
        out["phi1_c%d" % c] = mg.levels[1].phi.numpy().copy()
        out["phi2_c%d" % c] = mg.levels[2].phi.numpy().copy()
    np.savez_compressed(os.path.join(HERE, "golden_mg16_l3.npz"), **out)
    print("mg16 done", flush=True)


def tecbin_golden(ref):
    """The reference's own Hydro3D exchange (tests/h3d_bridge.py) on an 8^3
    cavity: the tecbin file its ``export`` writes from a freshly initialised
    case, the real cells it started from, and what its ``read_tecbin``
    returns for the file (golden_tecbin_8.npz)."""
    sys.path.insert(0, os.path.join(ref, "tests"))
    import h3d_bridge as hb
    from warpflow import NPL
    from warpflow.config import load_case
    from warpflow.solver import FlowSolver
    from warpflow.topology import build_topology

    tmp = tempfile.mkdtemp()
    path = os.path.join(tmp, "c8.yaml")
    with open(path, "w") as fh:
        fh.write(CASE.format(name="tecbin8", n=8, re=400, sgs="true", noise=0.01,
                             ulid=1.0, levels=2, steps=1, vdt="true"))
    hb.export(tmp, case=path)
    cfg = load_case(path)
    sol = FlowSolver(cfg, build_topology(cfg), "cpu")
    n = 8
    s = slice(NPL, NPL + n)
    out = {"tecbin": np.fromfile(os.path.join(tmp, "tecbin0000.bin"), np.uint8),
           "final_ctime": np.array(open(os.path.join(tmp, "final_ctime.dat")).read()),
           "n": np.array(n), "dx": np.array(sol.dx), "rey": np.array(sol.rey),
           "ulid": np.array(sol.ulid), "bnd": np.array(list(sol.bnd.items()))}
    for name in ("u", "v", "w", "p"):
        out["real_" + name] = sol.f[name].numpy()[s, s, s].copy()
    for raw in (False, True):
        got = hb.read_tecbin(os.path.join(tmp, "tecbin0000.bin"), n, raw=raw)
        for name, a in got.items():
            out[("raw_" if raw else "core_") + name] = a
    np.savez_compressed(os.path.join(HERE, "golden_tecbin_8.npz"), **out)
    print("tecbin done", flush=True)


def ranks_worker(ref, case_path, out_path):
    """One rank of a decomposed run (environment: REFSHIM_MPI_SIZE, RANK,
    MASTER_ADDR, MASTER_PORT): the reference's FlowSolver stepped for the
    case's n_steps; every field after every step, and the step infos."""
    sys.path.insert(0, os.path.join(HERE, "refshim"))
    sys.path.insert(0, ref)
    from warpflow.config import load_case
    from warpflow.solver import FlowSolver
    from warpflow.topology import build_topology

    cfg = load_case(case_path)
    topo = build_topology(cfg)
    sol = FlowSolver(cfg, topo, "cpu")
    out = {"coords": np.array(topo.coords), "local": np.array(topo.local_ncells),
           "neighbors": np.array([topo.neighbors[a] for a in "xyz"])}
    for name in ("u", "v", "w", "p", "vis"):
        out["init_" + name] = sol.f[name].numpy().copy()
    infos = []
    for s in range(1, cfg.time.n_steps + 1):
        info = sol.step()
        infos.append([info["ctime"], info["dt"], info["rmax"], info["iters"], info["cfl"]])
        for name in ALL_FIELDS:
            out["s%d_%s" % (s, name)] = sol.f[name].numpy().copy()
    out["info"] = np.array(infos, dtype=np.float64)
    np.savez(out_path, **out)


def ranks_golden(ref):
    """golden_<tag>.npz for every RANK_CASES entry: the per-rank files of
    one decomposed run, keys prefixed r<rank>_."""
    import socket
    import subprocess
    tmp = tempfile.mkdtemp()
    for tag, (nx, ny, nz), (dx, dy, dz), lev, steps in RANK_CASES:
        path = os.path.join(tmp, tag + ".yaml")
        with open(path, "w") as fh:
            fh.write(RANK_CASE.format(name=tag, nx=nx, ny=ny, nz=nz, levels=lev,
                                      steps=steps, dx=dx, dy=dy, dz=dz))
        nr = dx * dy * dz
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
        t0 = time.time()
        procs = []
        for r in range(nr):
            env = dict(os.environ, REFSHIM_MPI_SIZE=str(nr), RANK=str(r), WORLD_SIZE=str(nr),
                       MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
            procs.append(subprocess.Popen(
                [sys.executable, os.path.abspath(__file__), ref, "ranks-worker", path,
                 os.path.join(tmp, "%s_r%d.npz" % (tag, r))], env=env))
        for p in procs:
            if p.wait() != 0:
                sys.exit("rank process failed for %s" % tag)
        out = {"case_yaml": np.array(open(path).read()), "nranks": np.array(nr)}
        for r in range(nr):
            with np.load(os.path.join(tmp, "%s_r%d.npz" % (tag, r))) as z:
                for k in z.files:
                    out["r%d_%s" % (r, k)] = z[k]
        np.savez_compressed(os.path.join(HERE, "golden_%s.npz" % tag), **out)
        print(tag, "%.1fs" % (time.time() - t0), out["r0_info"][-1], flush=True)


if __name__ == "__main__":
    main()
