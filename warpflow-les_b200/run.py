"""Command-line driver (reference run.py:20-65, same flags and log lines).

    python warpflow-les_b200/run.py --case case.yaml [--device auto|cuda:0]
                                    [--steps N] [--outdir D] [--resume SNAP]

Runs `time.n_steps` (or --steps) FlowSolver steps, prints the reference's
log line every `output.log_interval` steps and writes a snapshot every
`output.n_out` steps and at the end.  --resume continues from a snapshot
written by this package's snapshot writer (it also holds vis and itime).

A case whose `mpi.domains` has more than one sub-domain runs one process
per rank under torchrun, where the reference runs under mpirun:

    torchrun --nproc-per-node 8 warpflow-les_b200/run.py --case case.yaml

Each rank joins the process group (NCCL between GPUs) on GPU LOCAL_RANK
and writes its own snapshot files (snap_<itime>_r<rank>.npz).
WF_DIST_BACKEND=gloo moves the halos through host memory instead, and
then ranks may share a GPU (LOCAL_RANK modulo the GPU count).
"""
import argparse
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from warpflow import FlowSolver, __version__, build_topology, load_case  # noqa: E402
from warpflow.io import SnapshotWriter, read_snapshot, restore  # noqa: E402


def _join_ranks(cfg):
    """Join the torch.distributed group for a decomposed case; returns the
    rank's GPU, or None for a single-domain case (or when torchrun did not
    start several processes: build_topology then reports the mismatch)."""
    sd = cfg.mpi.domains
    if sd[0] * sd[1] * sd[2] == 1 or int(os.environ.get("WORLD_SIZE", "1")) == 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", "0"))
    backend = os.environ.get("WF_DIST_BACKEND", "nccl")
    if backend not in ("nccl", "gloo"):
        raise ValueError("WF_DIST_BACKEND must be nccl or gloo")
    if backend == "gloo":
        local %= max(1, torch.cuda.device_count())
    if not dist.is_initialized():
        torch.cuda.set_device(local)
        kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300), **kw)
    return "cuda:%d" % local


def main(argv=None):
    ap = argparse.ArgumentParser(description="warpflow-les solver (B200 build)")
    ap.add_argument("--case", required=True, help="case YAML file")
    ap.add_argument("--device", default="auto", help="auto | cuda:N (no CPU path)")
    ap.add_argument("--steps", type=int, default=None,
                    help="override time.n_steps from the case file")
    ap.add_argument("--outdir", default=None, help="override output.outdir")
    ap.add_argument("--resume", default=None, help="snapshot .npz to continue from")
    args = ap.parse_args(argv)

    cfg = load_case(args.case)
    if args.outdir:
        cfg.output.outdir = args.outdir
    nsteps = args.steps if args.steps is not None else cfg.time.n_steps
    rank_dev = _join_ranks(cfg)
    topo = build_topology(cfg)
    device = args.device
    if device == "auto":
        device = rank_dev or "cuda:0"
    if topo.rank == 0:
        print("warpflow-les %s: case=%s grid=%dx%dx%d domains=%s device=%s"
              % (__version__, cfg.name, cfg.grid.nx, cfg.grid.ny, cfg.grid.nz,
                 list(cfg.mpi.domains), device), flush=True)
    sol = FlowSolver(cfg, topo, device=device)
    start = 0
    if args.resume:
        restore(sol, read_snapshot(args.resume))
        start = sol.itime
    snaps = SnapshotWriter(sol)
    t0 = time.time()
    for itime in range(start + 1, start + nsteps + 1):
        info = sol.step()
        if itime % cfg.output.log_interval == 0 and topo.rank == 0:
            print("it %6d  ctime %.6f  dt %.3e  rmax %.3e  outer %2d  cfl %.2f"
                  % (itime, info["ctime"], info["dt"], info["rmax"], info["iters"],
                     info["cfl"]), flush=True)
        if itime % cfg.output.n_out == 0:
            snaps.write(itime)
    last = start + nsteps
    if last % cfg.output.n_out != 0:
        snaps.write(last)
    snaps.close()
    if topo.rank == 0:
        print("done: itime=%d ctime=%.6f wall=%.1fs" % (last, sol.ctime, time.time() - t0),
              flush=True)
    sol.close()
    if rank_dev is not None:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
