"""Run a function as the ranks of a torch.distributed group, one process per
rank (spawned, so a parent that already touched CUDA is safe), and collect
what each returns.  Used by the sub-domain tests: on CPU the group is gloo;
on one GPU every rank uses cuda:0 and the halos still travel through gloo
(the ranks' kernels never wait on one another on the device)."""
import importlib
import os
import socket
import tempfile
import traceback

import numpy as np

from conftest import PKG, ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _child(rank, nranks, port, modname, fname, args, outdir):
    import sys
    for p in (ROOT, PKG, os.path.dirname(os.path.abspath(__file__))):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(nranks), LOCAL_RANK="0")
    import datetime

    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", rank=rank, world_size=nranks,
                                timeout=datetime.timedelta(seconds=120))
        fn = getattr(importlib.import_module(modname), fname)
        out = fn(rank, nranks, *args)
        np.savez(os.path.join(outdir, "r%d.npz" % rank), **out)
        dist.barrier()
        dist.destroy_process_group()
    except BaseException:
        with open(os.path.join(outdir, "err%d.txt" % rank), "w") as fh:
            fh.write(traceback.format_exc())
        raise


def run_ranks(modname, fname, nranks, args=(), timeout=600):
    """fn(rank, nranks, *args) -> dict of arrays, in `nranks` processes;
    returns the list of the ranks' dicts (raises with a rank's traceback)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    outdir = tempfile.mkdtemp()
    port = _free_port()
    procs = [ctx.Process(target=_child, args=(r, nranks, port, modname, fname, args, outdir))
             for r in range(nranks)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    errs = []
    for r in range(nranks):
        e = os.path.join(outdir, "err%d.txt" % r)
        if os.path.exists(e):
            errs.append("rank %d:\n%s" % (r, open(e).read()))
    if errs or any(p.exitcode != 0 for p in procs):
        raise RuntimeError("rank processes failed (exit codes %s)\n%s"
                           % ([p.exitcode for p in procs], "\n".join(errs)))
    res = []
    for r in range(nranks):
        with np.load(os.path.join(outdir, "r%d.npz" % r)) as z:
            res.append({k: z[k] for k in z.files})
    return res
