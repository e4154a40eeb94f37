"""Stand-in for ``mpi4py.MPI``: the calls the reference makes (topology.py
Create_cart/Shift, halo.py Sendrecv, solver.py allreduce, run.py Barrier).

One rank by default.  With ``REFSHIM_MPI_SIZE`` > 1 in the environment
(and RANK, MASTER_ADDR, MASTER_PORT), the ranks are separate processes
joined by a torch.distributed gloo group, and the calls follow the MPI
standard's documented semantics:

* ``Create_cart(dims, periods, reorder=False)`` numbers the ranks in
  row-major order of their cartesian coordinates (the last dimension
  varies fastest), and ``Shift(direction, 1)`` returns (source, dest): the
  ranks one step below and above along that dimension, or ``PROC_NULL``
  (negative) past a non-periodic end;
* ``Sendrecv`` sends one buffer and receives another, matched by peer and
  tag; ``allreduce`` with ``MAX`` / ``MIN`` reduces a float over all ranks;
  ``Barrier`` waits for every rank.

Golden-vector generation only: the product never imports this.
"""
import os

import numpy as np

MAX = "max"
MIN = "min"
PROC_NULL = -2

_SIZE = int(os.environ.get("REFSHIM_MPI_SIZE", "1"))
_RANK = int(os.environ.get("RANK", "0")) if _SIZE > 1 else 0
_dist = None


def _group():
    global _dist
    if _dist is None:
        import torch.distributed as dist
        dist.init_process_group("gloo", rank=_RANK, world_size=_SIZE)
        _dist = dist
    return _dist


class _Cart:
    def __init__(self, dims, periods):
        self.dims = tuple(int(d) for d in dims)
        self.periods = tuple(bool(p) for p in (periods or (False,) * len(self.dims)))

    def _coords(self, rank):
        c = []
        for d in reversed(self.dims):
            c.append(rank % d)
            rank //= d
        return list(reversed(c))

    def _rank(self, coords):
        r = 0
        for c, d in zip(coords, self.dims):
            r = r * d + c
        return r

    def Shift(self, direction, disp):
        c = self._coords(_RANK)
        out = []
        for step in (-disp, disp):
            cc = list(c)
            cc[direction] += step
            d = self.dims[direction]
            if self.periods[direction]:
                cc[direction] %= d
            elif not 0 <= cc[direction] < d:
                out.append(PROC_NULL)
                continue
            out.append(self._rank(cc))
        return tuple(out)


class Comm:
    def Get_rank(self):
        return _RANK

    def Get_size(self):
        return _SIZE

    def Create_cart(self, dims, periods=None, reorder=False):
        return _Cart(dims, periods)

    def allreduce(self, x, op=None):
        if _SIZE == 1:
            return x
        import torch
        dist = _group()
        t = torch.tensor([float(x)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == MAX else dist.ReduceOp.MIN)
        return float(t.item())

    def Sendrecv(self, sendbuf, dest, sendtag=0, recvbuf=None, source=None, recvtag=0):
        import torch
        dist = _group()
        snd = torch.from_numpy(np.ascontiguousarray(sendbuf))
        rcv = torch.from_numpy(recvbuf)
        req = dist.isend(snd, dst=dest, tag=sendtag)
        dist.recv(rcv, src=source, tag=recvtag)
        req.wait()

    def Barrier(self):
        if _SIZE > 1:
            _group().barrier()


COMM_WORLD = Comm()
