"""Domain decomposition (reference warpflow/topology.py).

``build_topology(cfg)`` returns the reference's ``Topology`` fields
(topology.py:18-53).  With ``mpi.domains`` [1, 1, 1] it is one rank owning
the whole grid, every neighbour a physical boundary (-1).  With more
domains, each rank of a torch.distributed process group (one process per
GPU: NCCL, or gloo on the CPU) owns one sub-domain:

* the group must have exactly sd_x * sd_y * sd_z ranks (the reference's
  rank-count check, topology.py:33-37);
* ``coords`` places the sub-domain x-fastest (topology.py:56-61), and
  ``global_offsets`` follow from it;
* ``neighbors`` are what the reference gets from
  ``Create_cart(sd, periods=False, reorder=False).Shift(axis, 1)``
  (topology.py:39-45): MPI numbers a cartesian communicator's ranks in
  row-major order of their coordinates (the last axis fastest), so the
  neighbours follow that order, not the x-fastest placement -- kept as the
  reference has it, since the halo exchange and the multigrid's seam faces
  are decided by them;
* ``comm`` offers the communicator calls the solver path makes
  (``Get_rank``, ``Get_size``, ``allreduce(x, op=MAX|MIN)``, ``Barrier``).
"""
from __future__ import annotations

from dataclasses import dataclass

from .config import CaseConfig

NPL = 3  # ghost layers per side (reference topology.py:15)

MAX = "max"   # reduction ops of Comm.allreduce (the reference's MPI.MAX / MPI.MIN)
MIN = "min"


class SingleRankComm:
    """The communicator calls the solver path makes, at one rank."""

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def allreduce(self, x, op=None):
        return x

    def Barrier(self):
        return None


class DistComm:
    """The same calls over the default torch.distributed process group.
    Scalars travel as one float64 tensor on ``device`` (the GPU for NCCL,
    the CPU for gloo)."""

    def __init__(self, device="cpu"):
        import torch.distributed as dist
        self._dist = dist
        self.device = device

    def Get_rank(self):
        return self._dist.get_rank()

    def Get_size(self):
        return self._dist.get_world_size()

    def allreduce(self, x, op=None):
        import torch
        d = self._dist
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        d.all_reduce(t, op=d.ReduceOp.MIN if op == MIN else d.ReduceOp.MAX)
        return float(t.item())

    def Barrier(self):
        self._dist.barrier()


@dataclass
class Topology:
    rank: int
    nranks: int
    comm: object
    sd: tuple
    coords: tuple
    neighbors: dict
    local_ncells: tuple
    global_offsets: tuple


def rank_to_coords(rank: int, sd: tuple) -> tuple:
    """x-fastest sub-domain ordering (reference topology.py:56-61)."""
    return (rank % sd[0], (rank // sd[0]) % sd[1], rank // (sd[0] * sd[1]))


def cart_neighbors(rank: int, sd: tuple) -> dict:
    """(low, high) neighbour ranks per axis of a non-periodic MPI cartesian
    communicator over sd (row-major rank order); -1 past an end."""
    c = [rank // (sd[1] * sd[2]), (rank // sd[2]) % sd[1], rank % sd[2]]
    out = {}
    for axis, name in enumerate("xyz"):
        pair = []
        for step in (-1, 1):
            cc = list(c)
            cc[axis] += step
            ok = 0 <= cc[axis] < sd[axis]
            pair.append((cc[0] * sd[1] + cc[1]) * sd[2] + cc[2] if ok else -1)
        out[name] = tuple(pair)
    return out


def _dist_backend():
    try:
        import torch.distributed as dist
    except ImportError:
        return None
    if dist.is_available() and dist.is_initialized():
        return dist
    return None


def build_topology(cfg: CaseConfig) -> Topology:
    sd = tuple(int(m) for m in cfg.mpi.domains)
    want = sd[0] * sd[1] * sd[2]
    gn = (cfg.grid.nx, cfg.grid.ny, cfg.grid.nz)
    if want == 1:
        return Topology(rank=0, nranks=1, comm=SingleRankComm(), sd=sd,
                        coords=(0, 0, 0),
                        neighbors={"x": (-1, -1), "y": (-1, -1), "z": (-1, -1)},
                        local_ncells=gn, global_offsets=(0, 0, 0))
    dist = _dist_backend()
    nranks = dist.get_world_size() if dist is not None else 1
    if nranks != want:
        raise ValueError(f"mpi.domains {sd} implies {want} ranks, "
                         f"but mpirun launched {nranks}")
    rank = dist.get_rank()
    dev = "cpu"
    if dist.get_backend() == "nccl":
        import torch
        dev = "cuda:%d" % torch.cuda.current_device()
    coords = rank_to_coords(rank, sd)
    local = tuple(g // s for g, s in zip(gn, sd))
    offsets = tuple(c * n for c, n in zip(coords, local))
    return Topology(rank=rank, nranks=nranks, comm=DistComm(dev), sd=sd, coords=coords,
                    neighbors=cart_neighbors(rank, sd), local_ncells=local,
                    global_offsets=offsets)
