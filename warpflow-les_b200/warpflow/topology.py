"""Domain decomposition, single-rank form.

The B200 build runs one case per GPU, so the topology is always one rank
owning the whole grid.  ``build_topology`` returns the same ``Topology``
fields as the reference (warpflow/topology.py:18-53) with every neighbour a
physical boundary (-1) and ``comm`` a one-rank communicator, and rejects a
multi-domain ``mpi.domains`` the way the reference rejects a rank-count
mismatch.
"""
from __future__ import annotations

from dataclasses import dataclass

from .config import CaseConfig

NPL = 3  # ghost layers per side (reference topology.py:15)


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


def build_topology(cfg: CaseConfig) -> Topology:
    sd = tuple(int(m) for m in cfg.mpi.domains)
    want = sd[0] * sd[1] * sd[2]
    if want != 1:
        raise ValueError(f"mpi.domains {sd} implies {want} ranks, but this build "
                         "runs one rank per case (set mpi.domains: [1, 1, 1])")
    ncell = (cfg.grid.nx, cfg.grid.ny, cfg.grid.nz)
    return Topology(rank=0, nranks=1, comm=SingleRankComm(), sd=sd,
                    coords=(0, 0, 0),
                    neighbors={"x": (-1, -1), "y": (-1, -1), "z": (-1, -1)},
                    local_ncells=ncell, global_offsets=(0, 0, 0))
