"""warpflow (B200 build): drop-in replacement of the warpflow-les per-step
hot path -- the Heun RK2 stage and the multigrid projection -- running as
hand-written sm_100a CUDA kernels (libwfb200.so) behind the reference's
Python API (reference warpflow/__init__.py:9-14)."""
from .config import load_case
from .topology import build_topology, NPL
from .solver import FlowSolver
from .multigrid import Multigrid

__version__ = "0.1.0"
__all__ = ["load_case", "build_topology", "FlowSolver", "Multigrid", "NPL",
           "__version__"]
