"""Bounded device-side waits give up, report, and leave the context usable.

The cooperative relax waits on a grid barrier and the point-to-point coarse
kernels wait on mbarriers that their neighbours complete.  Every such wait
is bounded: after its limit it records WF_ST_WAIT_TIMEOUT and the kernel
returns.  ``wf_wait_probe`` runs each of those waits once in a form that
can never complete (a barrier declared one block larger than the launch, an
mbarrier expecting bytes that nobody sends) with a short limit; the tests
check that the call returns quickly, that the status word says so, that the
solver raises its error from that status, and that later work still runs.
No GPU fault or hang is involved: nothing waits without a limit.
"""
import ctypes
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TRIES = 1 << 14


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("kind", [0, 1], ids=["grid_barrier", "mbarrier"])
def test_wait_gives_up_and_records_timeout(kind):
    from warpflow import _abi
    lib = _abi.load()
    gbar = torch.zeros(2, dtype=torch.int32, device="cuda:0")
    err = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    assert lib.wf_wait_probe(gbar.data_ptr(), err.data_ptr(), kind, TRIES, _stream()) == 0, \
        lib.wf_last_error()
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    assert int(err.item()) == _abi.ST_WAIT_TIMEOUT
    assert elapsed < 5.0, elapsed
    # the context still works after the timed-out wait
    x = torch.arange(1000, dtype=torch.float64, device="cuda:0")
    assert float(x.sum().item()) == 499500.0


def test_probe_rejects_bad_arguments():
    from warpflow import _abi
    lib = _abi.load()
    buf = torch.zeros(2, dtype=torch.int32, device="cuda:0")
    assert lib.wf_wait_probe(buf.data_ptr(), buf.data_ptr(), 2, TRIES, _stream()) == 1
    assert lib.wf_wait_probe(buf.data_ptr(), buf.data_ptr(), 0, 0, _stream()) == 1
    assert lib.wf_wait_probe(None, buf.data_ptr(), 0, TRIES, _stream()) == 1


def test_solver_raises_on_a_timed_out_wait():
    """A wait that gave up inside a step leaves WF_ST_WAIT_TIMEOUT in the
    case's scalar block; the solver turns it into its error."""
    from helpers import make_cfg
    from warpflow import FlowSolver, _abi, build_topology
    cfg = make_cfg(n=16, levels=3)
    sol = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    sol.step()
    gbar = torch.zeros(2, dtype=torch.int32, device="cuda:0")
    status = sol._sc.data_ptr() + _abi.WfScalars.status.offset
    lib = _abi.load()
    assert lib.wf_wait_probe(gbar.data_ptr(), status, 0, TRIES, _stream()) == 0
    with pytest.raises(RuntimeError, match="device-side wait timed out"):
        sol.finish_step()
    # the device stays usable: a fresh solver steps normally
    sol2 = FlowSolver(cfg, build_topology(cfg), "cuda:0")
    info = sol2.step()
    assert info["rmax"] < 1e-6
    assert np.isfinite(sol2.f["u"].numpy()).all()
