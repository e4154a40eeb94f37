"""The allocation-free multigrid solve (wf_mg_solve_noalloc).

Callers such as a host flow solver that owns every GPU buffer in its own
fixed pool cannot let this library allocate.  wf_mg_solve_noalloc serves
them with the coarse multigrid levels in a fixed array inside the library.
This test calls it through the C ABI, twice in a row with different
right-hand sides, and checks each result against the regular entry point
wf_mg_solve (whose level buffers the caller allocates), within the same
tolerance as the other multigrid tests, and reads the call's device status
word (no bounded wait may have given up).  It also checks the size limit.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _regular_solve(mg, su, pp):
    mg.solve(su, pp, 3)
    torch.cuda.synchronize()
    return pp.numpy()


# (112, 3) fills the static array almost to its end; (16, 1) runs the 300
# coarse sweeps on level 0 itself
@pytest.mark.parametrize("n,levels", [(32, 3), (80, 3), (112, 3), (16, 1)])
def test_noalloc_matches_regular_solve_twice(n, levels):
    from helpers import make_cfg
    from warpflow import Multigrid, _abi, build_topology
    from warpflow.fields import DeviceField

    lib = _abi.load()
    cfg = make_cfg(n=n, levels=levels)
    h = 1.0 / n
    mg = Multigrid(cfg, build_topology(cfg), "cuda:0", h, h, h)
    shape = (n + 6,) * 3
    su = DeviceField.zeros(shape, "cuda:0")
    pp_ref = DeviceField.zeros(shape, "cuda:0")
    pp_new = DeviceField.zeros(shape, "cuda:0")
    rng = np.random.default_rng(7)
    for call in range(2):
        rhs = rng.standard_normal(shape)
        su.assign(rhs)
        ref = _regular_solve(mg, su, pp_ref)
        pp_new.assign(rng.standard_normal(shape))  # must be overwritten
        rc = lib.wf_mg_solve_noalloc(su.ptr, pp_new.ptr, n, levels, h, h, h, _stream())
        assert rc == 0, lib.wf_last_error()
        status = ctypes.c_int32(-1)
        assert lib.wf_mg_noalloc_status(_stream(), ctypes.byref(status)) == 0
        assert status.value == _abi.ST_OK, status.value
        torch.cuda.synchronize()
        got = pp_new.numpy()
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 1e-12 * scale, (call, np.abs(got - ref).max())


def test_noalloc_rejects_oversize():
    from warpflow import _abi
    lib = _abi.load()
    n = 128
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    rc = lib.wf_mg_solve_noalloc(dummy.data_ptr(), dummy.data_ptr(), n, 3, 1.0 / n,
                                 1.0 / n, 1.0 / n, _stream())
    assert rc == 1
    assert b"multigrid scratch" in lib.wf_last_error()
