"""Ghost-layer fills of the lid-driven cavity (reference warpflow/bcs.py),
run by libwfb200's ordered fill kernels.

Only the cavity combination exists (walls W/E/B, slip S/N, moving lid on
top); anything else raises the reference's ValueError (bcs.py:173-184).
"""
from __future__ import annotations

import torch

from . import _abi
from .topology import NPL

_CAVITY = {"west": "wall", "east": "wall", "south": "slip", "north": "slip",
           "bottom": "wall", "top": "moving_lid"}


def _stream(dev):
    return _abi.ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


class BoundaryKernels:
    """Reference bcs.py:166-323 interface: apply_u/v/w/vis/pbound/p_mirror
    and the initial ``apply``; arguments are DeviceFields."""

    def __init__(self, bnd, device):
        self.device = device
        self.bnd = dict(bnd)
        if any(self.bnd.get(k) != v for k, v in _CAVITY.items()):
            raise ValueError("unsupported boundary combination for the Hydro3D "
                             "benchmark port: %s" % self.bnd)

    def _s(self, fld):
        return _stream(fld.t.device)

    def apply_u(self, fld, n, ulid, alfabc=1):
        _abi.call("wf_fill_u", fld.ptr, n, float(ulid), self._s(fld))

    def apply_v(self, fld, n, alfabc=1):
        _abi.call("wf_fill_v", fld.ptr, n, self._s(fld))

    def apply_w(self, fld, n, alfabc=1):
        _abi.call("wf_fill_w", fld.ptr, n, self._s(fld))

    def apply_vis(self, fld, n, rrey):
        _abi.call("wf_fill_vis", fld.ptr, n, float(rrey), self._s(fld))

    def apply_pbound(self, fld, n):
        _abi.call("wf_fill_pbound", fld.ptr, n, self._s(fld))

    def apply_p_mirror(self, fld, n, npl=NPL):
        _abi.call("wf_fill_p_mirror", fld.ptr, n, self._s(fld))

    def apply(self, fields, ncells, ulid, npl=NPL):
        n = ncells[0]
        if "u" in fields:
            self.apply_u(fields["u"], n, ulid, 1)
        if "v" in fields:
            self.apply_v(fields["v"], n, 1)
        if "w" in fields:
            self.apply_w(fields["w"], n, 1)
        if "p" in fields:
            self.apply_p_mirror(fields["p"], n, npl)
