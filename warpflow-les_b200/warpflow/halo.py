"""Halo exchange between sub-domains (reference warpflow/halo.py).

``HaloExchanger(topo, device, npl).exchange(field, nl=None)`` fills the
ghost layers of a device field that face neighbouring ranks, axis by axis
(x, then y, then z): the ``nl`` real layers next to each seam are packed on
the device (``wf_box_copy``), sent to the neighbour, and the neighbour's
layers are unpacked into this side's ghosts.  Each slab spans the whole
array in the other two axes, ghosts included, so the y and z slabs carry
the x (and y) ghosts just received and edges and corners follow without
diagonal messages (halo.py:1-9).  Physical-boundary ghosts are untouched.

Transport is torch.distributed point-to-point: with NCCL the packed device
buffers go GPU to GPU over NVLink; with gloo they are staged through pinned
host buffers.  The low-side pair is exchanged before the high-side pair,
each pair as one grouped send/receive, as the reference's two Sendrecv
calls per axis (halo.py:111-130).
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi


class HaloExchanger:
    def __init__(self, topo, device, npl):
        import torch.distributed as dist
        self.topo = topo
        self.device = torch.device(device)
        self.npl = npl
        self._dist = dist
        self._nccl = dist.get_backend() == "nccl"
        self._bufs = {}   # element count -> (send, recv[, host send, host recv])

    def _buffers(self, count):
        b = self._bufs.get(count)
        if b is None:
            dev = [torch.empty(count, dtype=torch.float64, device=self.device) for _ in range(2)]
            host = [] if self._nccl else [torch.empty(count, dtype=torch.float64,
                                                      pin_memory=True) for _ in range(2)]
            b = self._bufs[count] = tuple(dev + host)
        return b

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def exchange(self, arr, nl=None):
        """Fill the neighbour-side ghost layers of a (C-contiguous) device
        field, all three axes (halo.py:81)."""
        A, B, C = arr.shape
        self.exchange_view(arr.ptr, B * C, C, (A, B, C), nl)

    def exchange_view(self, ptr, sI, sJ, shape, nl=None):
        """The same on a strided box: ring cell (0, 0, 0) at ``ptr``,
        strides (sI, sJ, 1), extent ``shape`` (a multigrid level inside a
        padded field)."""
        npl = self.npl
        nl = npl if nl is None else nl
        A, B, C = shape
        d = self._dist
        for axis in range(3):
            lo, hi = self.topo.neighbors["xyz"[axis]]
            if lo < 0 and hi < 0:
                continue
            n = shape[axis] - 2 * npl
            send_lo, send_hi = npl, npl + n - nl
            recv_lo, recv_hi = npl - nl, npl + n
            ext = [A, B, C]
            ext[axis] = nl
            count = ext[0] * ext[1] * ext[2]
            bufs = self._buffers(count)
            pairs = []
            if lo >= 0:
                pairs.append((lo, send_lo, recv_lo, 21, 22))
            if hi >= 0:
                pairs.append((hi, send_hi, recv_hi, 22, 21))
            for peer, so, ro, stag, rtag in pairs:
                org = [0, 0, 0]
                org[axis] = so
                _abi.call("wf_box_copy", ptr, sI, sJ, org[0], org[1], org[2], ext[0], ext[1],
                          ext[2], bufs[0].data_ptr(), 0, self._stream())
                if self._nccl:
                    snd, rcv = bufs[0], bufs[1]
                else:
                    bufs[2].copy_(bufs[0])          # waits for the pack
                    snd, rcv = bufs[2], bufs[3]
                ops = [d.P2POp(d.isend, snd, peer, tag=stag),
                       d.P2POp(d.irecv, rcv, peer, tag=rtag)]
                for req in d.batch_isend_irecv(ops):
                    req.wait()
                if not self._nccl:
                    bufs[1].copy_(bufs[3])              # before bufs[3] is reused
                org[axis] = ro
                _abi.call("wf_box_copy", ptr, sI, sJ, org[0], org[1], org[2], ext[0], ext[1],
                          ext[2], bufs[1].data_ptr(), 1, self._stream())
