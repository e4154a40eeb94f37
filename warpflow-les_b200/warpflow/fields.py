"""Device arrays of the solver: float64 CUDA tensors (owned by torch) with
the small array interface the reference's fields expose (``numpy``,
``assign``, ``zero_``, ``fill_``, ``shape``; reference solver.py:47-48,
tests/test_cavity.py:78-104, tests/test_mg.py:17-21,45)."""
from __future__ import annotations

import numpy as np
import torch


def cuda_device(device) -> torch.device:
    """Resolve a reference-style device string; only CUDA devices exist
    here (the product path has no CPU fallback)."""
    dev = torch.device(device if device not in (None, "auto") else "cuda:0")
    if dev.type != "cuda":
        raise RuntimeError(
            "warpflow (B200 build) runs on CUDA devices only; got device=%r" % (device,))
    if not torch.cuda.is_available():
        raise RuntimeError("warpflow (B200 build): no CUDA device is visible")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


class DeviceField:
    """A contiguous CUDA tensor plus the reference array methods."""

    __slots__ = ("t",)

    def __init__(self, t: torch.Tensor):
        assert t.is_cuda and t.is_contiguous()
        self.t = t

    @classmethod
    def zeros(cls, shape, device, dtype=torch.float64):
        return cls(torch.zeros(tuple(shape), dtype=dtype, device=device))

    @property
    def shape(self):
        return tuple(self.t.shape)

    @property
    def ptr(self) -> int:
        return self.t.data_ptr()

    def numpy(self) -> np.ndarray:
        torch.cuda.current_stream(self.t.device).synchronize()
        return self.t.cpu().numpy()

    def assign(self, src):
        src = np.ascontiguousarray(np.asarray(src), dtype=np.float64
                                   if self.t.dtype == torch.float64 else np.float32)
        if src.shape != self.shape:
            raise ValueError("assign: shape %s != %s" % (src.shape, self.shape))
        self.t.copy_(torch.from_numpy(src))

    def zero_(self):
        self.t.zero_()

    def fill_(self, value):
        self.t.fill_(value)

    def __repr__(self):
        return "DeviceField(shape=%s, dtype=%s, device=%s)" % (
            self.shape, self.t.dtype, self.t.device)
