"""CPU stand-in for the parts of NVIDIA Warp (warp-lang >= 1.18) that the
reference solver uses, so the reference's own kernel source can run here
unmodified to produce golden vectors.

Test infrastructure only: the generator script in this folder puts it on
sys.path ahead of the reference package; nothing in the product imports it.

Semantics restated from Warp's documented execution model:
  * ``wp.launch(k, dim, inputs)`` runs the kernel body once per index of the
    launch grid; ``wp.tid()`` returns that index (a tuple for 2-D/3-D grids).
    Threads are run one after another in row-major order.  Every kernel in
    the reference writes each output element from exactly one thread and
    reads only elements no other thread of the same launch writes (RBGS
    updates one colour per launch), so the serial order gives the same
    result as any parallel schedule.
  * scalar types: ``float64`` is IEEE double, ``uint32`` wraps modulo 2**32
    (numpy uint32 scalars), ``int32`` is a Python int.
  * ``atomic_max`` / ``atomic_min`` are order-independent max/min.
  * arrays are C-ordered numpy buffers with ``numpy/assign/zero_/fill_``.
"""
import math
import warnings

import numpy as np

warnings.filterwarnings("ignore", category=RuntimeWarning,
                        message="overflow encountered")

float64 = np.float64
float32 = np.float32
uint32 = np.uint32


def int32(x):
    return int(x)


_TID = (0,)


def init():
    return None


def is_cuda_available():
    return False


class _ArrayType:
    def __init__(self, dtype=None, ndim=1):
        self.dtype = dtype
        self.ndim = ndim


def array(dtype=None, ndim=1):
    return _ArrayType(dtype, ndim)


def array3d(dtype=None):
    return _ArrayType(dtype, 3)


def func(f):
    return f


class Kernel:
    def __init__(self, f):
        self.f = f
        self.key = f.__name__


def kernel(f=None, **_kw):
    if f is None:
        return lambda g: Kernel(g)
    return Kernel(f)


def tid():
    return _TID if len(_TID) > 1 else _TID[0]


def where(c, a, b):
    return a if c else b


def abs(x):  # noqa: A001 - mirrors wp.abs
    return np.float64(math.fabs(x))


def pow(x, y):  # noqa: A001 - mirrors wp.pow
    return np.float64(math.pow(float(x), float(y)))


def atomic_max(arr, idx, val):
    if val > arr[idx]:
        arr[idx] = val


def atomic_min(arr, idx, val):
    if val < arr[idx]:
        arr[idx] = val


class ShimArray:
    def __init__(self, data):
        self.data = data

    @property
    def shape(self):
        return self.data.shape

    def numpy(self):
        return self.data

    def assign(self, src):
        self.data[...] = np.asarray(src, dtype=self.data.dtype)

    def zero_(self):
        self.data[...] = 0

    def fill_(self, v):
        self.data[...] = v


def zeros(shape, dtype=np.float64, device=None):
    if isinstance(shape, int):
        shape = (shape,)
    return ShimArray(np.zeros(shape, dtype=np.float64))


def empty(shape, dtype=np.float64, device=None):
    return zeros(shape, dtype, device)


def copy(dst, src):
    dst.data[...] = src.data


def _unwrap(x):
    return x.data if isinstance(x, ShimArray) else x


def launch(kernel, dim, inputs=(), device=None):
    global _TID
    if isinstance(dim, int):
        dim = (dim,)
    args = [_unwrap(a) for a in inputs]
    f = kernel.f
    for idx in np.ndindex(*dim):
        _TID = tuple(int(v) for v in idx)
        f(*args)
