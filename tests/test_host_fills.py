"""The composed one-launch ghost fills, checked on the CPU: each fill
kind's program (wf_fill_program), applied as the device applies it (every
entry reads the values from before the fill), must reproduce the reference's
ordered face launches (the oracle's fills, pinned to the reference's own
source) bit for bit, signed zeros included."""
import ctypes

import numpy as np
import pytest

from oracle import wf_oracle as O

KINDS = {0: "u", 1: "v", 2: "w", 3: "vis", 4: "pbound", 5: "pmirror"}


def _program(kind, n):
    from warpflow import _abi
    lib = _abi.load()
    ns, ng, ne = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
    assert lib.wf_fill_program(kind, n, ctypes.byref(ns), ctypes.byref(ng), ctypes.byref(ne),
                               None, None) == 0, lib.wf_last_error()
    ent = np.zeros(2 * ne.value, dtype=np.int32)
    gs = np.zeros(ng.value + 1, dtype=np.int32)
    assert lib.wf_fill_program(kind, n, ctypes.byref(ns), ctypes.byref(ng), ctypes.byref(ne),
                               ent.ctypes.data, gs.ctypes.data) == 0
    return ns.value, ng.value, ent.reshape(-1, 2), gs


def _apply(f, ent, K):
    old = f.ravel().copy()
    out = f.ravel().copy()
    dst, code = ent[:, 0].astype(np.int64), ent[:, 1].astype(np.int64)
    cst = (code & 1) == 1
    src = code >> 2
    val = np.where(cst, np.where(src == 0, 0.0, K), old[np.where(cst, 0, src)])
    val = np.where((code & 2) != 0, -val, val)
    out[dst] = val
    return out.reshape(f.shape)


def _reference(kind, f, n, K):
    if kind == 0:
        O.apply_u(f, n, K)
    elif kind == 1:
        O.apply_v(f, n)
    elif kind == 2:
        O.apply_w(f, n)
    elif kind == 3:
        O.apply_vis(f, n, K)
    elif kind == 4:
        O.apply_pbound(f, n)
    else:
        O.apply_p_mirror(f, n)


@pytest.mark.parametrize("n", [4, 5, 8, 13, 24])
@pytest.mark.parametrize("kind", sorted(KINDS))
def test_one_launch_fill_equals_ordered_faces(kind, n):
    ns, ng, ent, gs = _program(kind, n)
    assert gs[0] == 0 and gs[-1] == len(ent) - ns and (np.diff(gs) <= 16).all()
    dst = ent[:, 0]
    assert len(np.unique(dst)) == len(dst)          # every cell written once
    # a simple entry never reads a cell the program writes
    written = set(dst.tolist())
    code = ent[:ns, 1]
    srcs = (code >> 2)[(code & 1) == 0]
    assert not (set(srcs.tolist()) & written)
    # a group reads no cell that another group or a simple entry writes
    owner = {int(d): -1 for d in dst[:ns]}
    for g in range(ng):
        for d in dst[ns + gs[g]:ns + gs[g + 1]]:
            owner[int(d)] = g
    for g in range(ng):
        for c in ent[ns + gs[g]:ns + gs[g + 1], 1]:
            if (c & 1) == 0 and int(c >> 2) in owner:
                assert owner[int(c >> 2)] == g
    rng = np.random.default_rng(kind * 100 + n)
    P = n + 6
    for trial in range(3):
        f = rng.standard_normal((P, P, P))
        if trial == 2:   # signed zeros must come out as the faces leave them
            f[rng.random(f.shape) < 0.3] = 0.0
        K = 0.75 if trial != 1 else 0.0
        want = f.copy()
        _reference(kind, want, n, K)
        got = _apply(f, ent, K)
        assert np.array_equal(got.view(np.int64), want.view(np.int64)), (kind, n, trial)
