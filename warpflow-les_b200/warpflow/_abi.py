"""ctypes binding of libwfb200.so (declared in include/warpflow_b200.h).

The library is built in-tree by ``warpflow-les_b200/build.py``.  There is no
fallback: if the library is missing every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

NPL = 3
MAX_LEVELS = 8
NFIELDS = 13
FIELD_NAMES = ("u", "v", "w", "p", "ustar", "vstar", "wstar", "uoo", "voo",
               "woo", "vis", "su", "pp")

ST_OK, ST_DT_COLLAPSE, ST_DIVERGED, ST_NOT_CONVERGED, ST_WAIT_TIMEOUT = range(5)

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libwfb200.so")


class WfScalars(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_double),
        ("ctime", ctypes.c_double),
        ("rmax", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("dtmax", ctypes.c_double),
        ("umax", ctypes.c_double),
        ("vmax", ctypes.c_double),
        ("wmax", ctypes.c_double),
        ("dtvisc", ctypes.c_double),
        ("rrey", ctypes.c_double),
        ("ulid", ctypes.c_double),
        ("rmax_trace", ctypes.c_double * 32),
        ("red", ctypes.c_uint64 * 6),
        ("itime", ctypes.c_int32),
        ("iters", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("loop", ctypes.c_int32),
        ("ticket", ctypes.c_uint32),
        ("nmg", ctypes.c_int32),
        ("gbar", ctypes.c_uint32 * 2),
        ("bticket", ctypes.c_uint32),
        ("bflags", ctypes.c_int32),
    ]


class WfCase(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("nlev", ctypes.c_int32),
        ("sgs", ctypes.c_int32),
        ("variable_dt", ctypes.c_int32),
        ("maxcy", ctypes.c_int32),
        ("mg_fp32", ctypes.c_int32),
        ("n_pre", ctypes.c_int32),
        ("n_post", ctypes.c_int32),
        ("n_coarse", ctypes.c_int32),
        ("n_vcycles", ctypes.c_int32),
        ("dx", ctypes.c_double),
        ("dy", ctypes.c_double),
        ("dz", ctypes.c_double),
        ("rrey", ctypes.c_double),
        ("cw", ctypes.c_double),
        ("ulid", ctypes.c_double),
        ("dt_growth", ctypes.c_double),
        ("safety", ctypes.c_double),
        ("eps", ctypes.c_double),
        ("fld", ctypes.c_void_p * NFIELDS),
        ("mg_phi", ctypes.c_void_p * MAX_LEVELS),
        ("mg_rhs", ctypes.c_void_p * MAX_LEVELS),
        ("mg_tmp", ctypes.c_void_p * MAX_LEVELS),
        ("sc", ctypes.c_void_p),
        ("mg_cop", ctypes.c_void_p),
        ("mg_cop_part", ctypes.c_void_p),
    ]


_VP = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double
_CP = ctypes.POINTER(WfCase)

# name -> (restype, argtypes); every symbol include/warpflow_b200.h declares
SIGNATURES = {
    "wf_version": (_I32, []),
    "wf_last_error": (ctypes.c_char_p, []),
    "wf_struct_sizes": (_I32, [ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    "wf_scalars_init": (_I32, [_VP, _D, _D, _D, _VP]),
    "wf_set_coarse_strategy": (_I32, [_I32, _I32, _I32]),
    "wf_set_launch_shape": (_I32, [_I32, _I32, _I32, _I32, _I32]),
    "wf_launch_shape": (_I32, [_I32, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_I32),
                               ctypes.POINTER(_I32)]),
    "wf_set_bucket_cap": (_I32, [_I32, _I32, _I32]),
    "wf_bucket_cap": (_I32, [_I32, _I32, ctypes.POINTER(_I32)]),
    "wf_mg_level_elems": (_I32, [_I32, _I32, _I32, ctypes.POINTER(ctypes.c_int64)]),
    "wf_mg_coarse_op_elems": (_I32, [_CP, ctypes.POINTER(ctypes.c_int64),
                                     ctypes.POINTER(ctypes.c_int64)]),
    "wf_mg_build_coarse_op": (_I32, [_CP, _VP]),
    "wf_mg_coarse_solve": (_I32, [_CP, _VP, _VP, _VP]),
    "wf_init_noise": (_I32, [_VP, _VP, _VP, _I32, _D, _I32, _VP]),
    "wf_fill_initial": (_I32, [_CP, _VP]),
    "wf_fill_u": (_I32, [_VP, _I32, _D, _VP]),
    "wf_fill_v": (_I32, [_VP, _I32, _VP]),
    "wf_fill_w": (_I32, [_VP, _I32, _VP]),
    "wf_fill_vis": (_I32, [_VP, _I32, _D, _VP]),
    "wf_fill_pbound": (_I32, [_VP, _I32, _VP]),
    "wf_fill_p_mirror": (_I32, [_VP, _I32, _VP]),
    "wf_conv": (_I32, [_CP, _I32, _D, _VP, _VP]),
    "wf_diff": (_I32, [_CP, _I32, _D, _VP, _VP]),
    "wf_calvel": (_I32, [_CP, _D, _VP, _VP]),
    "wf_calmas": (_I32, [_CP, _VP]),
    "wf_wale_vis": (_I32, [_CP, _VP]),
    "wf_checkdt": (_I32, [_CP, _VP]),
    "wf_add_ring": (_I32, [_VP, _VP, _I32, _VP]),
    "wf_mg_solve": (_I32, [_CP, _VP]),
    "wf_mg_solve_noalloc": (_I32, [_VP, _VP, _I32, _I32, _D, _D, _D, _VP]),
    "wf_mg_noalloc_status": (_I32, [_VP, ctypes.POINTER(_I32)]),
    "wf_wait_probe": (_I32, [_VP, _VP, _I32, _I32, _VP]),
    "wf_mg_solve_bucket": (_I32, [_CP, _I32, _VP, _VP]),
    "wf_mg_bucket_table_bytes": (_I32, [_I32, ctypes.POINTER(ctypes.c_int64)]),
    "wf_mg_vcycle": (_I32, [_CP, _VP, _VP, _VP]),
    "wf_mg_relax": (_I32, [_CP, _VP, _VP, _I32, _VP]),
    "wf_mg_dc_cycle": (_I32, [_CP, _VP, _VP, _VP]),
    "wf_mg_residual_max": (_I32, [_CP, _VP, _VP, _VP, _VP]),
    "wf_mg_refill": (_I32, [_CP, _VP, _VP]),
    "wf_box_copy": (_I32, [_VP, _I64, _I64, _I32, _I32, _I32, _I32, _I32, _I32, _VP, _I32,
                           _VP]),
    "wf_copy_oo": (_I32, [_CP, _VP]),
    "wf_fill_program": (_I32, [_I32, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_I32),
                               ctypes.POINTER(_I64), _VP, _VP]),
    "wf_rk_mg_op": (_I32, [_CP, _I32, _I32, _I32, _I32, _VP]),
    "wf_rk_level_view": (_I32, [_CP, _I32, ctypes.POINTER(_VP), ctypes.POINTER(_I64),
                                ctypes.POINTER(_I64), ctypes.POINTER(_I32)]),
    "wf_stepper_create": (_I32, [_CP, _I32, ctypes.POINTER(_VP)]),
    "wf_stepper_step": (_I32, [_VP, _VP]),
    "wf_stepper_destroy": (_I32, [_VP]),
    "wf_ensemble_create": (_I32, [_CP, _I32, _I32, ctypes.POINTER(_VP)]),
    "wf_ensemble_step": (_I32, [_VP, _VP]),
    "wf_ensemble_destroy": (_I32, [_VP]),
    "wf_ensemble_layout": (_I32, [_VP, ctypes.POINTER(_I32), ctypes.POINTER(_I32),
                                  ctypes.POINTER(_I32)]),
    "wf_stepper_launch_counts": (_I32, [_VP, ctypes.POINTER(_I32)]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libwfb200.so and bind every entry point (raises if missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            "libwfb200.so not found at %s: build it with "
            "`python warpflow-les_b200/build.py` (there is no CPU fallback)" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    s, c = ctypes.c_int64(), ctypes.c_int64()
    lib.wf_struct_sizes(ctypes.byref(s), ctypes.byref(c))
    if s.value != ctypes.sizeof(WfScalars) or c.value != ctypes.sizeof(WfCase):
        raise RuntimeError("libwfb200.so struct layout mismatch (%d/%d vs %d/%d)"
                           % (s.value, c.value, ctypes.sizeof(WfScalars),
                              ctypes.sizeof(WfCase)))
    _lib = lib
    return lib


def check(rc: int, what: str = ""):
    if rc != 0:
        msg = load().wf_last_error().decode(errors="replace")
        raise RuntimeError("libwfb200 %s failed (code %d): %s" % (what, rc, msg))


def call(name: str, *args):
    rc = getattr(load(), name)(*args)
    check(rc, name)
    return rc
