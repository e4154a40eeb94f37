"""The C ABI library loads on a CPU-only machine and exports every symbol
that include/*.h declares; the ctypes struct layouts match the compiled ones.
No compute call is made."""
import ctypes
import glob
import os
import re

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(wf_\w+)\s*\(", src, re.M):
            names.add(m.group(1))
    return names


def test_library_exports_declared_symbols():
    from warpflow import _abi
    lib = _abi.load()
    decl = _declared()
    assert len(decl) >= 25, decl
    missing = [n for n in sorted(decl) if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding binds exactly the declared set
    assert set(_abi.SIGNATURES) == decl, set(_abi.SIGNATURES) ^ decl


def test_struct_layouts_match():
    from warpflow import _abi
    lib = _abi.load()
    s, c = ctypes.c_int64(), ctypes.c_int64()
    assert lib.wf_struct_sizes(ctypes.byref(s), ctypes.byref(c)) == 0
    assert s.value == ctypes.sizeof(_abi.WfScalars)
    assert c.value == ctypes.sizeof(_abi.WfCase)


def test_level_sizes_and_errors():
    from warpflow import _abi
    lib = _abi.load()
    e = ctypes.c_int64()
    assert lib.wf_mg_level_elems(80, 3, 2, ctypes.byref(e)) == 0
    assert e.value == 22 ** 3
    assert lib.wf_mg_level_elems(80, 3, 3, ctypes.byref(e)) != 0
    assert b"bad level" in lib.wf_last_error()


def test_validation_rejects_bad_case_without_gpu():
    """Argument validation happens on the host before any CUDA call."""
    from warpflow import _abi
    lib = _abi.load()
    c = _abi.WfCase()
    c.n = 10
    c.nlev = 3   # 10 is not divisible by 4
    st = ctypes.c_void_p()
    assert lib.wf_stepper_create(ctypes.byref(c), 0, ctypes.byref(st)) == 1
    assert b"divisible" in lib.wf_last_error()
    assert not st.value
