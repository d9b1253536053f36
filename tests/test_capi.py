"""The C-ABI library loads, exports every symbol of include/ua_ssa.h, and its
struct layout matches the ctypes binding (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np

from uasource_b200 import lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "ua_ssa.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ua_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = _declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
        assert n in L.SIGNATURES, f"{n} has no ctypes signature"


def test_struct_layout_matches_binding():
    lib = L.load()
    sizes = np.zeros(7, np.int64)
    assert lib.ua_struct_sizes(L.lptr(sizes), 7) == 0
    ours = [C.sizeof(t) for t in (L.ua_mesh_desc, L.ua_params, L.ua_fields, L.ua_bcs, L.ua_newton_iter,
                                  L.ua_newton_report, L.ua_tune_report)]
    assert list(sizes) == ours


def test_params_default_matches_reference_defaults():
    from uasource_b200 import CtrlVar
    p = L.ua_params()
    L.load().ua_params_default(C.byref(p))
    cv = CtrlVar()
    for name, _ in L.ua_params._fields_:
        a, b = getattr(p, name), getattr(cv, name)
        if isinstance(b, tuple):
            assert tuple(a) == b, name
        elif name == "SlidingLaw":
            assert a == L.SLIDING_LAWS[b], name
        else:
            assert a == b, name


def test_no_device_reports_error_not_crash():
    lib = L.load()
    if lib.ua_device_count() > 0:
        return
    coords = np.zeros((3, 2)); coords[1, 0] = 1; coords[2, 1] = 1
    conn = np.array([[0, 2, 1]], np.int32)
    d = L.ua_mesh_desc(3, 1, 3, 0, L.dptr(np.asfortranarray(coords).ravel(order="F")), L.iptr(conn.ravel()))
    h = C.c_void_p()
    rc = lib.ua_mesh_create(C.byref(d), 2, 0, C.byref(h))
    assert rc == L.UA_ERR_NO_DEVICE
    assert b"device" in lib.ua_last_error()
