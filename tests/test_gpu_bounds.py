"""The bounds-checked build (libuassa_debug.so, -DUA_BOUNDS_CHECK) runs the uv and uvh assembly,
the Newton solves with the node-slice PCG and the served loop without recording a single index
outside its range: connectivity node ids below Nnodes, patch element ids below Nele, contribution
elements inside their patch, tangent and residual indices inside their system.  Each case runs in
a child process that loads the debug library instead of the release one."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEBUG_LIB = os.path.join(ROOT, "uasource_b200", "libuassa_debug.so")

CHILD = r'''
import ctypes as C, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import uasource_b200 as ua
from uasource_b200 import lib as L, synth
assert L.LIB_PATH.endswith("libuassa_debug.so")
out = {}

def flag(mua):
    en, site, idx = C.c_int32(), C.c_int32(), C.c_int64()
    L.check(L.load().ua_debug_bounds(mua.handle, C.byref(en), C.byref(site), C.byref(idx)))
    return en.value, site.value, idx.value

for nod, nx, ny in ((3, 41, 21), (6, 13, 7)):
    P = synth.ice_stream_shelf(nx, ny, nod=nod, seed=1, transient=True)
    m = ua.CreateMUA(P.coordinates, P.connectivity)
    for prec in (L.UA_PREC_FP64, L.UA_PREC_MIXED):
        ctrl = ua.CtrlVar(precision=prec, krylov_rtol=1e-6 if prec else 1e-12).set_force_tolerance(1e-20)
        Fo, _, _, _, info = ua.uv(ctrl, m, ua.BCs.from_problem(P), ua.Fields.from_problem(P))
    out[f"uv{nod}"] = flag(m)
    m3 = ua.CreateMUA(P.coordinates, P.connectivity, ndof=3)
    F0 = ua.Fields.from_problem(P)
    F0.ub, F0.vb = Fo.ub, Fo.vb
    b = ua.BCs.from_problem(P)
    hb = ua.HBCs(ubFixedNode=b.ubFixedNode, ubFixedValue=b.ubFixedValue, vbFixedNode=b.vbFixedNode,
                 vbFixedValue=b.vbFixedValue)
    _, _, info = ua.uvh(ua.CtrlVar().set_force_tolerance(1e-20), m3, F0, F0.copy(), hb, 0.1)
    out[f"uvh{nod}"] = flag(m3)
probs = [synth.ice_stream_shelf(15, 8, seed=0), synth.ice_stream_shelf(31, 16, seed=3)]
mb = ua.CreateMUABatch([(P.coordinates, P.connectivity) for P in probs])
ua.uv_batch(ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20), mb,
            [ua.Fields.from_problem(P) for P in probs], [ua.BCs.from_problem(P) for P in probs])
out["batch"] = flag(mb)
print(json.dumps(out))
'''


def test_no_index_leaves_its_range_in_the_bounds_checked_build():
    if not os.path.exists(DEBUG_LIB):
        pytest.fail("libuassa_debug.so is missing: build it with `make -C uasource_b200/csrc debug`")
    env = dict(os.environ, UASOURCE_B200_LIBRARY=DEBUG_LIB)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], capture_output=True, text=True, env=env, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    for case, (enabled, site, index) in res.items():
        assert enabled == 1, case
        assert site == 0, f"{case}: bounds violation at site {site}, index {index}"
