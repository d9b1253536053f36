"""The allocation-free solve entry point matches the allocating one.

ua_solve_kape_symmetric_noalloc serves callers that cannot allocate device
memory themselves (a MEX working on gpuArray data, where MATLAB owns the
device allocator; a plugin whose host application forbids cudaMalloc on the
solve path): they pass device arrays they already hold, and the library runs
its temporaries out of a fixed static device array.  This test builds a real
uv tangent with its boundary-condition rows, solves it with the allocating
entry point ua_solve_kape_symmetric (host arrays), then calls the
allocation-free entry point twice in a row on device copies of the same
arrays through the C-ABI, and checks both results against the first within
the tolerance of the other solve tests.  It is named to run last.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import uasource_b200 as ua
from uasource_b200 import lib as L
from uasource_b200 import synth

pytestmark = pytest.mark.gpu
RTOL = 1e-9


def _system():
    P = synth.ice_stream_shelf(21, 11, nod=3, seed=0)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)
    rng = np.random.default_rng(11)
    F.ub = 1000 * rng.random(P.Nnodes)
    F.vb = 100 * rng.standard_normal(P.Nnodes)
    R, K = ua.uvMatrixAssembly(ua.CtrlVar(), mua, F)
    n = K.shape[0]
    dofs = np.concatenate([P.ubFixedNode, P.vbFixedNode + P.Nnodes]).astype(np.int64)
    vals = np.where(np.arange(dofs.size) % 3 == 0, 2.0, 1.0)  # a few scaled constraint rows
    B = sp.csr_matrix((vals, (np.arange(dofs.size), dofs)), shape=(dofs.size, n))
    g = rng.standard_normal(dofs.size)
    return K.tocsr(), B, -R, g, dofs, vals


def _noalloc(torch, K, dofs, vals, f, g):
    dev = torch.device("cuda", 0)
    rp = torch.tensor(K.indptr.astype(np.int32), device=dev)
    ci = torch.tensor(K.indices.astype(np.int32), device=dev)
    kv = torch.tensor(K.data, dtype=torch.float64, device=dev)
    ld = torch.tensor(dofs.astype(np.int32), device=dev)
    lv = torch.tensor(vals, dtype=torch.float64, device=dev)
    fd = torch.tensor(f, dtype=torch.float64, device=dev)
    gd = torch.tensor(g, dtype=torch.float64, device=dev)
    x = torch.full((K.shape[0],), np.nan, dtype=torch.float64, device=dev)
    y = torch.full((dofs.size,), np.nan, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    its = C.c_int32()
    rc = L.load().ua_solve_kape_symmetric_noalloc(K.shape[0], rp.data_ptr(), ci.data_ptr(), kv.data_ptr(),
                                                  dofs.size, ld.data_ptr(), lv.data_ptr(), fd.data_ptr(),
                                                  gd.data_ptr(), x.data_ptr(), y.data_ptr(), 1e-12, 0,
                                                  C.byref(its), 0)
    L.check(rc)
    torch.cuda.synchronize()
    return x.cpu().numpy(), y.cpu().numpy(), its.value


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    K, B, f, g, dofs, vals = _system()
    x_ref, y_ref, _ = ua.solveKApeSymmetric(K, B, f, g, rtol=1e-12)
    for _ in range(2):  # the scratch array keeps the previous call's contents
        x, y, its = _noalloc(torch, K, dofs, vals, f, g)
        assert its > 0
        assert np.linalg.norm(x - x_ref) <= RTOL * np.linalg.norm(x_ref)
        assert np.linalg.norm(y - y_ref) <= RTOL * np.linalg.norm(y_ref)


def test_noalloc_rejects_sizes_beyond_its_maximum():
    lib = L.load()
    its = C.c_int32()
    rc = lib.ua_solve_kape_symmetric_noalloc(131072 + 1, None, None, None, 0, None, None, None, None, None, None,
                                             1e-12, 0, C.byref(its), 0)
    assert rc == L.UA_ERR_INVALID
    assert b"UA_NOALLOC_MAX_ROWS" in lib.ua_last_error()
    rc = lib.ua_solve_kape_symmetric_noalloc(10, None, None, None, 16384 + 1, None, None, None, None, None, None,
                                             1e-12, 0, C.byref(its), 0)
    assert rc == L.UA_ERR_INVALID
    assert b"UA_NOALLOC_MAX_CONSTRAINTS" in lib.ua_last_error()


def test_noalloc_rejects_a_malformed_csr():
    """A column index outside [0, n) is reported as UA_ERR_INVALID before any product reads it."""
    torch = pytest.importorskip("torch")
    K, B, f, g, dofs, vals = _system()
    bad = K.copy()
    bad.indices = bad.indices.copy()
    bad.indices[bad.indptr[5]] = K.shape[0] + 7  # one column past the end
    with pytest.raises(L.UaError) as ei:
        _noalloc(torch, bad, dofs, vals, f, g)
    assert ei.value.code == L.UA_ERR_INVALID
    assert "CSR" in str(ei.value)
    # the entry point still works afterwards
    x_ref, _, _ = ua.solveKApeSymmetric(K, B, f, g, rtol=1e-12)
    x, _, _ = _noalloc(torch, K, dofs, vals, f, g)
    assert np.linalg.norm(x - x_ref) <= RTOL * np.linalg.norm(x_ref)
