"""The compiled restatement of the uv element loop (oracle/ua_ref_asm.cpp) agrees
with the numpy oracle (no GPU).

Both restate uvMatrixAssemblySSTREAM.m's element loop in the reference's
operation order; they differ only in the order numpy's matrix products sum the
integration-point interpolations, so K and R agree to a few units in the last
place and the stored patterns are identical.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import ua_ref as R
from uasource_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.join(os.path.dirname(HERE), "oracle")


@pytest.fixture(scope="module")
def compiled():
    if not os.path.exists(os.path.join(ORACLE, "libua_ref_asm.so")):
        subprocess.run(["make", "-C", ORACLE], check=True, capture_output=True)
    yield
    R.use_compiled_element_loop(False)


@pytest.mark.parametrize("nod,nx,ny", [(3, 41, 21), (6, 13, 7)])
@pytest.mark.parametrize("threads", [1, 3])
def test_compiled_element_loop_matches_numpy(compiled, nod, nx, ny, threads):
    P = synth.ice_stream_shelf(nx, ny, nod=nod, seed=2)
    m = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    rng = np.random.default_rng(4)
    F = R.prepare_fields(p, R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m,
                                     ub=100 * rng.random(P.Nnodes), vb=10 * rng.standard_normal(P.Nnodes)))
    R.use_compiled_element_loop(False)
    R0, K0, T0, F0 = R.uv_matrix_assembly(p, m, F, return_parts=True)
    R.use_compiled_element_loop(True, threads)
    R1, K1, T1, F1 = R.uv_matrix_assembly(p, m, F, return_parts=True)
    Rr, Kr = R.uv_matrix_assembly(p, m, F, Ronly=True)
    R.use_compiled_element_loop(False)
    assert abs(K1 - K0).max() <= 1e-14 * abs(K0).max()
    assert np.max(np.abs(T1 - T0)) <= 1e-14 * np.max(np.abs(T0))
    assert np.max(np.abs(F1 - F0)) <= 1e-14 * np.max(np.abs(F0))
    assert np.array_equal(K1.indptr, K0.indptr) and np.array_equal(K1.indices, K0.indices)
    assert Kr is None and np.array_equal(Rr, R1)


def test_compiled_newton_solve_matches_numpy(compiled):
    P = synth.ice_stream_shelf(21, 11, nod=3, seed=0)
    m = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    F = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    R.use_compiled_element_loop(False)
    a = R.uv(p, m, bcs, F)
    R.use_compiled_element_loop(True, 1)
    b = R.uv(p, m, bcs, F)
    R.use_compiled_element_loop(False)
    assert a.converged and b.converged and a.iterations == b.iterations
    ua_, ub_ = np.concatenate([a.ub, a.vb]), np.concatenate([b.ub, b.vb])
    assert np.linalg.norm(ub_ - ua_) <= 1e-12 * np.linalg.norm(ua_)
