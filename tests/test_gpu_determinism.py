"""Determinism under a reordered mesh: the same mesh with its elements in another order and each
element's nodes rotated (same orientation) gives the same tangent and residual up to the
reassociation of the per-entry sums (the segmented sum adds an entry's element contributions in
increasing element id, so a new element order changes only the order of those additions), and
the same converged solution.  Runs twice on the same input are bit-identical."""
import numpy as np
import pytest
import scipy.sparse as sp

import uasource_b200 as ua
from uasource_b200 import lib as L
from uasource_b200 import synth

pytestmark = pytest.mark.gpu


def _rotate(conn, nod, rng):
    """Each element's nodes rotated by 0, 1 or 2 corner positions (orientation kept)."""
    out = conn.copy()
    k = rng.integers(0, 3, conn.shape[0])
    step = 1 if nod == 3 else 2
    for e in range(conn.shape[0]):
        out[e] = np.roll(conn[e], -step * k[e])
    return out


@pytest.mark.parametrize("nod,nx,ny", [(3, 41, 21), (6, 13, 7)], ids=["P1", "P2"])
def test_permuted_elements_give_the_same_system_and_solution(nod, nx, ny):
    P = synth.ice_stream_shelf(nx, ny, nod=nod, seed=4)
    rng = np.random.default_rng(11)
    perm = rng.permutation(P.connectivity.shape[0])
    conn2 = _rotate(P.connectivity[perm], nod, rng)
    m1 = ua.CreateMUA(P.coordinates, P.connectivity)
    m2 = ua.CreateMUA(P.coordinates, conn2)
    F = ua.Fields.from_problem(P)
    F.ub = 100 + 200 * rng.random(P.Nnodes)
    F.vb = 30 * rng.standard_normal(P.Nnodes)
    R1, K1 = ua.uvMatrixAssembly(ua.CtrlVar(), m1, F)
    R2, K2 = ua.uvMatrixAssembly(ua.CtrlVar(), m2, F)
    K1, K2 = sp.csr_matrix(K1), sp.csr_matrix(K2)
    scale = np.maximum(abs(K1).max(axis=1).toarray().ravel(), 1e-300)
    assert np.max(abs(K1 - K2).max(axis=1).toarray().ravel() / scale) <= 1e-13
    assert np.max(np.abs(R1 - R2)) <= 1e-13 * np.max(np.abs(R1))
    ctrl = ua.CtrlVar().set_force_tolerance(1e-20)
    bcs = ua.BCs.from_problem(P)
    Fa, _, _, _, ia = ua.uv(ctrl, m1, bcs, ua.Fields.from_problem(P))
    Fb, _, _, _, ib = ua.uv(ctrl, m2, bcs, ua.Fields.from_problem(P))
    assert ia.converged and ib.converged
    ua_, ub_ = np.concatenate([Fa.ub, Fa.vb]), np.concatenate([Fb.ub, Fb.vb])
    assert np.linalg.norm(ua_ - ub_) <= 1e-11 * np.linalg.norm(ua_)
    # and the same input twice: bit for bit
    Fc, _, _, _, _ = ua.uv(ctrl, m1, bcs, ua.Fields.from_problem(P))
    assert np.array_equal(Fa.ub, Fc.ub) and np.array_equal(Fa.vb, Fc.vb)


def test_permuted_elements_mixed_precision():
    P = synth.ice_stream_shelf(61, 31, nod=3, seed=6)
    rng = np.random.default_rng(2)
    conn2 = _rotate(P.connectivity[rng.permutation(P.connectivity.shape[0])], 3, rng)
    ctrl = ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20)
    bcs = ua.BCs.from_problem(P)
    Fa, _, _, _, ia = ua.uv(ctrl, ua.CreateMUA(P.coordinates, P.connectivity), bcs, ua.Fields.from_problem(P))
    Fb, _, _, _, ib = ua.uv(ctrl, ua.CreateMUA(P.coordinates, conn2), bcs, ua.Fields.from_problem(P))
    assert ia.converged and ib.converged
    ua_, ub_ = np.concatenate([Fa.ub, Fa.vb]), np.concatenate([Fb.ub, Fb.vb])
    assert np.linalg.norm(ua_ - ub_) <= 1e-8 * np.linalg.norm(ua_)
