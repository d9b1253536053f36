"""GPU parity of the minimum-thickness active set of the implicit step (uvh.m:64-212,
ActiveSetInitialisation.m, ActiveSetUpdate.m, CalculateReactions.m) against the oracle,
through the C-ABI: the same final active set (node for node), the same number of active-set
iterations, and u, v, h within 1e-10 relative L2."""
import numpy as np
import pytest

import uasource_b200 as ua
from oracle import ua_ref as R
from tests.active_set_cases import SEED_NODES, SEED_THIN_NODE, thin_patch_problem

pytestmark = pytest.mark.gpu
U_TOL = 1e-10


@pytest.mark.parametrize("seeded", [False, True], ids=["activate", "release"])
def test_active_set_matches_oracle(seeded):
    P, h, as_ = thin_patch_problem()
    if seeded:
        h[SEED_THIN_NODE] = 1.05
    seed = SEED_NODES if seeded else None
    mua_o = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    p.uvhDesiredWorkAndForceTolerances = (np.inf, 1e-20)
    p.uvhDesiredWorkOrForceTolerances = (np.inf, 1e-20)
    F = R.Fields(h=h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    uv = R.uv(p, mua_o, bcs, F)
    S0 = R.UvhState(h.copy(), uv.ub.copy(), uv.vb.copy(), as_.copy(), P.ab.copy())
    ref = R.uvh_active_set(p, mua_o, bcs, F, S0, S0.copy(), 0.1, hPosNode=seed)
    assert ref.converged and ref.hPosNode.size > 0

    mua = ua.CreateMUA(P.coordinates, P.connectivity, ndof=3)
    F0 = ua.Fields.from_problem(P)
    F0.h, F0.ub, F0.vb, F0.as_ = h.copy(), uv.ub.copy(), uv.vb.copy(), as_.copy()
    hb = ua.HBCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                 vbFixedValue=P.vbFixedValue, hPosNode=np.zeros(0, np.int32) if seed is None else seed)
    ctrl = ua.CtrlVar().set_force_tolerance(1e-20).set_uvh_force_tolerance(1e-20)
    Fo, _, info = ua.uvh(ctrl, mua, F0, F0.copy(), hb, 0.1)
    assert info.converged
    a = info.active_set
    assert a["converged"] and a["iterations"] == ref.iterations and a["cyclical"] == ref.cyclical
    assert np.array_equal(np.asarray(a["hPosNode"]), ref.hPosNode)
    got = np.concatenate([Fo.ub, Fo.vb, Fo.h])
    want = np.concatenate([ref.res.ub, ref.res.vb, ref.res.h])
    assert np.linalg.norm(got - want) <= U_TOL * np.linalg.norm(want)
    assert np.all(Fo.h[ref.hPosNode] == 1.0)


def test_active_set_off_is_the_unconstrained_step():
    P, h, as_ = thin_patch_problem()
    mua = ua.CreateMUA(P.coordinates, P.connectivity, ndof=3)
    F0 = ua.Fields.from_problem(P)
    F0.h, F0.as_ = h.copy(), as_.copy()
    hb = ua.HBCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                 vbFixedValue=P.vbFixedValue)
    ctrl = ua.CtrlVar(ThicknessConstraints=0).set_force_tolerance(1e-20)
    Fo, _, info = ua.uvh(ctrl, mua, F0, F0.copy(), hb, 0.1)
    assert info.active_set is None
    assert np.min(Fo.h) < 1.0
