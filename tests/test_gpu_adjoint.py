"""GPU parity of the adjoint gradient of the velocity misfit with respect to C
(Misfit.m adjoint branch, dIdCq.m, ApplyAdjointGradientPreMultiplier.m) against the
oracle, through the C-ABI (ua_uv_adjoint_dIdC).

The misfit I and its gradient dI/d(u,v) come from the mass matrix and the data
alone (within 1e-12); the adjoint velocities lambda solve the constrained tangent
system iteratively here and directly in the oracle, so lambda satisfies the oracle's
adjoint system to a componentwise backward error of 1e-10, and lambda and the gradient dIdC are
compared within 1e-9 relative L2 with the inner tolerance at 1e-14.  The coarse P2
case (9 x 6 vertices) has a tangent of condition number about 1e11 (drag of order
1e15 next to the u = 0 inflow boundary), so any two solves of it agree only to about
cond x 1e-16: there lambda and dIdC are compared within 1e-5 beside the backward error.
"""
import numpy as np
import pytest

import uasource_b200 as ua
from oracle import ua_ref as R
from uasource_b200 import synth
from uasource_b200 import lib as L
from tests.sliding_cases import law_inputs, soften_C

pytestmark = pytest.mark.gpu
TOL_DATA = 1e-12
TOL_ADJ = 1e-9
TOL_ADJ_ILL = 1e-5   # the 9 x 6 P2 tangent, condition number ~1e11
TOL_BACKWARD = 1e-10


def _case(nod, nx, ny, law):
    P = synth.ice_stream_shelf(nx, ny, nod=nod, seed=3)
    if nod == 6:
        soften_C(P)
    name, _, extra = law_inputs(law, P.Nnodes, seed=4)
    p = R.Params()
    p.set_force_tolerance(1e-16)
    p.SlidingLaw = name
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    F = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb, **extra)
    mua = R.create_mua(P.coordinates, P.connectivity)
    res = R.uv(p, mua, bcs, F)  # the state: any velocity field serves, the solved one is typical
    rng = np.random.default_rng(8)
    us = res.ub * (1 + 0.05 * rng.standard_normal(P.Nnodes)) + rng.standard_normal(P.Nnodes)
    vs = res.vb + 2 * rng.standard_normal(P.Nnodes)
    ue = 1 + rng.random(P.Nnodes)
    ve = 1 + rng.random(P.Nnodes)
    Fs = F.copy()
    Fs.ub, Fs.vb = res.ub, res.vb
    badj = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=0 * P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                 vbFixedValue=0 * P.vbFixedValue)
    return P, p, mua, Fs, badj, (us, vs, ue, ve), name, extra


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("logC,prem", [(False, "I"), (True, "M")], ids=["C-I", "logC-M"])
@pytest.mark.parametrize("nod,nx,ny,law", [(3, 21, 11, "Weertman"), (6, 9, 6, "Weertman"), (3, 15, 8, "Budd"),
                                           (3, 15, 8, "Umbi"), (3, 15, 8, "Joughin")],
                         ids=["P1-Weertman", "P2-Weertman", "P1-Budd", "P1-Umbi", "P1-Joughin"])
def test_adjoint_gradient_matches_oracle(nod, nx, ny, law, logC, prem):
    P, p, mua_o, Fs, badj, data, name, extra = _case(nod, nx, ny, law)
    I_ref, dIduv_ref, lam_ref, g_ref = R.adjoint_gradient_C(p, mua_o, Fs, badj, *data, logC=logC,
                                                            premultiplier=prem)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)
    F.ub, F.vb = Fs.ub, Fs.vb
    for k, v in extra.items():
        setattr(F, k, v)
    bg = ua.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=0 * P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=0 * P.vbFixedValue)
    ctrl = ua.CtrlVar(SlidingLaw=name, krylov_rtol=1e-14)
    I, dIduv, lam, g, its = ua.adjoint_gradient_C(ctrl, mua, F, bg, *data, logC=logC, premultiplier=prem)
    assert its > 0
    assert abs(I - I_ref) <= TOL_DATA * abs(I_ref)
    assert _rel(dIduv, dIduv_ref) <= TOL_DATA
    # backward error in the oracle's system: K lambda = dI/duv on the free dofs, lambda = 0 on the fixed
    _, K = R.uv_matrix_assembly(p, mua_o, R.prepare_fields(p, Fs))
    Lm, _ = R.create_Luv(P.Nnodes, badj, mua_o)
    fixed = np.unique(Lm.nonzero()[1])
    free = np.setdiff1d(np.arange(2 * P.Nnodes), fixed)
    r = (K @ lam - dIduv_ref)[free]
    # componentwise (Oettli-Prager): rows next to the u = 0 inflow carry drag of order 1e15
    scale = (abs(K) @ np.abs(lam) + np.abs(dIduv_ref))[free]
    assert np.max(np.abs(r) / scale) <= TOL_BACKWARD
    assert np.max(np.abs(lam[fixed])) <= 1e-12 * np.max(np.abs(lam))
    tol = TOL_ADJ_ILL if nod == 6 else TOL_ADJ
    assert _rel(lam, lam_ref) <= tol
    assert _rel(g, g_ref) <= tol


def test_coulomb_has_no_C_gradient():
    P = synth.ice_stream_shelf(9, 6, nod=3, seed=3)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)
    F.muk = 0.01 + 0 * P.h
    z = np.zeros(P.Nnodes)
    with pytest.raises(L.UaError) as ei:
        ua.adjoint_gradient_C(ua.CtrlVar(SlidingLaw="Coulomb"), mua, F, ua.BCs.from_problem(P), z, z, z + 1, z + 1)
    assert ei.value.code == L.UA_ERR_INVALID
