"""GPU parity of the tied-node and fixed-normal-velocity constraints (CreateLuv.m:28-76,
CalcEdgeAndNodalNormals.m:9-40, ScaleL.m:28-33, ABfgPreEliminate.m) against the oracle, through
the C-ABI: the constraint matrix L and c row for row, uv Newton solutions and multipliers within
1e-10 relative (P1 and P2, FP64; 1e-8 with the mixed-precision preconditioner), the implicit uvh
step with ties (GMRES), and the refusals (a dof in two rows, a normal at an interior node,
BiCGStab with two-entry rows)."""
import numpy as np
import pytest

import uasource_b200 as ua
from oracle import ua_ref as R
from uasource_b200 import lib as L
from tests.constraint_cases import front_nodes, problem, tie_nodes

pytestmark = pytest.mark.gpu
U_TOL = 1e-10
U_TOL_MIXED = 1e-8
ANGLE = np.pi / 6


def _bc_kw(P, kind):
    if kind == "ties":
        bottom, top = tie_nodes(P)
        return dict(ubTiedNodeA=bottom, ubTiedNodeB=top)
    if kind == "normal":
        fr = front_nodes(P)
        return dict(ubvbFixedNormalNode=fr, ubvbFixedNormalValue=np.zeros(fr.size))
    bottom, top = tie_nodes(P)
    fr = front_nodes(P)
    return dict(ubTiedNodeA=bottom[:-1], ubTiedNodeB=top[:-1], ubvbFixedNormalNode=fr,
                ubvbFixedNormalValue=np.zeros(fr.size))


def _fixed(P, v_free=()):
    """The problem's fixed u and v nodes, without v at the nodes in v_free (whose v is tied)."""
    keep = ~np.isin(P.vbFixedNode, np.asarray(v_free, dtype=np.int64))
    return dict(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode[keep],
                vbFixedValue=np.asarray(P.vbFixedValue)[keep])


def test_constraint_matrix_matches_oracle():
    P = problem(9, 6, 3, ANGLE)
    bottom, top = tie_nodes(P)
    fr = front_nodes(P)
    kw = dict(ubTiedNodeA=bottom, ubTiedNodeB=top, vbTiedNodeA=bottom[:2], vbTiedNodeB=top[:2],
              ubvbFixedNormalNode=fr, ubvbFixedNormalValue=np.linspace(1.0, 2.0, fr.size))
    fx = _fixed(P, v_free=np.concatenate([bottom[:2], top[:2]]))
    Lr, cr = R.create_Luv(P.Nnodes, R.BCs(**fx, **kw), R.create_mua(P.coordinates, P.connectivity))
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    Lg, cg = ua.constraint_matrix(mua, ua.BCs(**fx, **kw))
    assert Lg.shape == Lr.shape
    assert np.max(np.abs((Lg - Lr).toarray())) <= 1e-15
    assert np.max(np.abs(cg - cr)) <= 1e-15 * np.max(np.abs(cr))


@pytest.mark.parametrize("nod,nx,ny", [(3, 21, 11), (6, 9, 6)], ids=["P1", "P2"])
@pytest.mark.parametrize("kind", ["ties", "normal", "both"])
def test_uv_newton_matches_oracle(kind, nod, nx, ny):
    P = problem(nx, ny, nod, 0.0 if kind == "ties" else ANGLE)
    kw = _bc_kw(P, kind)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    Fo = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    ref = R.uv(p, R.create_mua(P.coordinates, P.connectivity), R.BCs(**_fixed(P), **kw), Fo)
    assert ref.converged
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    Fg, lam, _, _, info = ua.uv(ua.CtrlVar().set_force_tolerance(1e-20), mua, ua.BCs(**_fixed(P), **kw),
                                ua.Fields.from_problem(P))
    assert info.converged
    u_ref = np.concatenate([ref.ub, ref.vb]); u = np.concatenate([Fg.ub, Fg.vb])
    assert np.linalg.norm(u - u_ref) <= U_TOL * np.linalg.norm(u_ref)
    assert lam.shape == ref.lubvb.shape
    assert np.linalg.norm(lam - ref.lubvb) <= 1e-8 * np.linalg.norm(ref.lubvb)
    Lg, cg = ua.constraint_matrix(mua, ua.BCs(**_fixed(P), **kw))
    assert np.max(np.abs(Lg @ u - cg)) <= 1e-9 * np.max(np.abs(u))


def test_uv_mixed_precision_with_ties_and_normals():
    P = problem(41, 21, 3, ANGLE)
    kw = _bc_kw(P, "both")
    p = R.Params()
    p.set_force_tolerance(1e-20)
    Fo = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    ref = R.uv(p, R.create_mua(P.coordinates, P.connectivity), R.BCs(**_fixed(P), **kw), Fo)
    assert ref.converged
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    ctrl = ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20)
    Fg, _, _, _, info = ua.uv(ctrl, mua, ua.BCs(**_fixed(P), **kw), ua.Fields.from_problem(P))
    assert info.converged
    u_ref = np.concatenate([ref.ub, ref.vb]); u = np.concatenate([Fg.ub, Fg.vb])
    assert np.linalg.norm(u - u_ref) <= U_TOL_MIXED * np.linalg.norm(u_ref)


def _uvh_case():
    P = problem(13, 7, 3)
    kw = _bc_kw(P, "ties")
    p = R.Params()
    p.set_force_tolerance(1e-20)
    p.uvhDesiredWorkAndForceTolerances = (np.inf, 1e-20)
    p.uvhDesiredWorkOrForceTolerances = (np.inf, 1e-20)
    Fo = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    mo = R.create_mua(P.coordinates, P.connectivity)
    uv = R.uv(p, mo, R.BCs(**_fixed(P), **kw), Fo)
    as_ = np.full(P.Nnodes, 0.3)
    S0 = R.UvhState(P.h.copy(), uv.ub.copy(), uv.vb.copy(), as_, np.zeros(P.Nnodes))
    F0 = ua.Fields.from_problem(P)
    F0.ub, F0.vb, F0.as_, F0.ab = uv.ub.copy(), uv.vb.copy(), as_.copy(), np.zeros(P.Nnodes)
    return P, kw, p, Fo, mo, S0, F0


def test_uvh_with_ties_matches_oracle():
    P, kw, p, Fo, mo, S0, F0 = _uvh_case()
    ref = R.sstream_transient_implicit(p, mo, R.BCs(**_fixed(P), **kw), Fo, S0, S0.copy(), 0.1)
    assert ref.converged
    mua = ua.CreateMUA(P.coordinates, P.connectivity, ndof=3)
    ctrl = ua.CtrlVar(uvh_krylov=L.UA_KRYLOV_GMRES, ThicknessConstraints=0).set_force_tolerance(1e-20) \
        .set_uvh_force_tolerance(1e-20)
    Fg, _, info = ua.uvh(ctrl, mua, F0, F0.copy(), ua.HBCs(**_fixed(P), **kw), 0.1)
    assert info.converged
    got = np.concatenate([Fg.ub, Fg.vb, Fg.h])
    want = np.concatenate([ref.ub, ref.vb, ref.h])
    assert np.linalg.norm(got - want) <= U_TOL * np.linalg.norm(want)
    bottom, top = kw["ubTiedNodeA"], kw["ubTiedNodeB"]
    assert np.max(np.abs(Fg.ub[bottom] - Fg.ub[top])) <= 1e-9 * np.max(np.abs(Fg.ub))


def test_uvh_bicgstab_refuses_two_entry_rows():
    P, kw, p, Fo, mo, S0, F0 = _uvh_case()
    mua = ua.CreateMUA(P.coordinates, P.connectivity, ndof=3)
    ctrl = ua.CtrlVar(uvh_krylov=L.UA_KRYLOV_BICGSTAB, ThicknessConstraints=0)
    with pytest.raises(L.UaError) as ei:
        ua.uvh(ctrl, mua, F0, F0.copy(), ua.HBCs(**_fixed(P), **kw), 0.1)
    assert ei.value.code == L.UA_ERR_INVALID and "GMRES" in str(ei.value)


def test_overlapping_constraints_are_refused():
    P = problem(9, 6, 3)
    bottom, top = tie_nodes(P)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    # the first tied node also has u fixed: two rows share a dof, B B' is not diagonal
    b = ua.BCs(ubFixedNode=np.concatenate([P.ubFixedNode, bottom[:1]]),
               ubFixedValue=np.concatenate([P.ubFixedValue, [0.0]]), vbFixedNode=P.vbFixedNode,
               vbFixedValue=P.vbFixedValue, ubTiedNodeA=bottom, ubTiedNodeB=top)
    with pytest.raises(L.UaError) as ei:
        ua.uv(ua.CtrlVar(), mua, b, ua.Fields.from_problem(P))
    assert ei.value.code == L.UA_ERR_INVALID and "not diagonal" in str(ei.value)


def test_normal_at_an_interior_node_is_refused():
    P = problem(9, 6, 3)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    x, y = P.coordinates[:, 0], P.coordinates[:, 1]
    inner = np.flatnonzero((x > x.min() + 1) & (x < x.max() - 1) & (y > y.min() + 1) & (y < y.max() - 1))[:1]
    b = ua.BCs(**_fixed(P), ubvbFixedNormalNode=inner, ubvbFixedNormalValue=np.zeros(1))
    with pytest.raises(L.UaError) as ei:
        ua.constraint_matrix(mua, b)
    assert ei.value.code == L.UA_ERR_INVALID and "boundary" in str(ei.value)
