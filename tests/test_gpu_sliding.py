"""GPU parity of the other sliding laws and the melange drag (BasalDrag.m) against
the oracle, through the C-ABI: uv and uvh tangents and residuals within 1e-12
(per-row max-norm relative) on P1 and P2 meshes for every CtrlVar.SlidingLaw,
and converged uv Newton solutions within 1e-10 relative L2."""
import numpy as np
import pytest
import scipy.sparse as sp

import uasource_b200 as ua
from oracle import ua_ref as R
from uasource_b200 import synth
from tests.sliding_cases import LAWS, law_inputs, soften_C

pytestmark = pytest.mark.gpu
K_TOL = 1e-12
R_TOL = 1e-12
U_TOL = 1e-10


def _row_rel(Kg, Kr):
    D = (sp.csr_matrix(Kg) - sp.csr_matrix(Kr)).tocsr()
    scale = np.maximum(abs(sp.csr_matrix(Kr)).max(axis=1).toarray().ravel(), 1e-300)
    return np.max(abs(D).max(axis=1).toarray().ravel() / scale)


def _inputs(law, nod, nx, ny, transient=False):
    P = soften_C(synth.ice_stream_shelf(nx, ny, nod=nod, seed=5, transient=transient))
    name, mel, extra = law_inputs(law, P.Nnodes, seed=2)
    p = R.Params()
    p.SlidingLaw = name
    p.IncludeMelangeModelPhysics = mel
    ctrl = ua.CtrlVar(SlidingLaw=name, IncludeMelangeModelPhysics=int(mel))
    return P, p, ctrl, extra


@pytest.mark.parametrize("nod,nx,ny", [(3, 21, 11), (6, 9, 6)], ids=["P1", "P2"])
@pytest.mark.parametrize("law", LAWS)
def test_uv_assembly_matches_oracle(law, nod, nx, ny):
    P, p, ctrl, extra = _inputs(law, nod, nx, ny)
    rng = np.random.default_rng(9)
    ub = 100 + 200 * rng.random(P.Nnodes)
    vb = 30 * rng.standard_normal(P.Nnodes)
    Fo = R.prepare_fields(p, R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=ub,
                                      vb=vb, **extra))
    Rref, Kref, Tref, _ = R.uv_matrix_assembly(p, R.create_mua(P.coordinates, P.connectivity), Fo,
                                              return_parts=True)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)
    F.ub, F.vb = ub, vb
    for k, v in extra.items():
        setattr(F, k, v)
    Rg, Kg = ua.uvMatrixAssembly(ctrl, mua, F)
    assert _row_rel(Kg, Kref) <= K_TOL
    assert np.max(np.abs(Rg - Rref)) <= R_TOL * max(np.max(np.abs(Rref)), np.max(np.abs(Tref)))
    Rr, _ = ua.uvMatrixAssembly(ctrl, mua, F, Ronly=True)
    assert np.array_equal(Rr, Rg)


@pytest.mark.parametrize("nod,nx,ny", [(3, 21, 11), (6, 9, 6)], ids=["P1", "P2"])
@pytest.mark.parametrize("law", LAWS)
def test_uvh_assembly_matches_oracle(law, nod, nx, ny):
    P, p, ctrl, extra = _inputs(law, nod, nx, ny, transient=True)
    rng = np.random.default_rng(4)
    n = P.Nnodes
    u0 = 100 + 100 * rng.random(n); v0 = 20 * rng.standard_normal(n)
    S0 = R.UvhState(P.h.copy(), u0, v0, P.as_.copy(), P.ab.copy())
    S1 = R.UvhState(P.h + 3 * rng.standard_normal(n), u0 * (1 + 0.05 * rng.standard_normal(n)),
                    v0 + 2 * rng.standard_normal(n), P.as_.copy(), P.ab.copy())
    Fo = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=u0, vb=v0, **extra)
    Rref, Kref = R.uvh_matrix_assembly(p, R.create_mua(P.coordinates, P.connectivity), Fo, S0, S1, 0.1)
    mua = ua.CreateMUA(P.coordinates, P.connectivity, ndof=3)
    F0 = ua.Fields.from_problem(P)
    F0.h, F0.ub, F0.vb = S0.h, S0.ub, S0.vb
    for k, v in extra.items():
        setattr(F0, k, v)
    F1 = F0.copy()
    F1.h, F1.ub, F1.vb = S1.h, S1.ub, S1.vb
    Rg, Kg = ua.uvhAssembly(ctrl, mua, F0, F1, 0.1)
    assert _row_rel(Kg, Kref) <= K_TOL
    assert np.max(np.abs(Rg - Rref)) <= R_TOL * np.max(np.abs(Rref))


@pytest.mark.parametrize("law", ["Budd", "Tsai", "Umbi", "Joughin", "melange"])
def test_uv_newton_matches_oracle(law):
    P, p, ctrl, extra = _inputs(law, 3, 21, 11)
    p.set_force_tolerance(1e-20)
    Fo = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb, **extra)
    bo = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
               vbFixedValue=P.vbFixedValue)
    ref = R.uv(p, R.create_mua(P.coordinates, P.connectivity), bo, Fo)
    assert ref.converged
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)
    for k, v in extra.items():
        setattr(F, k, v)
    Fg, _, _, _, info = ua.uv(ctrl.set_force_tolerance(1e-20), mua, ua.BCs.from_problem(P), F)
    assert info.converged
    u_ref = np.concatenate([ref.ub, ref.vb]); u = np.concatenate([Fg.ub, Fg.vb])
    assert np.linalg.norm(u - u_ref) <= U_TOL * np.linalg.norm(u_ref)


def test_missing_law_field_is_refused():
    P, p, ctrl, extra = _inputs("Budd", 3, 9, 6)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)  # no F.q
    from uasource_b200 import lib as L
    with pytest.raises(L.UaError) as ei:
        ua.uvMatrixAssembly(ctrl, mua, F)
    assert ei.value.code == L.UA_ERR_INVALID and "F.q" in str(ei.value)
