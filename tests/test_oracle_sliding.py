"""The oracle's sliding laws (no GPU): for every CtrlVar.SlidingLaw and the melange
terms, the uv tangent is the derivative of the residual (central difference), so
the drag derivatives restated in oracle/ua_ref.py (BasalDrag.m and its
rCWN0/rpCWN0/rCWV0 laws) are consistent with the drag stresses."""
import numpy as np
import pytest

from oracle import ua_ref as R
from uasource_b200 import synth
from tests.sliding_cases import LAWS, law_inputs


def _case(law, nod=3, seed=3):
    P = synth.ice_stream_shelf(9, 6, nod=nod, seed=seed)
    mua = R.create_mua(P.coordinates, P.connectivity)
    rng = np.random.default_rng(1)
    name, mel, extra = law_inputs(law, mua.Nnodes)
    p = R.Params()
    p.SlidingLaw = name
    p.IncludeMelangeModelPhysics = mel
    F = R.prepare_fields(p, R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m,
                                     ub=100 + 50 * rng.random(mua.Nnodes), vb=20 * rng.standard_normal(mua.Nnodes),
                                     **extra))
    return p, mua, F, rng


@pytest.mark.parametrize("law", LAWS)
def test_uv_tangent_is_derivative_of_residual_for_each_law(law):
    p, mua, F, rng = _case(law)
    Rv, K = R.uv_matrix_assembly(p, mua, F)
    assert abs(K - K.T).max() <= 1e-14 * abs(K).max()
    d = rng.standard_normal(2 * mua.Nnodes)
    eps = 1e-3
    Fp = F.copy(); Fp.ub = F.ub + eps * d[:mua.Nnodes]; Fp.vb = F.vb + eps * d[mua.Nnodes:]
    Fm = F.copy(); Fm.ub = F.ub - eps * d[:mua.Nnodes]; Fm.vb = F.vb - eps * d[mua.Nnodes:]
    Rp, _ = R.uv_matrix_assembly(p, mua, Fp, Ronly=True)
    Rm, _ = R.uv_matrix_assembly(p, mua, Fm, Ronly=True)
    fd = (Rp - Rm) / (2 * eps)
    Kd = K @ d
    assert np.linalg.norm(fd - Kd) < 1e-5 * np.linalg.norm(Kd)


@pytest.mark.parametrize("law", LAWS)
def test_each_law_changes_the_residual(law):
    """Every law is actually dispatched: its residual differs from Weertman's (except Weertman)."""
    p, mua, F, _ = _case(law)
    Rv, _ = R.uv_matrix_assembly(p, mua, F, Ronly=True)
    pw = R.Params()
    Rw, _ = R.uv_matrix_assembly(pw, mua, F, Ronly=True)
    if law == "Weertman":
        assert np.array_equal(Rv, Rw)
    else:
        assert np.max(np.abs(Rv - Rw)) > 1e-6 * np.max(np.abs(Rw))


def test_unknown_law_is_refused():
    p, mua, F, _ = _case("Weertman")
    p.SlidingLaw = "NoSuchLaw"
    with pytest.raises(ValueError):
        R.uv_matrix_assembly(p, mua, F, Ronly=True)
