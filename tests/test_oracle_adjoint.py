"""The oracle's adjoint gradient (Misfit.m adjoint branch, dIdCq.m) is the derivative of the
velocity misfit with respect to the nodal C: central differences of I(C) through full Newton
solves agree with it (no GPU)."""
import numpy as np
import pytest

from oracle import ua_ref as R
from uasource_b200 import synth


@pytest.mark.parametrize("law", ["Weertman", "Budd", "Joughin"])
def test_adjoint_gradient_is_the_derivative_of_the_misfit(law):
    P = synth.ice_stream_shelf(9, 6, nod=3, seed=1)
    mua = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    p.set_force_tolerance(1e-24)
    p.SlidingLaw = law
    rng = np.random.default_rng(0)
    extra = {}
    if law == "Budd":
        extra["q"] = 1.0 + 0.1 * rng.random(P.Nnodes)
    if law == "Joughin":
        extra["V0"] = 100.0 + 50 * rng.random(P.Nnodes)
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    F = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb, **extra)

    def solve(C):
        G = F.copy()
        G.C = C
        r = R.uv(p, mua, bcs, G)
        assert r.converged
        return r

    res = solve(P.C)
    us = res.ub * (1 + 0.05 * rng.standard_normal(P.Nnodes))
    vs = res.vb + 2 * rng.standard_normal(P.Nnodes)
    ue = 1 + rng.random(P.Nnodes)
    ve = 1 + rng.random(P.Nnodes)
    Fs = F.copy()
    Fs.ub, Fs.vb = res.ub, res.vb
    badj = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=0 * P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                 vbFixedValue=0 * P.vbFixedValue)
    _, _, _, g = R.adjoint_gradient_C(p, mua, Fs, badj, us, vs, ue, ve, logC=False, premultiplier="I")

    def I_of(C):
        r = solve(C)
        G = F.copy()
        G.C, G.ub, G.vb = C, r.ub, r.vb
        return R.misfit_uv(mua, R.prepare_fields(p, G), us, vs, ue, ve)[0]

    for k in (5, 17, 30):
        e = 1e-6 * P.C[k]
        Cp, Cm = P.C.copy(), P.C.copy()
        Cp[k] += e
        Cm[k] -= e
        fd = (I_of(Cp) - I_of(Cm)) / (2 * e)
        # relative to the node, plus finite-difference noise at the scale of the largest entry
        assert abs(g[k] - fd) <= 1e-5 * abs(fd) + 1e-7 * np.max(np.abs(g))


def test_log_and_mass_premultiplier_forms():
    """log10(C) scaling and the (M/Area) pre-multiplier are the reference's post-processing."""
    P = synth.ice_stream_shelf(9, 6, nod=6, seed=2)
    mua = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    rng = np.random.default_rng(1)
    F = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m,
                 ub=100 + 10 * rng.random(P.Nnodes), vb=rng.standard_normal(P.Nnodes))
    b = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=0 * P.ubFixedValue, vbFixedNode=P.vbFixedNode,
              vbFixedValue=0 * P.vbFixedValue)
    args = (p, mua, F, b, F.ub + 1, F.vb - 1, np.ones(P.Nnodes), np.ones(P.Nnodes))
    _, _, _, g0 = R.adjoint_gradient_C(*args, logC=False, premultiplier="I")
    _, _, _, g1 = R.adjoint_gradient_C(*args, logC=True, premultiplier="I")
    _, _, _, g2 = R.adjoint_gradient_C(*args, logC=True, premultiplier="M")
    assert np.allclose(g1, np.log(10) * P.C * g0, rtol=1e-13, atol=0)
    M = R.mass_matrix(mua) / R.mesh_area(mua)
    assert np.allclose(M @ g2, g1, rtol=1e-10, atol=1e-12 * np.max(np.abs(g1)))
