"""The oracle's minimum-thickness active set (uvh.m:64-212) on CPU: constraints are
activated where the step would go below ThickMin, seeded thick nodes are released by their
mass-flux reactions, and with thick ice everywhere the loop is the unconstrained step."""
import numpy as np

from oracle import ua_ref as R
from tests.active_set_cases import SEED_NODES, SEED_THIN_NODE, thin_patch_problem


def _setup(h):
    P, _, as_ = thin_patch_problem()
    mua = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    p.uvhDesiredWorkAndForceTolerances = (np.inf, 1e-20)
    p.uvhDesiredWorkOrForceTolerances = (np.inf, 1e-20)
    F = R.Fields(h=h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    uv = R.uv(p, mua, bcs, F)
    S0 = R.UvhState(h.copy(), uv.ub.copy(), uv.vb.copy(), as_.copy(), P.ab.copy())
    return P, p, mua, F, bcs, S0


def test_thinning_activates_constraints():
    P, h, _ = thin_patch_problem()
    P, p, mua, F, bcs, S0 = _setup(h)
    out = R.uvh_active_set(p, mua, bcs, F, S0, S0.copy(), 0.1)
    assert out.converged and out.res.converged and not out.cyclical
    assert out.hPosNode.size > 0 and out.iterations >= 2
    assert np.all(out.res.h[out.hPosNode] == p.ThickMin)
    assert np.min(out.res.h) >= p.ThickMin - 1e-9
    free = R.sstream_transient_implicit(p, mua, bcs, F, S0, S0.copy(), 0.1)
    assert np.min(free.h) < p.ThickMin  # without the constraints the step goes below ThickMin


def test_seeded_thick_nodes_are_released():
    P, h, _ = thin_patch_problem()
    h[SEED_THIN_NODE] = 1.05
    P, p, mua, F, bcs, S0 = _setup(h)
    out = R.uvh_active_set(p, mua, bcs, F, S0, S0.copy(), 0.1, hPosNode=SEED_NODES)
    assert out.converged
    released = np.setdiff1d(SEED_NODES, out.hPosNode)
    assert released.size >= 2 and np.all(h[released] > 1.0)


def test_thick_ice_is_the_unconstrained_step():
    P, _, _ = thin_patch_problem()
    P, p, mua, F, bcs, S0 = _setup(P.h.copy())
    S0.as_ = P.as_.copy()
    out = R.uvh_active_set(p, mua, bcs, F, S0, S0.copy(), 0.1)
    free = R.sstream_transient_implicit(p, mua, bcs, F, S0, S0.copy(), 0.1)
    assert out.hPosNode.size == 0 and out.iterations == 1
    assert np.array_equal(out.res.h, free.h) and np.array_equal(out.res.ub, free.ub)
