"""The oracle's tied-node and fixed-normal-velocity constraints on CPU (CreateLuv.m:28-76,
CalcEdgeAndNodalNormals.m:9-40, ScaleL.m:28-33): the nodal normals of a rectangle and of the
same rectangle turned, the rows of L and c in the order of the multipliers, and uv / uvh Newton
solves that meet the constraints."""
import numpy as np
import pytest

from oracle import ua_ref as R
from tests.constraint_cases import front_nodes, problem, tie_nodes


@pytest.mark.parametrize("nod,nx,ny", [(3, 21, 11), (6, 9, 6)], ids=["P1", "P2"])
@pytest.mark.parametrize("angle", [0.0, np.pi / 6], ids=["axes", "turned"])
def test_nodal_normals_of_a_rectangle(nod, nx, ny, angle):
    P = problem(nx, ny, nod, angle)
    Nx, Ny = R.nodal_normals(P.coordinates, P.connectivity)
    c, s = np.cos(angle), np.sin(angle)
    rot = lambda a, b: (c * a - s * b, s * a + c * b)  # noqa: E731
    fr = front_nodes(P)
    assert np.allclose(np.stack([Nx[fr], Ny[fr]]), np.array(rot(1.0, 0.0))[:, None], atol=1e-12)
    bottom, top = tie_nodes(P)
    inner = bottom[:-1]  # the last one is the corner at x = Lx
    assert np.allclose(np.stack([Nx[inner], Ny[inner]]), np.array(rot(0.0, -1.0))[:, None], atol=1e-12)
    assert np.allclose(np.stack([Nx[top[:-1]], Ny[top[:-1]]]), np.array(rot(0.0, 1.0))[:, None], atol=1e-12)
    corner = bottom[-1]  # the mean of (1, 0) and (0, -1), normalised
    assert np.allclose([Nx[corner], Ny[corner]], np.array(rot(1.0, -1.0)) / np.sqrt(2), atol=1e-12)
    xy = P.unrotated if angle else P.coordinates
    interior = (xy[:, 0] > 1) & (xy[:, 0] < xy[:, 0].max() - 1) & (xy[:, 1] > 1) & (xy[:, 1] < xy[:, 1].max() - 1)
    assert np.all(np.isnan(Nx[interior])) and np.all(np.isnan(Ny[interior]))  # not on an edge: NaN


def test_constraint_rows_in_multiplier_order():
    P = problem(9, 6, 3, np.pi / 6)
    Nn = P.Nnodes
    bottom, top = tie_nodes(P)
    fr = front_nodes(P)
    vals = np.linspace(1.0, 2.0, fr.size)
    keep = ~np.isin(P.vbFixedNode, np.concatenate([bottom[:2], top[:2]]))  # v tied there instead
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode[keep],
                vbFixedValue=np.asarray(P.vbFixedValue)[keep], ubTiedNodeA=bottom, ubTiedNodeB=top,
                vbTiedNodeA=bottom[:2], vbTiedNodeB=top[:2], ubvbFixedNormalNode=fr, ubvbFixedNormalValue=vals)
    mua = R.create_mua(P.coordinates, P.connectivity)
    L, c = R.create_Luv(Nn, bcs, mua)
    Ld_ = L.toarray()
    assert np.all(np.count_nonzero(Ld_, axis=0) <= 1)  # disjoint support: B B' diagonal
    nu, nv = np.unique(P.ubFixedNode).size, np.unique(P.vbFixedNode[keep]).size
    assert L.shape == (bottom.size + 2 + nu + nv + fr.size, 2 * Nn)
    Ld = L.toarray()
    assert np.allclose(np.sum(Ld * Ld, axis=1), 1.0, rtol=0, atol=1e-15)  # ScaleL: unit rows
    r = 0
    for a, b in zip(bottom, top):  # u ties: (e_a - e_b)/sqrt(2), c = 0
        assert Ld[r, a] == pytest.approx(2 ** -0.5) and Ld[r, b] == pytest.approx(-(2 ** -0.5)) and c[r] == 0
        r += 1
    for a, b in zip(bottom[:2], top[:2]):  # v ties
        assert Ld[r, Nn + a] == pytest.approx(2 ** -0.5) and Ld[r, Nn + b] == pytest.approx(-(2 ** -0.5))
        r += 1
    assert np.array_equal(np.flatnonzero(Ld[r:r + nu].any(axis=0)), np.unique(P.ubFixedNode))
    r += nu + nv
    Nx, Ny = R.nodal_normals(P.coordinates, P.connectivity)
    for k, n in enumerate(fr):  # Nx u + Ny v = -value (already unit length)
        assert Ld[r, n] == Nx[n] and Ld[r, Nn + n] == Ny[n] and c[r] == -vals[k]
        r += 1
    assert r == L.shape[0]


def _uv_case(nod, nx, ny, angle, **bc):
    P = problem(nx, ny, nod, angle)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    F = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue, **bc)
    return P, p, F, bcs, R.create_mua(P.coordinates, P.connectivity)


@pytest.mark.parametrize("nod,nx,ny", [(3, 21, 11), (6, 9, 6)], ids=["P1", "P2"])
def test_uv_with_periodic_u_sides(nod, nx, ny):
    P = problem(nx, ny, nod)
    bottom, top = tie_nodes(P)
    P, p, F, bcs, mua = _uv_case(nod, nx, ny, 0.0, ubTiedNodeA=bottom, ubTiedNodeB=top)
    res = R.uv(p, mua, bcs, F)
    assert res.converged
    scale = np.max(np.abs(res.ub))
    assert np.max(np.abs(res.ub[bottom] - res.ub[top])) <= 1e-9 * scale
    free = R.uv(p, mua, R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                              vbFixedValue=P.vbFixedValue), F)
    assert np.max(np.abs(free.ub[bottom] - free.ub[top])) > 1e-3 * scale  # the ties change the solution
    assert res.lubvb.size == bottom.size + np.unique(P.ubFixedNode).size + np.unique(P.vbFixedNode).size


@pytest.mark.parametrize("nod,nx,ny", [(3, 21, 11), (6, 9, 6)], ids=["P1", "P2"])
def test_uv_with_no_normal_flow_through_the_front(nod, nx, ny):
    P = problem(nx, ny, nod, np.pi / 6)
    fr = front_nodes(P)
    P, p, F, bcs, mua = _uv_case(nod, nx, ny, np.pi / 6, ubvbFixedNormalNode=fr, ubvbFixedNormalValue=0 * fr + 0.0)
    res = R.uv(p, mua, bcs, F)
    assert res.converged
    Nx, Ny = R.nodal_normals(P.coordinates, P.connectivity)
    scale = np.max(np.hypot(res.ub, res.vb))
    assert np.max(np.abs(Nx[fr] * res.ub[fr] + Ny[fr] * res.vb[fr])) <= 1e-12 * scale
    assert np.max(np.hypot(res.ub[fr], res.vb[fr])) > 1e-3 * scale  # tangential flow remains


def test_uvh_with_periodic_u_sides():
    P = problem(13, 7, 3)
    bottom, top = tie_nodes(P)
    P, p, F, bcs, mua = _uv_case(3, 13, 7, 0.0, ubTiedNodeA=bottom, ubTiedNodeB=top)
    p.uvhDesiredWorkAndForceTolerances = (np.inf, 1e-20)
    p.uvhDesiredWorkOrForceTolerances = (np.inf, 1e-20)
    uv = R.uv(p, mua, bcs, F)
    S0 = R.UvhState(P.h.copy(), uv.ub.copy(), uv.vb.copy(), np.full(P.Nnodes, 0.3), np.zeros(P.Nnodes))
    res = R.sstream_transient_implicit(p, mua, bcs, F, S0, S0.copy(), 0.1)
    assert res.converged
    assert np.max(np.abs(res.ub[bottom] - res.ub[top])) <= 1e-9 * np.max(np.abs(res.ub))
