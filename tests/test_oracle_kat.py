"""Pin the CPU oracle against the reference's known answers (no GPU)."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ua_ref as R
from uasource_b200 import synth
from tests.kat_problems import ice_shelf_problem, ice_stream_problem


def _fields(P):
    return R.Fields(h=P["h"], S=P["S"], B=P["B"], rho=P["rho"], AGlen=P["AGlen"], n=P["n"], C=P["C"], m=P["m"],
                    ub=P["ub"], vb=P["vb"], rhow=P["rhow"], g=P["g"])


def _bcs(P):
    return R.BCs(ubFixedNode=P["ubFixedNode"], ubFixedValue=P["ubFixedValue"], vbFixedNode=P["vbFixedNode"],
                 vbFixedValue=P["vbFixedValue"])


# --- quadrature (TestFEintegrate.m) -----------------------------------------------

@pytest.mark.parametrize("degree", [4, 8])
def test_quadrature_exact_for_monomials(degree):
    """The degree-d PI rule integrates x^i y^j exactly for i+j<=d on the unit triangle."""
    from math import factorial
    pts, w = R.quad_rule(degree)
    assert abs(w.sum() - 0.5) < 1e-15
    assert np.all(w > 0) and np.all(pts > 0) and np.all(pts.sum(1) < 1)
    for i in range(degree + 1):
        for j in range(degree + 1 - i):
            exact = factorial(i) * factorial(j) / factorial(i + j + 2)
            got = np.sum(w * pts[:, 0] ** i * pts[:, 1] ** j)
            assert abs(got - exact) < 1e-15, (i, j)


@pytest.mark.parametrize("nod,p", [(3, 1), (3, 4), (6, 1), (6, 8)])
def test_fe_integrate_two_element_square(nod, p):
    """TestFEintegrate.m:4-31: integrate (1+x+y)^p over the unit square split in two elements."""
    coords = np.array([[0, 0], [0, 1], [1, 1], [1, 0]], float)
    conn = np.array([[0, 1, 3], [3, 1, 2]])
    if nod == 6:
        coords, conn = synth.tri3to6(coords, conn)
    mua = R.create_mua(coords, conn)
    total = 0.0
    for ip in range(mua.nip):
        fun = R.shape_fun(nod, mua.points[ip])
        xy = mua.coordinates[mua.connectivity] @ np.eye(2)  # Nele x nod x 2
        xi = np.einsum("ean,a->en", xy, fun)
        total += np.sum((1 + xi[:, 0] + xi[:, 1]) ** p * mua.DetJ[:, ip] * mua.weights[ip])
    exact = (3 ** (p + 2) - 2 * 2 ** (p + 2) + 1) / ((p + 1) * (p + 2))
    assert abs(total - exact) < 1e-12 * exact


# --- saddle-point elimination (TestABfgPreEliminate.m) ---------------------------

def test_abfg_pre_eliminate_examples():
    A = sp.csr_matrix(np.array([[0, 1, 0], [1, 0, 0], [0, 0, 1.0]]))
    x, y = R.abfg_pre_eliminate(A, None, np.ones(3), None)
    assert np.allclose(x, [1, 1, 1])
    A = sp.csr_matrix(np.diag([0, 0, 1.0, 1.0]))
    B = sp.csr_matrix(np.array([[1, 0, 0, 0], [0, 1, 0, 0.0]]))
    f = np.array([10, 2, 10, 1000.0]); g = np.array([10, 10.0])
    x, y = R.abfg_pre_eliminate(A, B, f, g)
    T = np.block([[A.toarray(), B.toarray().T], [B.toarray(), np.zeros((2, 2))]])
    sol = np.linalg.lstsq(T, np.concatenate([f, g]), rcond=None)[0]
    assert np.allclose(x, [10, 10, 10, 1000]) and np.allclose(y, [10, 2])
    assert np.allclose(np.concatenate([x, y]), sol)


# --- analytic SSA solutions ---------------------------------------------------------

def _solve_kat(P, nod):
    p = R.Params(etaZero=0.0)
    p.set_force_tolerance(1e-24)
    mua = R.create_mua(P["coordinates"], P["connectivity"])
    res = R.uv(p, mua, _bcs(P), _fields(P))
    assert res.converged
    return res


@pytest.mark.parametrize("nod", [3, 6])
def test_ice_shelf_analytic(nod):
    """AnalyticalOneDimentionalIceShelf.m: FE velocity converges to (a x+q)/h, error O(dx^2)."""
    errs = []
    for nx in (21, 41):
        P, u_exact = ice_shelf_problem(nx=nx, nod=nod)
        res = _solve_kat(P, nod)
        errs.append(np.max(np.abs(res.ub - u_exact)) / np.max(u_exact))
        assert np.max(np.abs(res.vb)) < 1e-5 * np.max(u_exact)  # v is a discretisation artefact
    assert errs[1] < (2e-4 if nod == 3 else 5e-6)
    assert errs[1] < errs[0] / 3  # at least second order


@pytest.mark.parametrize("nod", [3, 6])
def test_ice_stream_analytic(nod):
    """Simple1dIceStreamSolution.m: grounded n=m=1 stream with calving front."""
    errs = []
    for nx in (21, 41):
        P, u_exact = ice_stream_problem(nx=nx, nod=nod)
        res = _solve_kat(P, nod)
        errs.append(np.max(np.abs(res.ub - u_exact)) / np.max(np.abs(u_exact)))
    assert errs[1] < (3e-3 if nod == 3 else 6e-5)
    assert errs[1] < errs[0] / 3


# --- Newton consistency --------------------------------------------------------------

@pytest.mark.parametrize("nod", [3, 6])
def test_tangent_is_derivative_of_residual(nod):
    """K equals the directional derivative of R (central difference) and is symmetric."""
    Pb = synth.ice_stream_shelf(9, 6, nod=nod, seed=3)
    mua = R.create_mua(Pb.coordinates, Pb.connectivity)
    rng = np.random.default_rng(1)
    F = R.prepare_fields(R.Params(), R.Fields(h=Pb.h, S=Pb.S, B=Pb.B, rho=Pb.rho, AGlen=Pb.AGlen, n=Pb.n,
                                              C=Pb.C, m=Pb.m, ub=100 + 50 * rng.random(mua.Nnodes),
                                              vb=20 * rng.standard_normal(mua.Nnodes)))
    p = R.Params()
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


def test_newton_converges_quadratically():
    P = synth.ice_stream_shelf(21, 11, seed=0)
    mua = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    F = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    res = R.uv(p, mua, bcs, F)
    assert res.converged
    r = [rec.r for rec in res.records]
    assert r[-1] < 1e-20
    # last steps: r_{k+1} <= C r_k^2 style reduction (ratio r/r0 falls super-linearly)
    assert res.records[-1].r / res.records[-1].r0 < 1e-6


# --- uvh (implicit transient) ---------------------------------------------------------

@pytest.mark.parametrize("nod", [3, 6])
def test_uvh_tangent_is_reference_jacobian(nod):
    """K of uvhMatrixAssembly matches the finite-difference derivative of R up to the
    term the reference leaves out: the h-derivative of b inside t1 (uvhNodalLoopSSTREAM.m
    :141-157 keeps (rho - rhow*Dddh)*dbdx but not (rho*h - rhow*d)*d(dbdx)/dh), which
    vanishes for floating ice and for grounded ice away from the grounding line."""
    Pb = synth.ice_stream_shelf(13, 7, nod=nod, seed=0, transient=True)
    mua = R.create_mua(Pb.coordinates, Pb.connectivity)
    rng = np.random.default_rng(1)
    F = R.Fields(h=Pb.h, S=Pb.S, B=Pb.B, rho=Pb.rho, AGlen=Pb.AGlen, n=Pb.n, C=Pb.C, m=Pb.m, ub=Pb.ub, vb=Pb.vb)
    N = mua.Nnodes
    S0 = R.UvhState(Pb.h.copy(), 100 + 50 * rng.random(N), 20 * rng.standard_normal(N), Pb.as_, Pb.ab)
    S1 = R.UvhState(Pb.h + 5 * rng.standard_normal(N), 100 + 50 * rng.random(N), 20 * rng.standard_normal(N),
                    Pb.as_, Pb.ab)
    p = R.Params()
    Rv, K = R.uvh_matrix_assembly(p, mua, F, S0, S1, 0.1)
    d = rng.standard_normal(3 * N)

    def Rat(eps):
        S = S1.copy()
        S.ub = S1.ub + eps * d[:N]; S.vb = S1.vb + eps * d[N:2 * N]; S.h = S1.h + eps * d[2 * N:]
        return R.uvh_matrix_assembly(p, mua, F, S0, S, 0.1, Ronly=True)[0]

    fd = (Rat(1e-3) - Rat(-1e-3)) / 2e-3
    assert np.linalg.norm(fd - K @ d) < 1e-3 * np.linalg.norm(K @ d)
    # the velocity blocks are exact: perturb u, v only
    d[2 * N:] = 0
    fd = (Rat(1e-3) - Rat(-1e-3)) / 2e-3
    assert np.linalg.norm(fd - K @ d) < 1e-6 * np.linalg.norm(K @ d)


def test_uvh_newton_converges():
    P = synth.ice_stream_shelf(21, 11, nod=3, seed=0, transient=True)
    mua = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    p.uvhDesiredWorkAndForceTolerances = (np.inf, 1e-20)
    p.uvhDesiredWorkOrForceTolerances = (np.inf, 1e-20)
    F = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    uv = R.uv(p, mua, bcs, F)
    S0 = R.UvhState(P.h.copy(), uv.ub, uv.vb, P.as_, P.ab)
    res = R.sstream_transient_implicit(p, mua, bcs, F, S0, S0.copy(), 0.1)
    assert res.converged and res.records[-1].rForce < 1e-20
    # mass conservation sanity: with u=v from the diagnostic state, h changes by O(dt*div(q))
    assert np.all(np.isfinite(res.h))
