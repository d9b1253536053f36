"""Parity of the CUDA path with the oracle beyond the golden toy meshes.

* The MATLAB sparsity pattern: after exact zeros are dropped (MATLAB's
  ``sparse`` keeps non-zeros only, ``sparseUA.m:17``), the GPU tangent's
  compressed-column arrays equal the oracle's, index for index
  (``uvMatrixAssemblySSTREAM.m:496-534``).  Checked on the golden meshes and
  on the full 141x71-vertex diagnostic workload, at u=v=0 (where the
  viscous couplings of a structured mesh cancel exactly) and at a perturbed
  solution.
* K and R within 1e-12 (per-row max-norm relative) on the full workload.
* The uvh implicit step on a 41x21-vertex P2 mesh (1,600 elements): K, R and
  the pattern at a perturbed state, and u, v, h after convergence within
  1e-10 relative L2.
* The Newton trajectory: with the inner solve held at a fixed tight tolerance
  (no forcing term), every iteration's backtracking count and step length
  equal the oracle's, rForce agrees to the stated tolerance, and the Newton
  update gamma*[du; dv; dl] returned through ua_newton_report.updates agrees
  with the oracle's (``SSTREAM2dNR2.m:367-369``).

All GPU calls go through the C-ABI (ctypes).
"""
import glob
import os

import numpy as np
import pytest
import scipy.sparse as sp

import uasource_b200 as ua
from oracle import ua_ref as R
from uasource_b200 import synth
from uasource_b200 import lib as L

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
UV_FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "uv_*.npz")))

K_TOL = 1e-12
R_TOL = 1e-12
U_TOL = 1e-10
# Newton trajectory with a fixed inner tolerance of 1e-13: step lengths to 1e-8 absolute,
# rForce to 1e-6 relative while it is above 1e-12 of its first value (below that the
# difference of the inner solves, about 1e-13 of each direction, dominates the residual),
# updates to 1e-7 of the first update's norm.
GAMMA_TOL = 1e-8
RFORCE_TOL = 1e-6
UPDATE_TOL = 1e-7


def _row_rel(Kg, Kr):
    D = (sp.csr_matrix(Kg) - sp.csr_matrix(Kr)).tocsr()
    scale = np.maximum(abs(sp.csr_matrix(Kr)).max(axis=1).toarray().ravel(), 1e-300)
    return np.max(abs(D).max(axis=1).toarray().ravel() / scale)


def _matlab_csc(K):
    """(jc, ir) of MATLAB's sparse double: CSC, sorted row indices, no stored zeros."""
    A = sp.csc_matrix(K, copy=True)
    A.sum_duplicates()
    A.eliminate_zeros()
    A.sort_indices()
    return A.indptr.astype(np.int64), A.indices.astype(np.int64)


def _assert_same_pattern(Kg, Kref):
    jc, ir = _matlab_csc(Kg)
    jc_r, ir_r = _matlab_csc(Kref)
    assert np.array_equal(jc, jc_r), "column pointers differ"
    assert np.array_equal(ir, ir_r), "row indices differ"


def _oracle_fields(P, ub=None, vb=None):
    return R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m,
                    ub=P.ub if ub is None else ub, vb=P.vb if vb is None else vb)


def _oracle_bcs(P):
    return R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                 vbFixedValue=P.vbFixedValue)


def _perturbed(ub, vb, seed):
    rng = np.random.default_rng(seed)
    n = ub.size
    return (ub * (1 + 0.1 * rng.standard_normal(n)) + 5 * rng.standard_normal(n),
            vb * (1 + 0.1 * rng.standard_normal(n)) + 5 * rng.standard_normal(n))


def _compare_uv_assembly(P, mua_g, mua_o, ub, vb):
    p = R.Params()
    Fo = R.prepare_fields(p, _oracle_fields(P, ub, vb))
    Rref, Kref, Tref, _ = R.uv_matrix_assembly(p, mua_o, Fo, return_parts=True)
    F = ua.Fields.from_problem(P)
    F.ub, F.vb = ub, vb
    Rg, Kg = ua.uvMatrixAssembly(ua.CtrlVar(), mua_g, F)
    assert _row_rel(Kg, Kref) <= K_TOL
    assert np.max(np.abs(Rg - Rref)) <= R_TOL * max(np.max(np.abs(Rref)), np.max(np.abs(Tref)))
    _assert_same_pattern(Kg, Kref)
    return Kg


# ----------------------------------------------------------------------------- pattern on the golden meshes

@pytest.mark.parametrize("state", ["golden", "zero"])
@pytest.mark.parametrize("path", UV_FIXTURES, ids=[os.path.basename(p) for p in UV_FIXTURES])
def test_pattern_after_zero_drop_equals_oracle_on_golden_meshes(path, state):
    z = np.load(path)
    mua = ua.CreateMUA(z["coordinates"], z["connectivity"])
    F = ua.Fields(h=z["h"], S=z["S"], B=z["B"], rho=z["rho"], AGlen=z["AGlen"], n=z["n"], C=z["C"], m=z["m"],
                  ub=np.zeros(len(z["h"])), vb=np.zeros(len(z["h"])), rhow=float(z["rhow"]), g=float(z["g"]))
    if state == "golden":
        F.ub, F.vb = z["state_ub"], z["state_vb"]
        Kref = sp.coo_matrix((z["K_val"], (z["K_row"], z["K_col"])), shape=(2 * len(z["h"]),) * 2)
    else:
        m = R.create_mua(z["coordinates"], z["connectivity"])
        p = R.Params()
        Fo = R.prepare_fields(p, R.Fields(h=z["h"], S=z["S"], B=z["B"], rho=z["rho"], AGlen=z["AGlen"], n=z["n"],
                                          C=z["C"], m=z["m"], ub=F.ub, vb=F.vb))
        _, Kref = R.uv_matrix_assembly(p, m, Fo)
    _, Kg = ua.uvMatrixAssembly(ua.CtrlVar(), mua, F)
    assert _row_rel(Kg, Kref) <= K_TOL
    _assert_same_pattern(Kg, Kref)
    # the C-ABI's structural pattern holds at least the MATLAB pattern
    assert Kg.nnz >= sp.csc_matrix(Kref).nnz


# ----------------------------------------------------------------------------- the full diagnostic workload

@pytest.fixture(scope="module")
def c0():
    """The 141x71-vertex diagnostic workload (19,600 P1 elements) and the oracle's Newton solve of it."""
    P = synth.ice_stream_shelf(141, 71, nod=3, seed=0)
    mua_o = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    ref = R.uv(p, mua_o, _oracle_bcs(P), _oracle_fields(P))
    assert ref.converged
    mua_g = ua.CreateMUA(P.coordinates, P.connectivity)
    return P, mua_o, mua_g, ref


def test_c0_assembly_and_pattern_at_zero_velocity(c0):
    P, mua_o, mua_g, _ = c0
    Kg = _compare_uv_assembly(P, mua_g, mua_o, np.zeros(P.Nnodes), np.zeros(P.Nnodes))
    # u=v=0 is the case with exact cancellations: the structural pattern is larger than MATLAB's
    assert mua_g.pattern()[1].size > _matlab_csc(Kg)[1].size


def test_c0_assembly_and_pattern_at_a_perturbed_solution(c0):
    P, mua_o, mua_g, ref = c0
    ub, vb = _perturbed(ref.ub, ref.vb, 7)
    _compare_uv_assembly(P, mua_g, mua_o, ub, vb)


def test_c0_newton_trajectory_and_updates_match_oracle(c0):
    """Fixed inner tolerance (no forcing term): the GPU takes the oracle's Newton path."""
    P, _, mua_g, ref = c0
    ctrl = ua.CtrlVar(krylov_adaptive=0, krylov_rtol=1e-13).set_force_tolerance(1e-20)
    Fg, lam, _, _, info = ua.uv(ctrl, mua_g, ua.BCs.from_problem(P), ua.Fields.from_problem(P),
                                return_updates=True)
    assert info.converged and not info.retried
    recs = ref.records
    assert info.iterations == ref.iterations == len(recs)
    assert len(info.iters) == len(recs)
    rF0 = recs[0].rForce
    for it, rr in zip(info.iters, recs):
        assert it["iteration"] == rr.iteration
        assert it["iarm"] == rr.iarm, (it, rr)
        assert abs(it["gamma"] - rr.gamma) <= GAMMA_TOL, (it, rr)
        if rr.rForce > 1e-12 * rF0:
            assert abs(it["rForce"] - rr.rForce) <= RFORCE_TOL * rr.rForce, (it, rr)
        else:
            assert it["rForce"] <= 1e-12 * rF0
    up = info.updates
    assert up.shape[0] == len(recs)
    scale = np.linalg.norm(recs[0].update)
    for k, rr in enumerate(recs):
        assert up[k].size == rr.update.size
        assert np.linalg.norm(up[k] - rr.update) <= UPDATE_TOL * scale, k
    # the updates add up to the solution from the start state (u=v=0 with the BCs imposed)
    u0 = np.zeros(2 * P.Nnodes)
    u0[P.ubFixedNode] = P.ubFixedValue
    u0[P.Nnodes + P.vbFixedNode] = P.vbFixedValue
    u = np.concatenate([Fg.ub, Fg.vb])
    assert np.linalg.norm(u0 + up[:, :2 * P.Nnodes].sum(axis=0) - u) <= 1e-12 * np.linalg.norm(u)
    assert np.linalg.norm(u - np.concatenate([ref.ub, ref.vb])) <= U_TOL * np.linalg.norm(u)


def test_update_buffer_stride_is_checked(c0):
    P, _, mua_g, _ = c0
    import ctypes as C
    from uasource_b200 import ua as host
    lib = L.load()
    keep = host._Keep()
    cf, _, _ = host._c_fields(ua.Fields.from_problem(P), keep, P.Nnodes)
    cb = host._c_bcs(ua.BCs.from_problem(P), keep)
    p = ua.CtrlVar().set_force_tolerance(1e-20).to_c()
    rep = L.ua_newton_report()
    buf = np.zeros((4, 10))
    rep.updates = buf.ctypes.data_as(C.POINTER(C.c_double))
    rep.update_stride = 10
    rc = lib.ua_uv_newton(mua_g.handle, C.byref(p), C.byref(cf), C.byref(cb), None, 0, C.byref(rep), None, None)
    assert rc == L.UA_ERR_INVALID
    assert b"update_stride" in lib.ua_last_error()


# ----------------------------------------------------------------------------- uvh on a 41x21-vertex P2 mesh

def _uvh_params():
    p = R.Params()
    p.set_force_tolerance(1e-20)
    p.uvhDesiredWorkAndForceTolerances = (np.inf, 1e-20)
    p.uvhDesiredWorkOrForceTolerances = (np.inf, 1e-20)
    return p


@pytest.fixture(scope="module")
def uvh41():
    """Implicit step dt = 0.1 a on the 41x21-vertex P2 mesh from the converged diagnostic state (oracle)."""
    P = synth.ice_stream_shelf(41, 21, nod=6, seed=0, transient=True)
    mua_o = R.create_mua(P.coordinates, P.connectivity)
    p = _uvh_params()
    Fo = _oracle_fields(P)
    uv = R.uv(p, mua_o, _oracle_bcs(P), Fo)
    assert uv.converged
    S0 = R.UvhState(P.h.copy(), uv.ub.copy(), uv.vb.copy(), P.as_.copy(), P.ab.copy())
    res = R.sstream_transient_implicit(p, mua_o, _oracle_bcs(P), Fo, S0, S0.copy(), 0.1)
    assert res.converged
    mua_g = ua.CreateMUA(P.coordinates, P.connectivity, ndof=3)
    return P, mua_o, mua_g, S0, res


def _uvh_gpu_levels(P, S0):
    F0 = ua.Fields.from_problem(P)
    F0.h, F0.ub, F0.vb = S0.h, S0.ub, S0.vb
    return F0, F0.copy()


def test_uvh_41x21_step_matches_oracle(uvh41):
    P, _, mua_g, S0, res = uvh41
    F0, F1 = _uvh_gpu_levels(P, S0)
    bcs = ua.HBCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                  vbFixedValue=P.vbFixedValue)
    ctrl = ua.CtrlVar().set_force_tolerance(1e-20).set_uvh_force_tolerance(1e-20)
    Fo, lam, info = ua.uvh(ctrl, mua_g, F0, F1, bcs, 0.1)
    assert info.converged
    ref = np.concatenate([res.ub, res.vb, res.h])
    got = np.concatenate([Fo.ub, Fo.vb, Fo.h])
    assert np.linalg.norm(got - ref) <= U_TOL * np.linalg.norm(ref)
    for a, b in ((Fo.ub, res.ub), (Fo.vb, res.vb), (Fo.h, res.h)):
        assert np.linalg.norm(a - b) <= U_TOL * np.linalg.norm(b)


def test_uvh_41x21_trajectory_and_updates_match_oracle(uvh41):
    P, _, mua_g, S0, res = uvh41
    F0, F1 = _uvh_gpu_levels(P, S0)
    bcs = ua.HBCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                  vbFixedValue=P.vbFixedValue)
    ctrl = ua.CtrlVar(krylov_adaptive=0, krylov_rtol=1e-13).set_force_tolerance(1e-20).set_uvh_force_tolerance(1e-20)
    Fo, _, info = ua.uvh(ctrl, mua_g, F0, F1, bcs, 0.1, return_updates=True)
    assert info.converged
    recs = res.records
    assert info.iterations == res.iterations == len(recs) == len(info.iters)
    rF0 = recs[0].rForce
    scale = np.linalg.norm(recs[0].update)
    for k, (it, rr) in enumerate(zip(info.iters, recs)):
        assert it["iarm"] == rr.iarm, (it, rr)
        assert abs(it["gamma"] - rr.gamma) <= GAMMA_TOL, (it, rr)
        if rr.rForce > 1e-12 * rF0:
            assert abs(it["rForce"] - rr.rForce) <= RFORCE_TOL * rr.rForce, (it, rr)
        assert np.linalg.norm(info.updates[k] - rr.update) <= UPDATE_TOL * scale, k


def test_uvh_41x21_assembly_and_pattern_match_oracle(uvh41):
    P, mua_o, mua_g, S0, res = uvh41
    rng = np.random.default_rng(5)
    n = P.Nnodes
    S1 = R.UvhState(res.h + 2 * rng.standard_normal(n), res.ub * (1 + 0.05 * rng.standard_normal(n)),
                    res.vb * (1 + 0.05 * rng.standard_normal(n)), P.as_.copy(), P.ab.copy())
    p = _uvh_params()
    Rref, Kref = R.uvh_matrix_assembly(p, mua_o, _oracle_fields(P), S0, S1, 0.1)
    F0, F1 = _uvh_gpu_levels(P, S0)
    F1.h, F1.ub, F1.vb = S1.h, S1.ub, S1.vb
    Rg, Kg = ua.uvhAssembly(ua.CtrlVar(), mua_g, F0, F1, 0.1)
    assert _row_rel(Kg, Kref) <= K_TOL
    assert np.max(np.abs(Rg - Rref)) <= R_TOL * np.max(np.abs(Rref))
    _assert_same_pattern(Kg, Kref)
