"""GPU parity of the uv assembly and Newton solve against the CPU oracle.

Every test calls libuassa.so through its C-ABI (via ctypes).  Tolerances:
K and R within 1e-12 (max-norm relative, per row), converged velocities
within 1e-10 relative L2 for the FP64 form and 1e-8 for the mixed form.
"""
import glob
import os

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ua_ref as R
from uasource_b200 import synth
import uasource_b200 as ua
from uasource_b200 import lib as L
from tests.kat_problems import ice_shelf_problem, ice_stream_problem

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "uv_*.npz")))

K_TOL = 1e-12
R_TOL = 1e-12
U_TOL_FP64 = 1e-10
U_TOL_MIXED = 1e-8


def _gpu_fields(z):
    return ua.Fields(h=z["h"], S=z["S"], B=z["B"], rho=z["rho"], AGlen=z["AGlen"], n=z["n"], C=z["C"], m=z["m"],
                     ub=np.zeros(len(z["h"])), vb=np.zeros(len(z["h"])), rhow=float(z["rhow"]), g=float(z["g"]))


def _gpu_bcs(z):
    return ua.BCs(ubFixedNode=z["ubFixedNode"], ubFixedValue=z["ubFixedValue"], vbFixedNode=z["vbFixedNode"],
                  vbFixedValue=z["vbFixedValue"])


def _compare_K(K_gpu, K_ref):
    """Per-row max-norm relative comparison on the union pattern; entries missing
    from the reference (exact zeros dropped by MATLAB's sparse) must be ~0."""
    D = (sp.csr_matrix(K_gpu) - sp.csr_matrix(K_ref)).tocsr()
    Kr = sp.csr_matrix(K_ref)
    row_scale = np.maximum(abs(Kr).max(axis=1).toarray().ravel(), 1e-300)
    rd = abs(D).max(axis=1).toarray().ravel()
    return np.max(rd / row_scale)


def _oracle_case(z):
    mua = R.create_mua(z["coordinates"], z["connectivity"])
    return mua


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_assembly_matches_golden(path):
    z = np.load(path)
    mua = ua.CreateMUA(z["coordinates"], z["connectivity"])
    F = _gpu_fields(z)
    F.ub, F.vb = z["state_ub"], z["state_vb"]
    ctrl = ua.CtrlVar()
    Rg, Kg = ua.uvMatrixAssembly(ctrl, mua, F)
    Kz = sp.coo_matrix((z["K_val"], (z["K_row"], z["K_col"])), shape=Kg.shape)
    assert _compare_K(Kg, Kz) <= K_TOL
    assert np.max(np.abs(Rg - z["R"])) <= R_TOL * np.max(np.abs(z["R"]))
    # pattern: the structural pattern holds the reference's non-zeros
    rp, ci = mua.pattern()
    S = sp.csr_matrix((np.ones(ci.size), ci, rp), shape=Kg.shape)
    Kzc = sp.csr_matrix(Kz)
    Kzc.eliminate_zeros()
    assert (abs(Kzc).sign() - abs(Kzc).sign().multiply(S)).nnz == 0
    # exactly symmetric (the reference symmetrises with (K+K.')/2)
    assert abs(Kg - Kg.T).max() == 0.0
    # residual-only mode gives the same R
    Rr, Kr = ua.uvMatrixAssembly(ctrl, mua, F, Ronly=True)
    assert Kr is None and np.array_equal(Rr, Rg)


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_newton_matches_golden(path):
    z = np.load(path)
    mua = ua.CreateMUA(z["coordinates"], z["connectivity"])
    ctrl = ua.CtrlVar().set_force_tolerance(1e-20)
    Fo, lam, _, _, info = ua.uv(ctrl, mua, _gpu_bcs(z), _gpu_fields(z))
    assert info.converged
    u_ref = np.concatenate([z["sol_ub"], z["sol_vb"]])
    u = np.concatenate([Fo.ub, Fo.vb])
    assert np.linalg.norm(u - u_ref) <= U_TOL_FP64 * np.linalg.norm(u_ref)
    assert np.linalg.norm(lam - z["sol_l"]) <= 1e-8 * max(np.linalg.norm(z["sol_l"]), 1.0)
    assert abs(info.iterations - int(z["sol_iterations"])) <= 2  # inexact-Newton inner tolerance


def test_zero_fields_and_parts_match_oracle():
    P = synth.ice_stream_shelf(15, 8, nod=3, seed=4)
    mua_o = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    rng = np.random.default_rng(3)
    ub = 100 * rng.random(P.Nnodes); vb = 10 * rng.standard_normal(P.Nnodes)
    Fo = R.prepare_fields(p, R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m,
                                      ub=ub, vb=vb))
    bo = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue + 7.0, vbFixedNode=P.vbFixedNode,
               vbFixedValue=P.vbFixedValue)
    R0, _ = R.uv_matrix_assembly(p, mua_o, Fo, bo, Ronly=True, ZeroFields=True)
    Rv, _, T, Fx = R.uv_matrix_assembly(p, mua_o, Fo, return_parts=True)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P); F.ub, F.vb = ub, vb
    bg = ua.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue + 7.0, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    ctrl = ua.CtrlVar()
    Rg0, _ = ua.uvMatrixAssembly(ctrl, mua, F, bg, Ronly=True, ZeroFields=True)
    assert np.max(np.abs(Rg0 - R0)) <= R_TOL * np.max(np.abs(R0))
    Rg, _, Tg, Fg = ua.uvMatrixAssembly(ctrl, mua, F, Ronly=True, return_parts=True)
    assert np.max(np.abs(Tg - T)) <= R_TOL * np.max(np.abs(T))
    assert np.max(np.abs(Fg - Fx)) <= R_TOL * np.max(np.abs(Fx))


def test_diagnostic_workload_matches_oracle():
    """The full diagnostic workload (141x71 vertices, ~20k P1 elements)."""
    P = synth.ice_stream_shelf(141, 71, nod=3, seed=0)
    mua_o = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params(); p.set_force_tolerance(1e-20)
    Fo = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bo = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
               vbFixedValue=P.vbFixedValue)
    ref = R.uv(p, mua_o, bo, Fo)
    assert ref.converged
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    ctrl = ua.CtrlVar().set_force_tolerance(1e-20)
    Fg, lam, Kg, Rg, info = ua.uv(ctrl, mua, ua.BCs.from_problem(P), ua.Fields.from_problem(P), return_K=True)
    assert info.converged and info.rForce < 1e-20
    u_ref = np.concatenate([ref.ub, ref.vb]); u = np.concatenate([Fg.ub, Fg.vb])
    assert np.linalg.norm(u - u_ref) <= U_TOL_FP64 * np.linalg.norm(u_ref)
    # the returned tangent is the last one assembled (SSTREAM2dNR2 returns Kuv)
    assert Kg is not None and Kg.nnz == mua.pattern()[1].size
    # mixed precision form against the FP64 oracle
    ctrl_m = ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20)
    Fm, _, _, _, info_m = ua.uv(ctrl_m, mua, ua.BCs.from_problem(P), ua.Fields.from_problem(P))
    assert info_m.converged
    um = np.concatenate([Fm.ub, Fm.vb])
    assert np.linalg.norm(um - u_ref) <= U_TOL_MIXED * np.linalg.norm(u_ref)


def test_p2_mixed_precision():
    z = np.load(os.path.join(HERE, "golden", "uv_P2_9x6.npz"))
    mua = ua.CreateMUA(z["coordinates"], z["connectivity"])
    ctrl = ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20)
    Fo, _, _, _, info = ua.uv(ctrl, mua, _gpu_bcs(z), _gpu_fields(z))
    assert info.converged
    u_ref = np.concatenate([z["sol_ub"], z["sol_vb"]]); u = np.concatenate([Fo.ub, Fo.vb])
    assert np.linalg.norm(u - u_ref) <= U_TOL_MIXED * np.linalg.norm(u_ref)


def test_batch_is_bit_identical_to_alone():
    """Each system's result is the same alone and in a batch of uneven meshes."""
    probs = [synth.ice_stream_shelf(21, 11, seed=0), synth.ice_stream_shelf(31, 16, seed=5),
             synth.ice_stream_shelf(15, 8, seed=9)]
    ctrl = ua.CtrlVar().set_force_tolerance(1e-20)
    alone = []
    for P in probs:
        mua = ua.CreateMUA(P.coordinates, P.connectivity)
        Fo, _, _, _, info = ua.uv(ctrl, mua, ua.BCs.from_problem(P), ua.Fields.from_problem(P))
        assert info.converged
        alone.append(np.concatenate([Fo.ub, Fo.vb]))
    batch = ua.CreateMUABatch([(P.coordinates, P.connectivity) for P in probs])
    out = ua.uv_batch(ctrl, batch, [ua.Fields.from_problem(P) for P in probs], [ua.BCs.from_problem(P) for P in probs])
    for k, (ub, vb, info) in enumerate(out):
        assert info.converged
        assert np.array_equal(np.concatenate([ub, vb]), alone[k])
    # caller-owned output arrays (ua_fields.ub_out/vb_out): same solutions, start velocities untouched
    Fs = [ua.Fields.from_problem(P) for P in probs]
    for F in Fs:
        F.ub = np.full(F.ub.shape, 5.0)
        F.vb = np.full(F.vb.shape, -2.0)
    dst = [(np.full(P.Nnodes, np.nan), np.full(P.Nnodes, np.nan)) for P in probs]
    out2 = ua.uv_batch(ctrl, batch, Fs, [ua.BCs.from_problem(P) for P in probs], out=dst)
    for k, (ub, vb, info) in enumerate(out2):
        assert info.converged and ub is dst[k][0] and vb is dst[k][1]
        assert np.all(Fs[k].ub == 5.0) and np.all(Fs[k].vb == -2.0)
        ref = ua.uv(ctrl, ua.CreateMUA(probs[k].coordinates, probs[k].connectivity), ua.BCs.from_problem(probs[k]),
                    Fs[k].copy())[0]
        assert np.array_equal(ub, ref.ub) and np.array_equal(vb, ref.vb)


def test_repeat_is_deterministic():
    P = synth.ice_stream_shelf(31, 16, seed=2)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)
    rng = np.random.default_rng(0)
    F.ub = 1000 * rng.random(P.Nnodes); F.vb = 100 * rng.standard_normal(P.Nnodes)
    a = ua.uvMatrixAssembly(ua.CtrlVar(), mua, F)
    b = ua.uvMatrixAssembly(ua.CtrlVar(), mua, F)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1].data, b[1].data)


def test_inside_out_elements_are_flipped():
    P = synth.ice_stream_shelf(15, 8, seed=1)
    conn = P.connectivity.copy()
    conn[::3] = conn[::3][:, [0, 2, 1]]           # make every third element inside-out
    mua = ua.CreateMUA(P.coordinates, conn)
    assert mua.flipped() == len(conn[::3])
    mua_ok = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)
    F.ub = np.linspace(0, 100, P.Nnodes); F.vb = np.linspace(0, 10, P.Nnodes)
    Ra, _ = ua.uvMatrixAssembly(ua.CtrlVar(), mua, F, Ronly=True)
    Rb, _ = ua.uvMatrixAssembly(ua.CtrlVar(), mua_ok, F, Ronly=True)
    assert np.max(np.abs(Ra - Rb)) <= 1e-12 * np.max(np.abs(Rb))


def test_nan_inputs_are_rejected():
    P = synth.ice_stream_shelf(15, 8, seed=1)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)
    F.ub = F.ub.copy(); F.ub[3] = np.nan
    with pytest.raises(ua.UaError) as e:
        ua.uvMatrixAssembly(ua.CtrlVar(), mua, F)
    assert e.value.code == L.UA_ERR_NAN_INPUT and "uvMatrixAssembly:NaN" in str(e.value)
    F = ua.Fields.from_problem(P)
    F.C = F.C.copy(); F.C[5] = np.nan
    with pytest.raises(ua.UaError) as e:
        ua.uv(ua.CtrlVar(), mua, ua.BCs.from_problem(P), F)
    assert e.value.code == L.UA_ERR_NAN_INPUT


def test_nan_inputs_are_rejected_in_a_batch():
    """The NaN tests of a batch's host fields run on the device after the upload and report what
    a scan on the host would: fields before velocities, the lowest system first; the handle then
    solves clean inputs."""
    probs = [synth.ice_stream_shelf(15, 8, seed=s) for s in (1, 2, 3)]
    batch = ua.CreateMUABatch([(P.coordinates, P.connectivity) for P in probs])
    bcs = [ua.BCs.from_problem(P) for P in probs]
    Fs = [ua.Fields.from_problem(P) for P in probs]
    Fs[2].h = Fs[2].h.copy(); Fs[2].h[4] = np.nan
    Fs[1].C = Fs[1].C.copy(); Fs[1].C[7] = np.nan
    Fs[0].ub = Fs[0].ub.copy(); Fs[0].ub[2] = np.nan
    with pytest.raises(ua.UaError) as e:
        ua.uv_batch(ua.CtrlVar(), batch, Fs, bcs)
    assert e.value.code == L.UA_ERR_NAN_INPUT and "nan in C (system 1)" in str(e.value)
    Fs = [ua.Fields.from_problem(P) for P in probs]
    Fs[2].vb = Fs[2].vb.copy(); Fs[2].vb[0] = np.nan
    with pytest.raises(ua.UaError) as e:
        ua.uv_batch(ua.CtrlVar(), batch, Fs, bcs)
    assert e.value.code == L.UA_ERR_NAN_INPUT and "uvMatrixAssembly:NaN" in str(e.value)
    out = ua.uv_batch(ua.CtrlVar().set_force_tolerance(1e-20), batch, [ua.Fields.from_problem(P) for P in probs], bcs)
    assert all(o[2].converged for o in out)


def test_bad_mesh_is_rejected():
    coords = np.array([[0, 0], [1, 0], [2, 0.0]])
    with pytest.raises(ua.UaError) as e:
        ua.CreateMUA(coords, np.array([[0, 1, 2]]))
    assert e.value.code == L.UA_ERR_BAD_MESH


def test_iteration_cap_reports_not_converged():
    """NRitmax reached: converged=0 and the reset-and-retry of uv.m:107-112 runs."""
    P = synth.ice_stream_shelf(21, 11, seed=0)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    ctrl = ua.CtrlVar(NRitmax=2).set_force_tolerance(1e-20)
    _, _, _, _, info = ua.uv(ctrl, mua, ua.BCs.from_problem(P), ua.Fields.from_problem(P))
    assert not info.converged and info.retried


def test_solve_kape_symmetric_examples():
    """TestABfgPreEliminate.m: [A B';B 0][x;y]=[f;g] examples."""
    A = sp.csr_matrix(np.diag([0, 0, 1.0, 1.0]))
    A = A + sp.csr_matrix((np.zeros(2), ([0, 1], [0, 1])), shape=(4, 4))  # explicit diagonal entries
    B = sp.csr_matrix(np.array([[1, 0, 0, 0], [0, 1, 0, 0.0]]))
    x, y, its = ua.solveKApeSymmetric(A, B, np.array([10, 2, 10, 1000.0]), np.array([10, 10.0]))
    assert np.allclose(x, [10, 10, 10, 1000]) and np.allclose(y, [10, 2])
    # an SPD system with a scaled selection constraint against a dense solve
    rng = np.random.default_rng(0)
    M = rng.standard_normal((30, 30)); A = sp.csr_matrix(M @ M.T + 30 * np.eye(30))
    B = sp.csr_matrix((np.array([2.0, -3.0]), ([0, 1], [4, 17])), shape=(2, 30))
    f = rng.standard_normal(30); g = rng.standard_normal(2)
    x, y, its = ua.solveKApeSymmetric(A, B, f, g)
    T = np.block([[A.toarray(), B.toarray().T], [B.toarray(), np.zeros((2, 2))]])
    sol = np.linalg.solve(T, np.concatenate([f, g]))
    assert np.allclose(np.concatenate([x, y]), sol, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("nod", [3, 6])
def test_analytic_ice_shelf_on_gpu(nod):
    P, u_exact = ice_shelf_problem(nx=41, nod=nod)
    mua = ua.CreateMUA(P["coordinates"], P["connectivity"])
    F = ua.Fields(h=P["h"], S=P["S"], B=P["B"], rho=P["rho"], AGlen=P["AGlen"], n=P["n"], C=P["C"], m=P["m"],
                  ub=P["ub"], vb=P["vb"], rhow=P["rhow"], g=P["g"])
    b = ua.BCs(ubFixedNode=P["ubFixedNode"], ubFixedValue=P["ubFixedValue"], vbFixedNode=P["vbFixedNode"],
               vbFixedValue=P["vbFixedValue"])
    ctrl = ua.CtrlVar(etaZero=0.0).set_force_tolerance(1e-24)
    Fo, _, _, _, info = ua.uv(ctrl, mua, b, F)
    assert info.converged
    err = np.max(np.abs(Fo.ub - u_exact)) / np.max(u_exact)
    assert err < (2e-4 if nod == 3 else 5e-6)


@pytest.mark.parametrize("nod", [3, 6])
def test_analytic_ice_stream_on_gpu(nod):
    P, u_exact = ice_stream_problem(nx=41, nod=nod)
    mua = ua.CreateMUA(P["coordinates"], P["connectivity"])
    F = ua.Fields(h=P["h"], S=P["S"], B=P["B"], rho=P["rho"], AGlen=P["AGlen"], n=P["n"], C=P["C"], m=P["m"],
                  ub=P["ub"], vb=P["vb"], rhow=P["rhow"], g=P["g"])
    b = ua.BCs(ubFixedNode=P["ubFixedNode"], ubFixedValue=P["ubFixedValue"], vbFixedNode=P["vbFixedNode"],
               vbFixedValue=P["vbFixedValue"])
    ctrl = ua.CtrlVar(etaZero=0.0).set_force_tolerance(1e-24)
    Fo, _, _, _, info = ua.uv(ctrl, mua, b, F)
    assert info.converged
    err = np.max(np.abs(Fo.ub - u_exact)) / np.max(np.abs(u_exact))
    assert err < (3e-3 if nod == 3 else 6e-5)


@pytest.mark.parametrize("nod", [3, 6])
def test_amg_and_jacobi_preconditioners_agree(nod):
    """The aggregation-AMG and point-Jacobi inner solves reach the same Newton solution;
    AMG needs far fewer Krylov iterations."""
    P = synth.ice_stream_shelf(61, 31, nod=nod, seed=3)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    res = {}
    for pc in (L.UA_PC_JACOBI, L.UA_PC_AMG):
        ctrl = ua.CtrlVar(krylov_precond=pc).set_force_tolerance(1e-20)
        Fo, _, _, _, info = ua.uv(ctrl, mua, ua.BCs.from_problem(P), ua.Fields.from_problem(P))
        assert info.converged
        res[pc] = (np.concatenate([Fo.ub, Fo.vb]), info.krylov_its_total)
    uj, u_amg = res[L.UA_PC_JACOBI][0], res[L.UA_PC_AMG][0]
    assert np.linalg.norm(u_amg - uj) <= U_TOL_FP64 * np.linalg.norm(uj)
    assert res[L.UA_PC_AMG][1] * 3 < res[L.UA_PC_JACOBI][1]


@pytest.mark.parametrize("precision,rtol", [(L.UA_PREC_FP64, 1e-12), (L.UA_PREC_MIXED, 1e-6)])
def test_graph_replay_equals_direct_launches(precision, rtol):
    """PCG chunks replayed from a captured CUDA graph give bit-identical results to the
    same kernels launched one by one (profile=1 launches them directly)."""
    P = synth.ice_stream_shelf(41, 21, seed=4)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    out = []
    for prof in (0, 1, 0):
        ctrl = ua.CtrlVar(precision=precision, krylov_rtol=rtol, profile=prof).set_force_tolerance(1e-20)
        Fo, _, _, _, info = ua.uv(ctrl, mua, ua.BCs.from_problem(P), ua.Fields.from_problem(P))
        assert info.converged
        out.append(np.concatenate([Fo.ub, Fo.vb]))
        if prof:  # phase timings: the set-ups and the Krylov ranges, which hold the SpMVs
            k = info.kernels
            assert k["setup_n"] >= info.iterations and k["setup_ms"] > 0
            assert k["krylov_n"] >= info.iterations and k["krylov_ms"] >= k["spmv_ms"] > 0
            assert k["krylov_ms"] + k["setup_ms"] < info.device_ms
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


@pytest.mark.parametrize("precision,rtol", [(L.UA_PREC_FP64, 1e-12), (L.UA_PREC_MIXED, 1e-6)])
def test_active_block_lists_equal_full_grid(precision, rtol):
    """The PCG launched over the device-compacted lists of active row and node blocks gives
    bit-identical results and iteration counts to launching every block of the batch (a
    batch of uneven meshes, so systems converge at different iterations)."""
    probs = [synth.ice_stream_shelf(21, 11, seed=0), synth.ice_stream_shelf(41, 21, seed=5),
             synth.ice_stream_shelf(15, 8, seed=9), synth.ice_stream_shelf(31, 16, seed=2)]
    batch = ua.CreateMUABatch([(P.coordinates, P.connectivity) for P in probs])
    res = []
    for full in (0, 1):
        ctrl = ua.CtrlVar(precision=precision, krylov_rtol=rtol, krylov_full_grid=full).set_force_tolerance(1e-20)
        out = ua.uv_batch(ctrl, batch, [ua.Fields.from_problem(P) for P in probs],
                          [ua.BCs.from_problem(P) for P in probs])
        assert all(o[2].converged for o in out)
        res.append(([np.concatenate([o[0], o[1]]) for o in out], [o[2].krylov_its_total for o in out]))
    assert len(set(res[0][1])) > 1  # the systems finish at different PCG iterations
    assert res[0][1] == res[1][1]
    assert all(np.array_equal(a, b) for a, b in zip(res[0][0], res[1][0]))


@pytest.mark.parametrize("precision,rtol,tol", [(L.UA_PREC_FP64, 1e-12, U_TOL_FP64), (L.UA_PREC_MIXED, 1e-6, U_TOL_MIXED)])
def test_node_slices_agree_with_csr_kernels(precision, rtol, tol):
    """The node-sliced (sliced ELL) SpMV and finest-level V-cycle passes, both rows of a node
    per thread, give the CSR row kernels' solution within the form's tolerance on a batch of
    uneven meshes (P1 and P2), and a batch solve equals each mesh solved alone bit for bit."""
    probs = [synth.ice_stream_shelf(21, 11, seed=0), synth.ice_stream_shelf(41, 21, seed=5),
             synth.ice_stream_shelf(15, 8, seed=9), synth.ice_stream_shelf(9, 6, nod=6, seed=0)]
    res = {}
    for sell in (1, 0):
        ctrl = ua.CtrlVar(precision=precision, krylov_rtol=rtol, krylov_sell=sell).set_force_tolerance(1e-20)
        out = []
        for P in probs:
            mua = ua.CreateMUA(P.coordinates, P.connectivity)
            Fo, _, _, _, info = ua.uv(ctrl, mua, ua.BCs.from_problem(P), ua.Fields.from_problem(P))
            assert info.converged
            out.append(np.concatenate([Fo.ub, Fo.vb]))
        res[sell] = out
    for a, b in zip(res[1], res[0]):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < tol
    P2 = [p for p in probs if p.nod == 3]
    batch = ua.CreateMUABatch([(P.coordinates, P.connectivity) for P in P2])
    ctrl = ua.CtrlVar(precision=precision, krylov_rtol=rtol).set_force_tolerance(1e-20)
    outb = ua.uv_batch(ctrl, batch, [ua.Fields.from_problem(P) for P in P2], [ua.BCs.from_problem(P) for P in P2])
    for o, a in zip(outb, res[1][:len(P2)]):
        assert np.array_equal(np.concatenate([o[0], o[1]]), a)


@pytest.mark.parametrize("precision,rtol", [(L.UA_PREC_FP64, 1e-12), (L.UA_PREC_MIXED, 1e-6)])
def test_tangent_assembled_ahead_matches_assembly_per_iteration(precision, rtol):
    """With the tangent assembled ahead (K with R at the start iterate and at every full Newton
    step, used when that point is accepted) the solve takes the same Newton iterations and ends
    at the same solution as assembling K at the start of every iteration (the form used when
    the caller reads the last tangent back)."""
    for P in (synth.ice_stream_shelf(21, 11, seed=0), synth.ice_stream_shelf(41, 21, seed=5),
              synth.ice_stream_shelf(9, 6, nod=6, seed=0)):
        mua = ua.CreateMUA(P.coordinates, P.connectivity)
        ctrl = ua.CtrlVar(precision=precision, krylov_rtol=rtol).set_force_tolerance(1e-20)
        Fa, _, _, _, ia = ua.uv(ctrl, mua, ua.BCs.from_problem(P), ua.Fields.from_problem(P))
        Fb, _, Kb, _, ib = ua.uv(ctrl, mua, ua.BCs.from_problem(P), ua.Fields.from_problem(P), return_K=True)
        assert ia.converged and ib.converged and Kb is not None
        assert ia.iterations == ib.iterations
        a, b = np.concatenate([Fa.ub, Fa.vb]), np.concatenate([Fb.ub, Fb.vb])
        assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b)


@pytest.mark.parametrize("refresh", [1, 2, 100])
def test_prolongator_refresh_interval(refresh):
    """Prolongators kept over Newton steps (the coarse operators recomputed from each tangent):
    the solve converges to the same solution within the tolerance of the inner solve, FP64 and
    mixed, and a batch equals each mesh alone bit for bit with the interval in use."""
    probs = [synth.ice_stream_shelf(41, 21, seed=1), synth.ice_stream_shelf(21, 11, seed=6)]
    ref = []
    for P in probs:
        c = ua.CtrlVar(amg_P_refresh=1).set_force_tolerance(1e-20)
        Fo, _, _, _, info = ua.uv(c, ua.CreateMUA(P.coordinates, P.connectivity), ua.BCs.from_problem(P),
                                  ua.Fields.from_problem(P))
        ref.append(np.concatenate([Fo.ub, Fo.vb]))
    for prec, tol in ((L.UA_PREC_FP64, 1e-10), (L.UA_PREC_MIXED, 1e-8)):
        ctrl = ua.CtrlVar(precision=prec, krylov_rtol=1e-12 if prec == L.UA_PREC_FP64 else 1e-6,
                          amg_P_refresh=refresh).set_force_tolerance(1e-20)
        mb = ua.CreateMUABatch([(P.coordinates, P.connectivity) for P in probs])
        batch = ua.uv_batch(ctrl, mb, [ua.Fields.from_problem(P) for P in probs], [ua.BCs.from_problem(P) for P in probs])
        for k, P in enumerate(probs):
            Fo, _, _, _, info = ua.uv(ctrl, ua.CreateMUA(P.coordinates, P.connectivity), ua.BCs.from_problem(P),
                                      ua.Fields.from_problem(P))
            u = np.concatenate([Fo.ub, Fo.vb])
            assert info.converged and np.linalg.norm(u - ref[k]) <= tol * np.linalg.norm(ref[k])
            assert np.array_equal(batch[k][0], Fo.ub) and np.array_equal(batch[k][1], Fo.vb)
