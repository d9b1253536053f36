"""The MEX gateways run end to end on the GPU, outside MATLAB.

Each gateway under mex/ is built with a small C implementation of the mx*
calls (tests/mex_host/mxhost.c) into its own shared library and is called
with MATLAB-shaped arguments: structs of double column vectors, a 1-based
double connectivity, 1-based boundary-condition node lists.  What it returns
is what MATLAB would receive: the tangent as a sparse double (CSC jc/ir/pr,
sorted rows, no stored zeros) is compared index for index with the oracle's
MATLAB-semantics sparse matrix and value by value within 1e-12; the residual
is a sparse-typed column; the Newton gateways return the converged fields
(within 1e-10 of the oracle), the multipliers and the constraint matrix L.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ua_ref as R
from uasource_b200 import synth

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
HOST = os.path.join(HERE, "mex_host")
K_TOL = 1e-12
U_TOL = 1e-10
_mw = C.c_size_t
K_DOUBLE, K_SPARSE, K_STRUCT, K_CHAR = 1, 2, 3, 4


class Gateway:
    """One MEX gateway loaded through the mx host."""

    def __init__(self, name):
        path = os.path.join(HOST, "_build", f"lib{name}.so")
        lib = C.CDLL(path)
        vp = C.c_void_p
        for fn, res, args in (
            ("mxCreateDoubleMatrix", vp, [_mw, _mw, C.c_int]), ("mxCreateString", vp, [C.c_char_p]),
            ("mxCreateStructMatrix", vp, [_mw, _mw, C.c_int, C.POINTER(C.c_char_p)]),
            ("mxSetField", None, [vp, _mw, C.c_char_p, vp]), ("mxGetPr", C.POINTER(C.c_double), [vp]),
            ("mxGetJc", C.POINTER(_mw), [vp]), ("mxGetIr", C.POINTER(_mw), [vp]), ("mxGetM", _mw, [vp]),
            ("mxGetN", _mw, [vp]), ("mxDestroyArray", None, [vp]), ("mxArrayToString", C.c_char_p, [vp]),
            ("mxhost_call", C.c_int, [C.c_int, C.POINTER(vp), C.c_int, C.POINTER(vp)]),
            ("mxhost_error_id", C.c_char_p, []), ("mxhost_error_msg", C.c_char_p, []), ("mxhost_unload", None, []),
            ("mxhost_kind", C.c_int, [vp]), ("mxhost_nfields", C.c_int, [vp]),
            ("mxhost_field_name", C.c_char_p, [vp, C.c_int]), ("mxhost_field_value", vp, [vp, C.c_int])):
            f = getattr(lib, fn)
            f.restype = res
            f.argtypes = args
        self.lib = lib

    # ---- MATLAB values -> mxArray
    def double(self, a):
        a = np.asarray(a, dtype=np.float64)
        if a.ndim == 0:
            a = a.reshape(1, 1)
        elif a.ndim == 1:
            a = a.reshape(-1, 1)
        m, n = a.shape
        p = self.lib.mxCreateDoubleMatrix(m, n, 0)
        if m * n:
            af = np.asfortranarray(a)  # held until the copy is done: a temporary could be freed first
            C.memmove(self.lib.mxGetPr(p), af.ctypes.data, 8 * m * n)
        return p

    def struct(self, d):
        names = (C.c_char_p * len(d))(*[k.encode() for k in d])
        s = self.lib.mxCreateStructMatrix(1, 1, len(d), names)
        for k, v in d.items():
            if isinstance(v, dict):
                mv = self.struct(v)
            elif isinstance(v, str):
                mv = self.lib.mxCreateString(v.encode())
            else:
                mv = self.double(v)
            self.lib.mxSetField(s, 0, k.encode(), mv)
        return s

    # ---- mxArray -> Python
    def value(self, p):
        kind = self.lib.mxhost_kind(p)
        m, n = self.lib.mxGetM(p), self.lib.mxGetN(p)
        if kind == K_DOUBLE:
            return np.ctypeslib.as_array(self.lib.mxGetPr(p), shape=(m * n,)).reshape((m, n), order="F").copy() \
                if m * n else np.zeros((m, n))
        if kind == K_SPARSE:
            jc = np.ctypeslib.as_array(self.lib.mxGetJc(p), shape=(n + 1,)).astype(np.int64).copy()
            nz = int(jc[-1])
            ir = np.ctypeslib.as_array(self.lib.mxGetIr(p), shape=(max(nz, 1),))[:nz].astype(np.int64).copy()
            pr = np.ctypeslib.as_array(self.lib.mxGetPr(p), shape=(max(nz, 1),))[:nz].copy()
            return sp.csc_matrix((pr, ir, jc), shape=(m, n))
        if kind == K_CHAR:
            return self.lib.mxArrayToString(p).decode()
        if kind == K_STRUCT:
            return {self.lib.mxhost_field_name(p, k).decode(): self.value(self.lib.mxhost_field_value(p, k))
                    for k in range(self.lib.mxhost_nfields(p))}
        raise ValueError(kind)

    def __call__(self, nlhs, *args):
        prhs = (C.c_void_p * len(args))(*[a for a in args])
        plhs = (C.c_void_p * nlhs)()
        rc = self.lib.mxhost_call(nlhs, plhs, len(args), prhs)
        if rc:
            raise RuntimeError(f"{self.lib.mxhost_error_id().decode()}: {self.lib.mxhost_error_msg().decode()}")
        out = [self.value(plhs[k]) if plhs[k] else None for k in range(nlhs)]
        for k in range(nlhs):
            if plhs[k]:
                self.lib.mxDestroyArray(plhs[k])
        return out

    def close(self):
        self.lib.mxhost_unload()


@pytest.fixture(scope="module")
def gateways():
    r = subprocess.run(["make", "-C", HOST], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    g = {name: Gateway(name) for name in ("uvMatrixAssemblySSTREAM_mex", "SSTREAM2dNR2_mex", "uvhAssembly_mex",
                                          "SSTREAM_TransientImplicit_mex")}
    yield g
    for v in g.values():
        v.close()


def _mua(g, P):
    return g.struct({"coordinates": P.coordinates, "connectivity": P.connectivity.astype(np.float64) + 1})


def _F(P, ub=None, vb=None, extra=None):
    d = {"h": P.h, "S": P.S, "B": P.B, "rho": P.rho, "AGlen": P.AGlen, "n": P.n, "C": P.C, "m": P.m,
         "ub": P.ub if ub is None else ub, "vb": P.vb if vb is None else vb, "rhow": P.rhow, "g": P.g,
         "alpha": 0.0}
    d.update(extra or {})
    return d


def _bcs(P):
    return {"ubFixedNode": P.ubFixedNode + 1.0, "ubFixedValue": P.ubFixedValue,
            "vbFixedNode": P.vbFixedNode + 1.0, "vbFixedValue": P.vbFixedValue}


def _csc_equal(A, B, tol):
    A = sp.csc_matrix(A); B = sp.csc_matrix(B, copy=True)
    B.sum_duplicates(); B.eliminate_zeros(); B.sort_indices()
    assert A.shape == B.shape
    assert np.array_equal(A.indptr, B.indptr) and np.array_equal(A.indices, B.indices)
    Bd = B.data
    scale = np.maximum(abs(B).max(axis=0).toarray().ravel(), 1e-300)
    col = np.repeat(np.arange(B.shape[1]), np.diff(B.indptr))
    assert np.max(np.abs(A.data - Bd) / scale[col]) <= tol


@pytest.mark.parametrize("state", ["perturbed", "zero"])
def test_uv_assembly_gateway(gateways, state):
    g = gateways["uvMatrixAssemblySSTREAM_mex"]
    P = synth.ice_stream_shelf(21, 11, nod=3, seed=0)
    rng = np.random.default_rng(3)
    ub = 100 * rng.random(P.Nnodes) if state == "perturbed" else np.zeros(P.Nnodes)
    vb = 10 * rng.standard_normal(P.Nnodes) if state == "perturbed" else np.zeros(P.Nnodes)
    Rm, Km = g(2, g.struct({"kH": 1.0}), _mua(g, P), g.struct(_F(P, ub, vb)), g.struct(_bcs(P)))
    p = R.Params()
    Fo = R.prepare_fields(p, R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=ub,
                                      vb=vb))
    Rref, Kref = R.uv_matrix_assembly(p, R.create_mua(P.coordinates, P.connectivity), Fo)
    assert sp.issparse(Rm) and Rm.shape == (2 * P.Nnodes, 1)
    assert np.max(np.abs(Rm.toarray().ravel() - Rref)) <= K_TOL * np.max(np.abs(Rref))
    _csc_equal(Km, Kref, K_TOL)
    # Ronly: K is [] (0 x 0)
    Rr, Kr = g(2, g.struct({"uvMatrixAssembly": {"Ronly": 1.0}}), _mua(g, P), g.struct(_F(P, ub, vb)),
               g.struct(_bcs(P)))
    assert Kr.shape == (0, 0) and np.array_equal(Rr.toarray(), Rm.toarray())


def test_uv_assembly_gateway_sliding_law(gateways):
    g = gateways["uvMatrixAssemblySSTREAM_mex"]
    P = synth.ice_stream_shelf(15, 8, nod=3, seed=1)
    rng = np.random.default_rng(5)
    ub, vb = 100 * rng.random(P.Nnodes), 10 * rng.standard_normal(P.Nnodes)
    q = 1.0 + 0.1 * rng.random(P.Nnodes)
    Rm, Km = g(2, g.struct({"SlidingLaw": "Budd"}), _mua(g, P), g.struct(_F(P, ub, vb, {"q": q})),
               g.struct(_bcs(P)))
    p = R.Params()
    p.SlidingLaw = "Budd"
    Fo = R.prepare_fields(p, R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=ub,
                                      vb=vb, q=q))
    Rref, Kref = R.uv_matrix_assembly(p, R.create_mua(P.coordinates, P.connectivity), Fo)
    assert np.max(np.abs(Rm.toarray().ravel() - Rref)) <= K_TOL * np.max(np.abs(Rref))
    _csc_equal(Km, Kref, K_TOL)


def test_uv_assembly_gateway_reports_nan_with_the_reference_identifier(gateways):
    g = gateways["uvMatrixAssemblySSTREAM_mex"]
    P = synth.ice_stream_shelf(9, 6, nod=3, seed=0)
    ub = np.zeros(P.Nnodes); ub[3] = np.nan
    with pytest.raises(RuntimeError) as ei:
        g(2, g.struct({}), _mua(g, P), g.struct(_F(P, ub, np.zeros(P.Nnodes))), g.struct(_bcs(P)))
    assert str(ei.value).startswith("uvMatrixAssembly:NaN")


def test_newton_gateway(gateways):
    g = gateways["SSTREAM2dNR2_mex"]
    P = synth.ice_stream_shelf(21, 11, nod=3, seed=0)
    ctrl = {"uvDesiredWorkAndForceTolerances": [np.inf, 1e-20], "uvDesiredWorkOrForceTolerances": [np.inf, 1e-20],
            "uvAcceptableWorkAndForceTolerances": [np.inf, 1e-20],
            "uvAcceptableWorkOrForceTolerances": [np.inf, 1e-20]}
    ub, vb, lam, K, Rv, info, L = g(7, g.struct(ctrl), _mua(g, P), g.struct(_bcs(P)), g.struct(_F(P)),
                                    g.double(np.zeros((0, 0))))
    p = R.Params()
    p.set_force_tolerance(1e-20)
    ref = R.uv(p, R.create_mua(P.coordinates, P.connectivity),
               R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                     vbFixedValue=P.vbFixedValue),
               R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb))
    u = np.concatenate([ub.ravel(), vb.ravel()]); u_ref = np.concatenate([ref.ub, ref.vb])
    assert info["uvConverged"][0, 0] == 1
    assert np.linalg.norm(u - u_ref) <= U_TOL * np.linalg.norm(u_ref)
    assert np.linalg.norm(lam.ravel() - ref.lubvb) <= 1e-8 * max(np.linalg.norm(ref.lubvb), 1.0)
    # L: the reference's constraint matrix (AssembleLuvSSTREAM -> CreateLuv -> ScaleL), index for index
    Lc = sp.csc_matrix(ref.L)
    assert L.shape == Lc.shape
    _csc_equal(L, Lc, 0.0)
    assert sp.issparse(K) and K.shape == (2 * P.Nnodes, 2 * P.Nnodes) and sp.issparse(Rv)


def test_newton_gateway_with_ties_and_normals(gateways):
    """BCs.ubTiedNodeA/B and ubvbFixedNormalNode/Value through the gateway: the solution and the
    two-entry rows of L (CreateLuv.m:28-76, ScaleL.m) as the oracle has them."""
    from tests.constraint_cases import front_nodes, problem, tie_nodes
    g = gateways["SSTREAM2dNR2_mex"]
    P = problem(21, 11, 3, np.pi / 6)
    bottom, top = tie_nodes(P)
    fr = front_nodes(P)
    kw = dict(ubTiedNodeA=bottom[:-1], ubTiedNodeB=top[:-1], ubvbFixedNormalNode=fr,
              ubvbFixedNormalValue=np.zeros(fr.size))
    b = _bcs(P)
    b.update({"ubTiedNodeA": kw["ubTiedNodeA"] + 1.0, "ubTiedNodeB": kw["ubTiedNodeB"] + 1.0,
              "ubvbFixedNormalNode": fr + 1.0, "ubvbFixedNormalValue": np.zeros(fr.size)})
    ctrl = {"uvDesiredWorkAndForceTolerances": [np.inf, 1e-20], "uvDesiredWorkOrForceTolerances": [np.inf, 1e-20]}
    ub, vb, lam, K, Rv, info, L = g(7, g.struct(ctrl), _mua(g, P), g.struct(b), g.struct(_F(P)),
                                    g.double(np.zeros((0, 0))))
    p = R.Params()
    p.set_force_tolerance(1e-20)
    ref = R.uv(p, R.create_mua(P.coordinates, P.connectivity),
               R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                     vbFixedValue=P.vbFixedValue, **kw),
               R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb))
    u = np.concatenate([ub.ravel(), vb.ravel()]); u_ref = np.concatenate([ref.ub, ref.vb])
    assert info["uvConverged"][0, 0] == 1
    assert np.linalg.norm(u - u_ref) <= U_TOL * np.linalg.norm(u_ref)
    _csc_equal(L, sp.csc_matrix(ref.L), 1e-15)


def test_gateway_refuses_unequal_tie_lists(gateways):
    g = gateways["SSTREAM2dNR2_mex"]
    P = synth.ice_stream_shelf(9, 6, nod=3, seed=0)
    b = _bcs(P)
    b.update({"ubTiedNodeA": np.array([2.0, 3.0]), "ubTiedNodeB": np.array([5.0])})
    with pytest.raises(RuntimeError) as ei:
        g(7, g.struct({}), _mua(g, P), g.struct(b), g.struct(_F(P)), g.double(np.zeros((0, 0))))
    assert str(ei.value).startswith("Ua:mex:BCs")


def _uvh_fixture():
    import glob
    path = sorted(glob.glob(os.path.join(HERE, "golden", "uvh_P2_*.npz")))[0]
    return np.load(path)


def _uvh_F(z, level):
    if level == 0:
        h, ub, vb = z["h0"], z["u0"], z["v0"]
    else:
        h, ub, vb = z["state_h"], z["state_ub"], z["state_vb"]
    return {"h": h, "S": z["S"], "B": z["B"], "rho": z["rho"], "AGlen": z["AGlen"], "n": z["n"], "C": z["C"],
            "m": z["m"], "ub": ub, "vb": vb, "rhow": float(z["rhow"]), "g": float(z["g"]), "alpha": 0.0,
            "as": z["as_"], "ab": z["ab"]}


def test_uvh_assembly_gateway(gateways):
    g = gateways["uvhAssembly_mex"]
    z = _uvh_fixture()
    Rm, Km = g(2, g.struct({"dt": float(z["dt"])}),
               g.struct({"coordinates": z["coordinates"], "connectivity": z["connectivity"] + 1.0}),
               g.struct(_uvh_F(z, 0)), g.struct(_uvh_F(z, 1)))
    Kref = sp.coo_matrix((z["K_val"], (z["K_row"], z["K_col"])), shape=Km.shape)
    assert np.max(np.abs(Rm.toarray().ravel() - z["R"])) <= K_TOL * np.max(np.abs(z["R"]))
    _csc_equal(Km, Kref, K_TOL)


def test_uvh_newton_gateway(gateways):
    g = gateways["SSTREAM_TransientImplicit_mex"]
    z = _uvh_fixture()
    F1 = _uvh_F(z, 0)  # the step starts from the state at t
    ctrl = {"dt": float(z["dt"]), "uvhDesiredWorkAndForceTolerances": [np.inf, 1e-20],
            "uvhDesiredWorkOrForceTolerances": [np.inf, 1e-20]}
    bcs = {"ubFixedNode": z["ubFixedNode"] + 1.0, "ubFixedValue": z["ubFixedValue"],
           "vbFixedNode": z["vbFixedNode"] + 1.0, "vbFixedValue": z["vbFixedValue"]}
    ub, vb, h, lam, info = g(5, g.struct(ctrl),
                             g.struct({"coordinates": z["coordinates"], "connectivity": z["connectivity"] + 1.0}),
                             g.struct(bcs), g.struct(_uvh_F(z, 0)), g.struct(F1), g.double(np.zeros((0, 0))))
    got = np.concatenate([ub.ravel(), vb.ravel(), h.ravel()])
    ref = np.concatenate([z["sol_ub"], z["sol_vb"], z["sol_h"]])
    assert np.linalg.norm(got - ref) <= U_TOL * np.linalg.norm(ref)


def test_uvh_newton_gateway_active_set(gateways):
    """CtrlVar.ThicknessConstraints through the gateway: the final BCs1.hPosNode (1-based) and
    the step match the oracle's active-set loop (uvh.m:64-212)."""
    from tests.active_set_cases import thin_patch_problem
    g = gateways["SSTREAM_TransientImplicit_mex"]
    P, h, as_ = thin_patch_problem()
    p = R.Params()
    p.set_force_tolerance(1e-20)
    p.uvhDesiredWorkAndForceTolerances = (np.inf, 1e-20)
    p.uvhDesiredWorkOrForceTolerances = (np.inf, 1e-20)
    mo = R.create_mua(P.coordinates, P.connectivity)
    Fo = R.Fields(h=h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bo = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
               vbFixedValue=P.vbFixedValue)
    uv = R.uv(p, mo, bo, Fo)
    S0 = R.UvhState(h.copy(), uv.ub.copy(), uv.vb.copy(), as_.copy(), P.ab.copy())
    ref = R.uvh_active_set(p, mo, bo, Fo, S0, S0.copy(), 0.1)
    assert ref.converged and ref.hPosNode.size > 0
    F = _F(P, uv.ub, uv.vb, {"h": h, "as": as_, "ab": P.ab})
    ctrl = {"dt": 0.1, "ThicknessConstraints": 1.0, "ThickMin": 1.0,
            "uvhDesiredWorkAndForceTolerances": [np.inf, 1e-20], "uvhDesiredWorkOrForceTolerances": [np.inf, 1e-20]}
    ub, vb, hh, lam, info = g(5, g.struct(ctrl), _mua(g, P), g.struct(_bcs(P)), g.struct(F), g.struct(dict(F)),
                              g.double(np.zeros((0, 0))))
    assert info["uvhConverged"][0, 0] == 1 and info["activeSetConverged"][0, 0] == 1
    assert info["activeSetIterations"][0, 0] == ref.iterations
    assert np.array_equal(info["hPosNode"].ravel().astype(np.int64) - 1, ref.hPosNode)
    got = np.concatenate([ub.ravel(), vb.ravel(), hh.ravel()])
    want = np.concatenate([ref.res.ub, ref.res.vb, ref.res.h])
    assert np.linalg.norm(got - want) <= U_TOL * np.linalg.norm(want)
