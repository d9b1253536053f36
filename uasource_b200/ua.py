"""Host-side mirror of Úa's SSA hot-path interface, running on the B200 library.

Names and argument meaning follow the reference MATLAB functions:

* ``CreateMUA(coordinates, connectivity)`` — CreateMUA.m:1 (resident mesh)
* ``uvMatrixAssembly(CtrlVar, MUA, F, BCs, Ronly=, ZeroFields=)`` —
  uvMatrixAssembly.m:5 / uvMatrixAssemblySSTREAM.m:6, returns ``(Ruv, Kuv)``
* ``uv(CtrlVar, MUA, BCs, F, l)`` — uv.m:6 -> SSTREAM2dNR2.m:3, returns
  ``(F, l, Kuv, Ruv, RunInfo)``
* ``solveKApeSymmetric(A, B, f, g)`` — solveKApeSymmetric.m:1

Errors raise ``UaError`` carrying the reference's error identifiers in the
message (``uvMatrixAssembly:NaN`` etc.).  Every call goes to libuassa.so on
the GPU; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field, fields as dc_fields

import numpy as np

from . import lib as L


@dataclass
class CtrlVar:
    """CtrlVar fields that change hot-path arithmetic (Ua2D_DefaultParameters.m defaults)."""
    kH: float = 1.0
    Hh0: float = 0.0
    SpeedZero: float = 1e-4
    EpsZero: float = 1e-10
    etaZero: float = 10.0
    Czero: float = 0.0
    Cmin: float = 1e-20
    AGlenmin: float = 1e-20
    Picard: int = 0
    NRviscosity: float = 1.0
    NRitmax: int = 50
    NRitmin: int = 1
    NewtonAcceptRatio: float = 0.5
    BacktrackingGammaMin: float = 1e-10
    LineSearchAllowedToUseExtrapolation: int = 0
    BackTrackBeta: float = 0.1
    BackTrackMaxIterations: int = 50
    BackTrackMaxExtrapolations: int = 50
    BackTrackExtrapolationRatio: float = 2.5
    BackTrackMinXfrac: float = 1e-10
    BackTrackMaxFuncSame: int = 3
    BackTrackGuardLower: float = 0.25
    BackTrackGuardUpper: float = 0.95
    NLtol: float = 1e-15
    uvDesiredWorkAndForceTolerances: tuple = (math.inf, 1e-15)
    uvDesiredWorkOrForceTolerances: tuple = (math.inf, 1e-15)
    uvExitBackTrackingStepLength: float = 1e-10
    uvAcceptableWorkAndForceTolerances: tuple = (math.inf, 1e-15)
    uvAcceptableWorkOrForceTolerances: tuple = (math.inf, 1e-15)
    ModifiedNRuvIntervalCriterion: int = 1
    ModifiedNRuvReductionCriterion: float = 0.5
    theta: float = 0.5
    SUPG_beta0: float = 1.0
    uvh_SUPG_tauMultiplier: float = 1.0
    uvh_SUPG_tau: int = 0
    uvhDesiredWorkAndForceTolerances: tuple = (math.inf, 1e-15)
    uvhDesiredWorkOrForceTolerances: tuple = (math.inf, 1e-15)
    uvhExitBackTrackingStepLength: float = 1e-3
    uvhAcceptableWorkAndForceTolerances: tuple = (math.inf, 1e-6)
    uvhAcceptableWorkOrForceTolerances: tuple = (1.0, 1e-8)
    krylov_rtol: float = 1e-12
    krylov_maxit: int = 20000
    precision: int = L.UA_PREC_FP64
    patch_nodes: int = 0
    verbose: int = 0
    profile: int = 0
    krylov_adaptive: int = 1
    krylov_precond: int = L.UA_PC_AMG
    spmv_lanes: int = 0
    asm_threads: int = 0
    asm_regs: int = 0
    uvh_krylov: int = L.UA_KRYLOV_GMRES
    krylov_restart: int = 40
    krylov_eta_c: float = 0.5
    krylov_eta_max: float = 0.1
    precond_bf16: int = 1
    amg_smoothed: int = 1
    krylov_full_grid: int = 0
    amg_P_refresh: int = 0
    uvh_h_sweeps: int = 0
    krylov_sell: int = 1
    SlidingLaw: str = "Weertman"          # any name of L.SLIDING_LAWS
    Nzero: float = 1e-20
    IncludeMelangeModelPhysics: int = 0
    ThicknessConstraints: int = 1         # uvh active set (uvh.m:64-212)
    ThickMin: float = 1.0
    ThicknessConstraintsItMax: int = 10
    MaxNumberOfNewlyIntroducedActiveThicknessConstraints: int = 1000
    MinNumberOfNewlyIntroducedActiveThicknessConstraints: int = 0

    def set_force_tolerance(self, tol):
        """Set every uv force tolerance (desired and acceptable) to ``tol`` (rForce < tol)."""
        for name in ("uvDesiredWorkAndForceTolerances", "uvDesiredWorkOrForceTolerances",
                     "uvAcceptableWorkAndForceTolerances", "uvAcceptableWorkOrForceTolerances"):
            setattr(self, name, (math.inf, tol))
        return self

    def set_uvh_force_tolerance(self, tol):
        """Set the desired uvh force tolerances (rForce < tol); acceptable ones keep their defaults."""
        self.uvhDesiredWorkAndForceTolerances = (math.inf, tol)
        self.uvhDesiredWorkOrForceTolerances = (math.inf, tol)
        return self

    def to_c(self) -> L.ua_params:
        p = L.ua_params()
        L.load().ua_params_default(C.byref(p))
        for f in dc_fields(self):
            v = getattr(self, f.name)
            if isinstance(v, tuple):
                arr = getattr(p, f.name)
                arr[0], arr[1] = float(v[0]), float(v[1])
            elif f.name == "SlidingLaw":
                if v not in L.SLIDING_LAWS:
                    raise ValueError(f"BasalDrag:CaseNotFound what sliding law? ({v!r})")
                p.SlidingLaw = L.SLIDING_LAWS[v]
            else:
                setattr(p, f.name, v)
        return p


@dataclass
class Fields:
    """F (UaFields.m): nodal column vectors and the scalars rhow, g, alpha."""
    h: np.ndarray
    S: np.ndarray
    B: np.ndarray
    rho: np.ndarray
    AGlen: np.ndarray
    n: np.ndarray
    C: np.ndarray
    m: np.ndarray
    ub: np.ndarray
    vb: np.ndarray
    rhow: float = 1030.0
    g: float = 9.81 / 1000
    alpha: float = 0.0
    as_: np.ndarray = None      # surface mass balance F.as (transient solves)
    ab: np.ndarray = None       # basal mass balance F.ab
    dadh: np.ndarray = None     # d(as+ab)/dh (MassBalanceGeometryFeedback=3), None = 0
    q: np.ndarray = None        # Budd sliding-law exponent
    muk: np.ndarray = None      # Coulomb friction coefficient (Tsai, Coulomb, Cornford, Umbi)
    V0: np.ndarray = None       # Joughin speed scale
    uo: np.ndarray = None       # melange: ocean velocity, drag coefficient and exponent
    vo: np.ndarray = None
    Co: np.ndarray = None
    mo: np.ndarray = None
    ua: np.ndarray = None       # melange: atmosphere velocity, drag coefficient and exponent
    va: np.ndarray = None
    Ca: np.ndarray = None
    ma: np.ndarray = None

    @staticmethod
    def from_problem(P):
        return Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m,
                      ub=P.ub.copy(), vb=P.vb.copy(), rhow=P.rhow, g=P.g, alpha=P.alpha,
                      as_=None if P.as_ is None else P.as_.copy(), ab=None if P.ab is None else P.ab.copy())

    def copy(self):
        return Fields(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()})


@dataclass
class BCs:
    """Fixed-node velocity boundary conditions (0-based node indices)."""
    ubFixedNode: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    ubFixedValue: np.ndarray = field(default_factory=lambda: np.zeros(0))
    vbFixedNode: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    vbFixedValue: np.ndarray = field(default_factory=lambda: np.zeros(0))
    ubTiedNodeA: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    ubTiedNodeB: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    vbTiedNodeA: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    vbTiedNodeB: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    ubvbFixedNormalNode: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    ubvbFixedNormalValue: np.ndarray = field(default_factory=lambda: np.zeros(0))

    @staticmethod
    def from_problem(P):
        return BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue,
                   vbFixedNode=P.vbFixedNode, vbFixedValue=P.vbFixedValue)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class _Keep:
    """Keeps the numpy buffers behind ctypes structs alive for a call."""

    def __init__(self):
        self.refs = []

    def d(self, a):
        if a is None:
            return None
        a = _f64(a)
        self.refs.append(a)
        return L.dptr(a)

    def i(self, a):
        if a is None:
            return None
        a = _i32(a)
        self.refs.append(a)
        return L.iptr(a)


def _c_fields(F: Fields, keep: _Keep, Nn: int, copy_uv=True):
    cf = L.ua_fields()
    cf.location = L.UA_HOST

    def full(v):
        v = np.asarray(v, dtype=np.float64)
        return np.full(Nn, float(v)) if v.ndim == 0 else v

    for name in ("h", "S", "B", "rho", "AGlen", "n", "C", "m"):
        setattr(cf, name, keep.d(full(getattr(F, name))))
    # the solution overwrites ub, vb unless the caller gives output arrays (copy_uv=False)
    ub = _f64(F.ub).copy() if copy_uv else _f64(F.ub)
    vb = _f64(F.vb).copy() if copy_uv else _f64(F.vb)
    keep.refs += [ub, vb]
    cf.ub = L.dptr(ub)
    cf.vb = L.dptr(vb)
    cf.rhow, cf.g, cf.alpha = float(F.rhow), float(F.g), float(F.alpha)
    for name in ("q", "muk", "V0", "uo", "vo", "Co", "mo", "ua", "va", "Ca", "ma"):
        v = getattr(F, name)
        if v is not None:
            setattr(cf, name, keep.d(full(v)))
    return cf, ub, vb


def _c_bcs(B: BCs, keep: _Keep):
    cb = L.ua_bcs()
    if B is None:
        return cb
    cb.n_ufixed = len(B.ubFixedNode); cb.ufixed_node = keep.i(B.ubFixedNode); cb.ufixed_value = keep.d(B.ubFixedValue)
    cb.n_vfixed = len(B.vbFixedNode); cb.vfixed_node = keep.i(B.vbFixedNode); cb.vfixed_value = keep.d(B.vbFixedValue)
    cb.n_utied = len(B.ubTiedNodeA); cb.utied_a = keep.i(B.ubTiedNodeA); cb.utied_b = keep.i(B.ubTiedNodeB)
    cb.n_vtied = len(B.vbTiedNodeA); cb.vtied_a = keep.i(B.vbTiedNodeA); cb.vtied_b = keep.i(B.vbTiedNodeB)
    if len(B.ubvbFixedNormalNode):
        cb.n_normal = len(B.ubvbFixedNormalNode); cb.normal_node = keep.i(B.ubvbFixedNormalNode)
        cb.normal_value = keep.d(B.ubvbFixedNormalValue)
    hn = getattr(B, "hFixedNode", None)
    if hn is not None and len(hn):
        cb.n_hfixed = len(hn); cb.hfixed_node = keep.i(hn); cb.hfixed_value = keep.d(B.hFixedValue)
    hp = getattr(B, "hPosNode", None)
    if hp is not None and len(hp):
        cb.n_hpos = len(hp); cb.hpos_node = keep.i(hp)
    return cb


class MUA:
    """Device-resident mesh (one system, or a batch of independent systems)."""

    def __init__(self, meshes, ndof=2, device=0):
        lib = L.load()
        self.ndof = ndof
        self.device = device
        self.meshes = []
        descs = (L.ua_mesh_desc * len(meshes))()
        keep = _Keep()
        for k, (coords, conn) in enumerate(meshes):
            coords = np.asarray(coords, dtype=np.float64)
            conn = np.asarray(conn)
            self.meshes.append((coords, conn))
            cm = np.asfortranarray(coords).ravel(order="F")      # Nnodes x 2, column-major
            cc = np.asfortranarray(conn.astype(np.int32)).ravel(order="F")
            descs[k].nnodes = coords.shape[0]
            descs[k].nele = conn.shape[0]
            descs[k].nod = conn.shape[1]
            descs[k].index_base = 0
            descs[k].coordinates = keep.d(cm)
            descs[k].connectivity = keep.i(cc)
        h = C.c_void_p()
        L.check(lib.ua_mesh_create_batch(descs, len(meshes), ndof, device, C.byref(h)))
        self._h = h
        self._pattern = {}

    @property
    def handle(self):
        return self._h

    @property
    def nsys(self):
        return len(self.meshes)

    def Nnodes(self, s=0):
        return self.meshes[s][0].shape[0]

    def Nele(self, s=0):
        return self.meshes[s][1].shape[0]

    @property
    def nod(self):
        return self.meshes[0][1].shape[1]

    def device_bytes(self):
        b = C.c_int64()
        L.check(L.load().ua_mesh_info(self._h, 0, None, None, None, C.byref(b)))
        return b.value

    def flipped(self):
        n = C.c_int32()
        L.check(L.load().ua_mesh_flipped(self._h, C.byref(n)))
        return n.value

    def nnz(self, s=0):
        """Non-zeros of system s's structural tangent pattern."""
        nnz = C.c_int64()
        L.check(L.load().ua_mesh_pattern(self._h, s, C.byref(nnz), None, None))
        return nnz.value

    def pattern(self, s=0):
        """(rowptr, colind) of the structural tangent pattern (0-based, sorted)."""
        if s not in self._pattern:
            lib = L.load()
            nnz = C.c_int64()
            L.check(lib.ua_mesh_pattern(self._h, s, C.byref(nnz), None, None))
            n = self.ndof * self.Nnodes(s)
            rp = np.zeros(n + 1, np.int64)
            ci = np.zeros(nnz.value, np.int64)
            L.check(lib.ua_mesh_pattern(self._h, s, C.byref(nnz), L.lptr(rp), L.lptr(ci)))
            self._pattern[s] = (rp, ci)
        return self._pattern[s]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            L.load().ua_mesh_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def CreateMUA(coordinates, connectivity, ndof=2, device=0, index_base=0):
    """CreateMUA.m: resident mesh on the GPU (inside-out elements are flipped)."""
    conn = np.asarray(connectivity) - index_base
    return MUA([(coordinates, conn)], ndof=ndof, device=device)


def CreateMUABatch(meshes, ndof=2, device=0):
    """Batch of independent meshes [(coordinates, connectivity), ...] in one handle."""
    return MUA(list(meshes), ndof=ndof, device=device)


def _csr(mua, s, vals, drop_zeros):
    import scipy.sparse as sp
    rp, ci = mua.pattern(s)
    n = mua.ndof * mua.Nnodes(s)
    K = sp.csr_matrix((vals, ci, rp), shape=(n, n))
    if drop_zeros:  # MATLAB sparse() keeps non-zeros only
        K.eliminate_zeros()
    return K


def uvMatrixAssembly(ctrl: CtrlVar, mua: MUA, F: Fields, bcs: BCs = None, Ronly=False, ZeroFields=False,
                     drop_zeros=False, return_parts=False):
    """uvMatrixAssembly.m:5 -> uvMatrixAssemblySSTREAM.m:6-553 on the GPU.

    Returns ``(Ruv, Kuv)``; Kuv is a scipy CSR on the structural pattern (None
    when Ronly).  With ``return_parts`` also ``(Tint, Fext)``.
    """
    lib = L.load()
    keep = _Keep()
    Nn = mua.Nnodes()
    cf, _, _ = _c_fields(F, keep, Nn)
    cb = _c_bcs(bcs, keep)
    p = ctrl.to_c()
    mode = L.UA_ASM_ZERO_R if ZeroFields else (L.UA_ASM_R if Ronly else L.UA_ASM_RK)
    if ZeroFields and not Ronly:
        raise ValueError("ZeroFields assembly is residual-only")
    R = np.zeros(2 * Nn)
    Kv = None
    if mode == L.UA_ASM_RK:
        nnz = mua.pattern()[1].size
        Kv = np.zeros(nnz)
    T = np.zeros(2 * Nn) if return_parts else None
    Fx = np.zeros(2 * Nn) if return_parts else None
    L.check(lib.ua_uv_assemble(mua.handle, C.byref(p), C.byref(cf), C.byref(cb), mode, L.dptr(R), L.dptr(Kv),
                               L.dptr(T), L.dptr(Fx)))
    K = _csr(mua, 0, Kv, drop_zeros) if Kv is not None else None
    if return_parts:
        return R, K, T, Fx
    return R, K


@dataclass
class RunInfo:
    converged: bool
    iterations: int
    backtrack_steps: int
    krylov_its_total: int
    cauchy_fallbacks: int
    retried: bool
    r: float
    rForce: float
    rWork: float
    assembly_ms: float
    solve_ms: float
    total_ms: float
    device_ms: float
    kernels: dict
    gpu_launches: int
    iters: list
    updates: np.ndarray = None  # per iteration gamma*[du; dv; (dh;) dl] when requested
    active_set: dict = None     # uvh: iterations, cyclical, converged, hPosNode (the final active set)


def _updates_buffer(rep, cap, stride):
    """Caller-owned buffer for the per-iteration Newton updates (SSTREAM2dNR2.m:367-369)."""
    buf = np.full((cap, stride), np.nan)
    rep.updates = buf.ctypes.data_as(C.POINTER(C.c_double))
    rep.update_stride = stride
    return buf


def _report(rep, recs, updates=None):
    its = []
    for k in range(rep.n_iter_records):
        it = recs[k]
        its.append(dict(iteration=it.iteration, iarm=it.iarm, krylov_its=it.krylov_its, direction=it.direction,
                        gamma=it.gamma, r0=it.r0, r=it.r, rForce=it.rForce, rWork=it.rWork))
    kern = dict(asmK_ms=rep.kasmK_ms, asmK_n=rep.kasmK_n, asmR_ms=rep.kasmR_ms, asmR_n=rep.kasmR_n,
                spmv_ms=rep.kspmv_ms, spmv_n=rep.kspmv_n, amgR_ms=rep.kamgR_ms, amgR_n=rep.kamgR_n,
                amgP_ms=rep.kamgP_ms, amgP_n=rep.kamgP_n, setup_ms=rep.ksetup_ms, setup_n=rep.ksetup_n,
                krylov_ms=rep.kkrylov_ms, krylov_n=rep.kkrylov_n,
                work_nnz=dict(zip(("asmK", "asmR", "spmv", "amgR", "amgP"), list(rep.kwork_nnz))),
                work_rows=dict(zip(("asmK", "asmR", "spmv", "amgR", "amgP"), list(rep.kwork_rows))))
    return RunInfo(bool(rep.converged), rep.iterations, rep.backtrack_steps, rep.krylov_its_total,
                   rep.cauchy_fallbacks, bool(rep.retried), rep.r, rep.rForce, rep.rWork, rep.assembly_ms,
                   rep.solve_ms, rep.total_ms, rep.device_ms, kern, rep.gpu_launches, its,
                   None if updates is None else updates[:rep.n_iter_records].copy())


def uv(ctrl: CtrlVar, mua: MUA, bcs: BCs, F: Fields, l=None, return_K=False, return_updates=False):
    """uv.m:6 -> SSTREAM2dNR2.m:3-431 on the GPU (one mesh).

    Returns ``(F, l, Kuv, Ruv, RunInfo)``: F with the solved ub, vb, the
    Lagrange multipliers l.ubvb, and (if ``return_K``) the last tangent and
    residual.  With ``return_updates`` RunInfo.updates holds, per Newton
    iteration, the accepted update ``gamma*[du; dv; dl]`` (SSTREAM2dNR2.m:367-369).
    """
    lib = L.load()
    keep = _Keep()
    Nn = mua.Nnodes()
    cf, ub, vb = _c_fields(F, keep, Nn)
    cb = _c_bcs(bcs, keep)
    p = ctrl.to_c()
    nc = C.c_int32()
    L.check(lib.ua_constraint_count(mua.handle, C.byref(cb), 2, C.byref(nc)))
    lam = np.zeros(nc.value) if l is None or len(l) != nc.value else _f64(l).copy()
    rep = L.ua_newton_report()
    recs = (L.ua_newton_iter * ((ctrl.NRitmax + 2) * 2))()
    rep.iters = C.cast(recs, C.POINTER(L.ua_newton_iter))
    rep.iters_capacity = (ctrl.NRitmax + 2) * 2
    upd = _updates_buffer(rep, rep.iters_capacity, 2 * Nn + nc.value) if return_updates else None
    Kv = np.zeros(mua.pattern()[1].size) if return_K else None
    Rv = np.zeros(2 * Nn) if return_K else None
    rc = lib.ua_uv_newton(mua.handle, C.byref(p), C.byref(cf), C.byref(cb), L.dptr(lam), len(lam), C.byref(rep),
                          L.dptr(Kv), L.dptr(Rv))
    L.check(rc, allow=(L.UA_ERR_NOT_CONVERGED,))
    Fo = Fields(**{f.name: getattr(F, f.name) for f in dc_fields(F)})
    Fo.ub, Fo.vb = ub, vb
    K = _csr(mua, 0, Kv, False) if return_K else None
    return Fo, lam, K, Rv, _report(rep, recs, upd)


def uv_batch(ctrl: CtrlVar, mua: MUA, Fs, bcss, out=None):
    """Batched uv Newton: all systems of a batch handle in the same launches.

    ``out`` (optional): per system a pair ``(ub, vb)`` of caller-owned float64 arrays of the
    system's node count that receive the solution (``ua_fields.ub_out/vb_out``); ``Fs[s].ub/vb``
    are then read in place as the start velocities (no copies: pinned host buffers stay pinned).
    Without it the solution goes into fresh copies of ``Fs[s].ub/vb``.

    Returns a list of ``(ub, vb, RunInfo)``.
    """
    lib = L.load()
    keep = _Keep()
    ns = mua.nsys
    cfs = (L.ua_fields * ns)()
    cbs = (L.ua_bcs * ns)()
    outs = []
    reps = (L.ua_newton_report * ns)()
    recs = []
    if out is not None and len(out) != ns:
        raise ValueError(f"uv_batch: out holds {len(out)} pairs for {ns} systems")
    for s in range(ns):
        if out is None:
            cf, ub, vb = _c_fields(Fs[s], keep, mua.Nnodes(s))
        else:
            cf, ub, vb = _c_fields(Fs[s], keep, mua.Nnodes(s), copy_uv=False)
            ub, vb = out[s]
            for a in (ub, vb):
                if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
                        and a.size == mua.Nnodes(s)):
                    raise ValueError("uv_batch: out arrays must be contiguous float64 of the node count")
            keep.refs += [ub, vb]
            cf.ub_out = L.dptr(ub)
            cf.vb_out = L.dptr(vb)
        cfs[s] = cf
        cbs[s] = _c_bcs(bcss[s], keep)
        outs.append((ub, vb))
        r = (L.ua_newton_iter * ((ctrl.NRitmax + 2) * 2))()
        recs.append(r)
        reps[s].iters = C.cast(r, C.POINTER(L.ua_newton_iter))
        reps[s].iters_capacity = (ctrl.NRitmax + 2) * 2
    p = ctrl.to_c()
    rc = lib.ua_uv_newton_batch(mua.handle, C.byref(p), cfs, cbs, reps)
    L.check(rc, allow=(L.UA_ERR_NOT_CONVERGED,))
    return [(outs[s][0], outs[s][1], _report(reps[s], recs[s])) for s in range(ns)]


def uv_batch_resident(ctrl: CtrlVar, mua: MUA, F_devs, bcss, rhow=1030.0, g=9.81 / 1000, alpha=0.0):
    """Batched uv Newton with every system's fields already resident in device memory.

    ``F_devs[s]`` maps h, S, B, rho, AGlen, n, C, m, ub, vb to device addresses of
    system s (see ``uv_resident``); ub/vb are overwritten with the solutions.
    Returns a list of RunInfo.
    """
    lib = L.load()
    keep = _Keep()
    ns = mua.nsys
    cfs = (L.ua_fields * ns)()
    cbs = (L.ua_bcs * ns)()
    reps = (L.ua_newton_report * ns)()
    recs = []
    for s in range(ns):
        cf = cfs[s]
        cf.location = L.UA_DEVICE
        for name in ("h", "S", "B", "rho", "AGlen", "n", "C", "m", "ub", "vb"):
            setattr(cf, name, C.cast(C.c_void_p(int(F_devs[s][name])), L._dp))
        cf.rhow, cf.g, cf.alpha = float(rhow), float(g), float(alpha)
        cbs[s] = _c_bcs(bcss[s], keep)
        r = (L.ua_newton_iter * ((ctrl.NRitmax + 2) * 2))()
        recs.append(r)
        reps[s].iters = C.cast(r, C.POINTER(L.ua_newton_iter))
        reps[s].iters_capacity = (ctrl.NRitmax + 2) * 2
    p = ctrl.to_c()
    rc = lib.ua_uv_newton_batch(mua.handle, C.byref(p), cfs, cbs, reps)
    L.check(rc, allow=(L.UA_ERR_NOT_CONVERGED,))
    return [_report(reps[s], recs[s]) for s in range(ns)]


def _c_fields_uvh(F0: Fields, F1: Fields, dt, keep: _Keep, Nn: int):
    """uvh inputs: time-independent fields and level-1 state from F1, level 0 from F0."""
    cf, ub, vb = _c_fields(F1, keep, Nn)
    h1 = _f64(F1.h).copy()
    keep.refs.append(h1)
    cf.h1 = L.dptr(h1)
    cf.h0 = keep.d(F0.h); cf.u0 = keep.d(F0.ub); cf.v0 = keep.d(F0.vb)
    z = np.zeros(Nn)
    cf.as0 = keep.d(F0.as_ if F0.as_ is not None else z); cf.ab0 = keep.d(F0.ab if F0.ab is not None else z)
    cf.as1 = keep.d(F1.as_ if F1.as_ is not None else z); cf.ab1 = keep.d(F1.ab if F1.ab is not None else z)
    cf.dadh = keep.d(F1.dadh) if F1.dadh is not None else None
    cf.dt = float(dt)
    return cf, ub, vb, h1


def uvhAssembly(ctrl: CtrlVar, mua: MUA, F0: Fields, F1: Fields, dt, Ronly=False, ZeroFields=False,
                return_parts=False):
    """uvhAssembly.m:1 -> uvhMatrixAssembly.m:6-585 on the GPU (ndof=3 handle).

    Returns ``(R, K)``: R = Tint-Fext (3Nn), K the unsymmetric tangent (scipy
    CSR on the structural pattern; None when Ronly or ZeroFields).
    """
    lib = L.load()
    keep = _Keep()
    Nn = mua.Nnodes()
    cf, _, _, _ = _c_fields_uvh(F0, F1, dt, keep, Nn)
    p = ctrl.to_c()
    mode = L.UA_ASM_ZERO_R if ZeroFields else (L.UA_ASM_R if Ronly else L.UA_ASM_RK)
    R = np.zeros(3 * Nn)
    Kv = np.zeros(mua.pattern()[1].size) if mode == L.UA_ASM_RK else None
    T = np.zeros(3 * Nn) if return_parts else None
    Fx = np.zeros(3 * Nn) if return_parts else None
    L.check(lib.ua_uvh_assemble(mua.handle, C.byref(p), C.byref(cf), mode, L.dptr(R), L.dptr(Kv), L.dptr(T),
                                L.dptr(Fx)))
    K = _csr(mua, 0, Kv, False) if Kv is not None else None
    if return_parts:
        return R, K, T, Fx
    return R, K


@dataclass
class HBCs(BCs):
    """Velocity and thickness boundary conditions (0-based node indices); hPosNode is the active
    minimum-thickness set carried from the previous step (BCs1.hPosNode)."""
    hFixedNode: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    hFixedValue: np.ndarray = field(default_factory=lambda: np.zeros(0))
    hPosNode: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))


def uvh(ctrl: CtrlVar, mua: MUA, F0: Fields, F1: Fields, bcs: BCs, dt, l=None, return_updates=False):
    """uvh.m:5 -> uvh2D.m:20 -> SSTREAM_TransientImplicit.m:6-717 on the GPU.

    F0: state at t (h, ub, vb, as_, ab); F1: start values at t+dt and the
    time-independent fields.  Returns ``(F1, luvh, RunInfo)`` with F1.ub,
    F1.vb, F1.h solved.  With ``return_updates`` RunInfo.updates holds the
    per-iteration updates ``gamma*[du; dv; dh; dl]``
    (SSTREAM_TransientImplicit.m:478-483).
    """
    lib = L.load()
    keep = _Keep()
    Nn = mua.Nnodes()
    cf, ub, vb, h1 = _c_fields_uvh(F0, F1, dt, keep, Nn)
    cb = _c_bcs(bcs, keep)
    p = ctrl.to_c()
    nc = C.c_int32()
    L.check(lib.ua_constraint_count(mua.handle, C.byref(cb), 3, C.byref(nc)))
    lam = np.zeros(nc.value) if l is None or len(l) != nc.value else _f64(l).copy()
    rep = L.ua_newton_report()
    cap = (ctrl.NRitmax + 2) * 2
    recs = (L.ua_newton_iter * cap)()
    rep.iters = C.cast(recs, C.POINTER(L.ua_newton_iter))
    rep.iters_capacity = cap
    upd = _updates_buffer(rep, cap, 3 * Nn + nc.value) if return_updates else None
    hpos_out = np.zeros(Nn, np.int32)
    rep.hpos_node = L.iptr(hpos_out)
    rep.hpos_capacity = Nn
    rc = lib.ua_uvh_newton(mua.handle, C.byref(p), C.byref(cf), C.byref(cb), L.dptr(lam), len(lam), C.byref(rep))
    L.check(rc, allow=(L.UA_ERR_NOT_CONVERGED,))
    Fo = F1.copy()
    Fo.ub, Fo.vb, Fo.h = ub, vb, h1
    info = _report(rep, recs, upd)
    if ctrl.ThicknessConstraints:
        info.active_set = dict(iterations=rep.active_set_iterations, cyclical=bool(rep.active_set_cyclical),
                               converged=bool(rep.active_set_converged),
                               hPosNode=hpos_out[:rep.n_hpos].copy())
    return Fo, lam, info


def adjoint_gradient_C(ctrl: CtrlVar, mua: MUA, F: Fields, bcs_adjoint: BCs, us, vs, usErr, vsErr, logC=True,
                       premultiplier="M"):
    """Adjoint gradient of the "-uv-" velocity misfit with respect to C at the solved state F
    (Misfit.m adjoint branch -> solveKApeSymmetric -> dIdCq.m -> ApplyAdjointGradientPreMultiplier.m)
    on the GPU.  ``logC``: the gradient with respect to log10(C); ``premultiplier`` "M" or "I"
    (CtrlVar.Inverse.AdjointGradientPreMultiplier).  Returns (I, dIduv, lambda, dIdC, krylov_its)
    with lambda = [uAdjoint; vAdjoint]."""
    if premultiplier not in ("M", "I"):
        raise ValueError("AdjointGradientPreMultiplier must be 'M' or 'I'")
    lib = L.load()
    keep = _Keep()
    Nn = mua.Nnodes()
    cf, _, _ = _c_fields(F, keep, Nn)
    cb = _c_bcs(bcs_adjoint, keep)
    p = ctrl.to_c()
    ms = L.ua_measurements(keep.d(us), keep.d(vs), keep.d(usErr), keep.d(vsErr))
    flags = (L.UA_ADJ_LOGC if logC else 0) | (L.UA_ADJ_PREMUL_M if premultiplier == "M" else 0)
    I = C.c_double()
    its = C.c_int32()
    dIduv = np.zeros(2 * Nn); lam = np.zeros(2 * Nn); g = np.zeros(Nn)
    L.check(lib.ua_uv_adjoint_dIdC(mua.handle, C.byref(p), C.byref(cf), C.byref(cb), C.byref(ms), flags,
                                   C.byref(I), L.dptr(dIduv), L.dptr(lam), L.dptr(g), C.byref(its)))
    return I.value, dIduv, lam, g, its.value


def autotune(ctrl: CtrlVar, mua: MUA, F, reps=3):
    """Tunes the assembly schedule of a uv handle (patch shape and P1 CTA size) at the fields F
    (one Fields for every system, or a list with one per system) and makes the fastest the
    process-wide schedule for this device, element type and dof count (used by every handle with
    ``patch_nodes``, ``asm_threads`` and ``asm_regs`` at 0).  Returns a dict with the candidates, their mean
    launch times (ms), the chosen one and the default schedule's time.  Results do not depend on
    the schedule."""
    lib = L.load()
    keep = _Keep()
    Fs = F if isinstance(F, (list, tuple)) else [F]
    cfs = (L.ua_fields * len(Fs))()
    for k, Fk in enumerate(Fs):
        Nn = mua.Nnodes(k) if len(Fs) > 1 else mua.Nnodes()
        cf, _, _ = _c_fields(Fk, keep, Nn)
        cfs[k] = cf
    p = ctrl.to_c()
    rep = L.ua_tune_report()
    L.check(lib.ua_autotune(mua.handle, C.byref(p), cfs, len(Fs), reps, C.byref(rep)))
    n = rep.n_candidates
    cands = [dict(div=rep.div[i], cap=rep.cap[i], threads=rep.threads[i], regs=rep.regs[i], ms=rep.ms[i])
             for i in range(n)]
    return dict(candidates=cands, chosen=cands[rep.chosen], default_ms=rep.default_ms,
                gain=rep.default_ms / cands[rep.chosen]["ms"])


def constraint_matrix(mua: MUA, bcs: BCs):
    """The constraint matrix L and right-hand side c of ``bcs`` on a single-mesh handle, as the
    solvers impose them (BCs2MLC.m -> CreateLuv.m, createLh.m for fixed h on an ndof=3 handle,
    ScaleL.m): rows u ties, v ties, fixed u, fixed v, fixed normal velocities, fixed h, each scaled
    to unit length.  Returns (L as a scipy CSR matrix of ndof*Nnodes columns, c)."""
    import scipy.sparse as sp
    lib = L.load()
    keep = _Keep()
    cb = _c_bcs(bcs, keep)
    nc = C.c_int32()
    L.check(lib.ua_constraint_matrix(mua.handle, C.byref(cb), C.byref(nc), None, None, None))
    n = nc.value
    dof = np.zeros(2 * n, np.int32)
    val = np.zeros(2 * n)
    rhs = np.zeros(n)
    L.check(lib.ua_constraint_matrix(mua.handle, C.byref(cb), C.byref(nc), L.iptr(dof), L.dptr(val), L.dptr(rhs)))
    rows = np.repeat(np.arange(n), 2)
    keep_ = dof >= 0
    Lm = sp.csr_matrix((val[keep_], (rows[keep_], dof[keep_])), shape=(n, mua.ndof * mua.Nnodes()))
    return Lm, rhs


def solveKApeSymmetric(A, B, f, g, rtol=1e-12, maxit=0, device=0):
    """solveKApeSymmetric.m -> ABfgPreEliminate.m for SPD A and selection-type B.

    A, B: scipy sparse matrices.  Returns (x, y, iterations).
    """
    import scipy.sparse as sp
    lib = L.load()
    A = sp.csr_matrix(A)
    A.sort_indices()
    n = A.shape[0]
    arp = A.indptr.astype(np.int64); aci = A.indices.astype(np.int64); av = _f64(A.data)
    if B is None or B.shape[0] == 0:
        nl = 0
        brp = bci = bv = None
        g = np.zeros(0)
    else:
        B = sp.csr_matrix(B)
        nl = B.shape[0]
        brp = B.indptr.astype(np.int64); bci = B.indices.astype(np.int64); bv = _f64(B.data)
    x = np.zeros(n)
    y = np.zeros(nl)
    its = C.c_int32()
    f = _f64(f); g = _f64(g)
    L.check(lib.ua_solve_kape_symmetric(n, L.lptr(arp), L.lptr(aci), L.dptr(av), nl, L.lptr(brp), L.lptr(bci),
                                        L.dptr(bv), L.dptr(f), L.dptr(g), L.dptr(x), L.dptr(y), rtol, maxit,
                                        C.byref(its), device))
    return x, y, its.value


def uv_resident(ctrl: CtrlVar, mua: MUA, bcs: BCs, F_dev: dict, rhow=1030.0, g=9.81 / 1000, alpha=0.0,
                l=None):
    """uv Newton solve with fields already resident in device memory.

    ``F_dev`` maps h, S, B, rho, AGlen, n, C, m, ub, vb to device addresses
    (integers, e.g. ``tensor.data_ptr()`` of contiguous float64 CUDA tensors
    on the handle's device).  ub/vb are overwritten with the solution.  The
    caller must have completed all writes to these buffers before the call.
    """
    lib = L.load()
    keep = _Keep()
    cf = L.ua_fields()
    cf.location = L.UA_DEVICE
    for name in ("h", "S", "B", "rho", "AGlen", "n", "C", "m", "ub", "vb"):
        setattr(cf, name, C.cast(C.c_void_p(int(F_dev[name])), L._dp))
    cf.rhow, cf.g, cf.alpha = float(rhow), float(g), float(alpha)
    cb = _c_bcs(bcs, keep)
    p = ctrl.to_c()
    nc = C.c_int32()
    L.check(lib.ua_constraint_count(mua.handle, C.byref(cb), 2, C.byref(nc)))
    lam = np.zeros(nc.value) if l is None or len(l) != nc.value else _f64(l).copy()
    rep = L.ua_newton_report()
    cap = (ctrl.NRitmax + 2) * 2
    recs = (L.ua_newton_iter * cap)()
    rep.iters = C.cast(recs, C.POINTER(L.ua_newton_iter))
    rep.iters_capacity = cap
    rc = lib.ua_uv_newton(mua.handle, C.byref(p), C.byref(cf), C.byref(cb), L.dptr(lam), len(lam), C.byref(rep),
                          None, None)
    L.check(rc, allow=(L.UA_ERR_NOT_CONVERGED,))
    return lam, _report(rep, recs)
