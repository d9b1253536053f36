"""CPU oracle for the Úa SSA (SSTREAM) Newton hot path.

TEST INFRASTRUCTURE ONLY.  This module is a plain numpy/scipy restatement of
the reference MATLAB code and exists to check the CUDA implementation.  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it; the product path (``uasource_b200``) never does.

Parity status: the reference is MATLAB and cannot run here (no MATLAB, no
Octave).  The restatement is pinned by the reference's own known-answer
material instead: the analytic floating-shelf solution
(``UaUtilities/AnalyticalOneDimentionalIceShelf.m``), the analytic grounded
ice-stream solution (``UaMain/Simple1dIceStreamSolution.m``), the saddle-point
examples of ``UaMain/TestABfgPreEliminate.m`` and the quadrature exactness of
``UaMain/TestFEintegrate.m``; see ``tests/test_oracle_kat.py``.

Every function names the reference file:line it follows (paths relative to
the reference project root).  The vectorisation mirrors MATLAB's: arrays are
``Nele x nod`` gathers, with loops over integration points and local nodes in
the reference's order.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

EPS = np.finfo(float).eps

# ---------------------------------------------------------------------------
# Quadrature rules (UaMain/quadtriangle.m)
# ---------------------------------------------------------------------------


def _orbit_points(m, b1, b2, w):
    """Expand symmetric orbits to points on the domain [0 0;1 0;0 1].

    Follows quadTrianglePointsAndWeights (UaMain/quadtriangle.m:3674-3750):
    vertices a=(0,0), b=(1,0), c=(0,1), area=1/2; a barycentric triple
    (β1,β2,β3) maps to (x,y)=(β2,β3).
    """
    pts, wts = [], []
    for mi, p, q, wi in zip(m, b1, b2, w):
        if mi == 1:
            q = p
        r = 1.0 - (p + q)
        if mi == 1:
            orbit = [(p, q, r)]
        elif mi == 3:
            orbit = [(p, q, r), (q, r, p), (r, p, q)]
        elif mi == 6:
            orbit = [(p, q, r), (q, r, p), (r, p, q), (p, r, q), (q, p, r), (r, q, p)]
        else:  # pragma: no cover - not used by the rules below
            raise ValueError(mi)
        for (_, bb, cc) in orbit:
            pts.append((bb, cc))
            wts.append(0.5 * wi)
    return np.array(pts, dtype=float), np.array(wts, dtype=float)


def quad_rule(degree: int):
    """Degree-4 (6 point) and degree-8 (16 point) fully symmetric PI rules.

    quadTriangleNonProductDegree4 (UaMain/quadtriangle.m:505-516) and
    quadTriangleNonProductDegree8 'full' branch (UaMain/quadtriangle.m:725-745);
    selected by QuadratureRuleDegree.m:13-21 (TriNodes 3 -> 4, 6 -> 8).
    """
    if degree == 4:
        s = math.sqrt(38.0 - 44.0 * math.sqrt(2.0 / 5.0))
        b1 = [(8.0 - math.sqrt(10.0) + s) / 18.0, (8.0 - math.sqrt(10.0) - s) / 18.0]
        t = math.sqrt(213125.0 - 53320.0 * math.sqrt(10.0))
        w = [(620.0 + t) / 3720.0, (620.0 - t) / 3720.0]
        return _orbit_points([3, 3], b1, b1, w)
    if degree == 8:
        b1 = [0.3333333333333333333333333333333333, 0.1705693077517602066222935014914645,
              0.0505472283170309754584235505965989, 0.4592925882927231560288155144941693,
              0.2631128296346381134217857862846436]
        b2 = list(b1)
        b2[4] = 0.0083947774099576053372138345392944
        w = [0.1443156076777871682510911104890646, 0.1032173705347182502817915502921290,
             0.0324584976231980803109259283417806, 0.0950916342672846247938961043885843,
             0.0272303141744349942648446900739089]
        return _orbit_points([1, 3, 3, 3, 6], b1, b2, w)
    raise ValueError(f"quadrature degree {degree} not restated")


def rule_degree_for_nod(nod: int) -> int:
    """QuadratureRuleDegree.m:11-21."""
    return {3: 4, 6: 8}[nod]


# ---------------------------------------------------------------------------
# Shape functions (UaMain/shape_fun.m, UaMain/shape_der.m)
# ---------------------------------------------------------------------------


def shape_fun(nod, pt):
    """shape_fun.m:52-71 (2-D, nod=3 and nod=6)."""
    c1, c2 = pt
    c3 = 1.0 - c1 - c2
    if nod == 3:
        return np.array([c1, c3, c2])
    if nod == 6:
        return np.array([(2 * c1 - 1) * c1, 4 * c3 * c1, (2 * c3 - 1) * c3,
                         4 * c2 * c3, (2 * c2 - 1) * c2, 4 * c1 * c2])
    raise ValueError(nod)


def shape_der(nod, pt):
    """shape_der.m:54-98 (2-D, nod=3 and nod=6); rows d/dxi, d/deta."""
    c1, c2 = pt
    c3 = 1.0 - c1 - c2
    if nod == 3:
        return np.array([[1.0, -1.0, 0.0], [0.0, -1.0, 1.0]])
    if nod == 6:
        return np.array([[4 * c1 - 1, 4 * (c3 - c1), -(4 * c3 - 1), -4 * c2, 0.0, 4 * c2],
                         [0.0, -4 * c1, -(4 * c3 - 1), 4 * (c3 - c2), 4 * c2 - 1, 4 * c1]])
    raise ValueError(nod)


# ---------------------------------------------------------------------------
# Mesh (MUA) — CreateMUA.m:31-98, derivVector.m:96-109
# ---------------------------------------------------------------------------


@dataclass
class MUA:
    coordinates: np.ndarray            # Nnodes x 2
    connectivity: np.ndarray           # Nele x nod, 0-based
    points: np.ndarray = None
    weights: np.ndarray = None
    Deriv: np.ndarray = None           # Nele x 2 x nod x nip
    DetJ: np.ndarray = None            # Nele x nip
    EleAreas: np.ndarray = None

    @property
    def Nnodes(self):
        return self.coordinates.shape[0]

    @property
    def Nele(self):
        return self.connectivity.shape[0]

    @property
    def nod(self):
        return self.connectivity.shape[1]

    @property
    def nip(self):
        return self.points.shape[0]


def deriv_vector(coordinates, connectivity, points, Iint):
    """derivVector.m:25-109."""
    nod = connectivity.shape[1]
    coox = coordinates[connectivity, 0]
    cooy = coordinates[connectivity, 1]
    der = shape_der(nod, points[Iint])
    J11 = coox @ der[0]
    J12 = cooy @ der[0]
    J21 = coox @ der[1]
    J22 = cooy @ der[1]
    detJ = J11 * J22 - J12 * J21
    Deriv = np.zeros((connectivity.shape[0], 2, nod))
    for J in range(nod):
        Deriv[:, 0, J] = (J22 * der[0, J] - J12 * der[1, J]) / detJ
        Deriv[:, 1, J] = (-J21 * der[0, J] + J11 * der[1, J]) / detJ
    return Deriv, detJ


def create_mua(coordinates, connectivity):
    """CreateMUA.m:31-98 restricted to what the SSA kernels use.

    Quadrature from QuadratureRuleDegree/quadtriangle (CreateMUA.m:36-47),
    inside-out flip (TestAndCorrectForInsideOutElements.m), Deriv/DetJ
    (CalcMuaMeshDerivatives.m:27-31) and element areas.
    """
    coordinates = np.asarray(coordinates, dtype=float)
    connectivity = np.asarray(connectivity, dtype=np.int64).copy()
    nod = connectivity.shape[1]
    points, weights = quad_rule(rule_degree_for_nod(nod))
    # TestAndCorrectForInsideOutElements.m: detJ at the centroid must be > 0
    _, detc = deriv_vector(coordinates, connectivity, np.array([[1 / 3, 1 / 3]]), 0)
    bad = detc < 0
    if np.any(bad):
        connectivity[bad] = flip_elements(connectivity[bad])
    mua = MUA(coordinates, connectivity, points, weights)
    nip = points.shape[0]
    mua.Deriv = np.zeros((mua.Nele, 2, nod, nip))
    mua.DetJ = np.zeros((mua.Nele, nip))
    for Iint in range(nip):
        D, dJ = deriv_vector(coordinates, connectivity, points, Iint)
        mua.Deriv[:, :, :, Iint] = D
        mua.DetJ[:, Iint] = dJ
    # TriAreaFE: area = sum_ip detJ*w
    mua.EleAreas = mua.DetJ @ weights
    return mua


def flip_elements(conn):
    """FlipElements.m: reverse orientation (P1: swap nodes 2,3; P2: corners 3<->5, mids 2<->6)."""
    conn = conn.copy()
    if conn.shape[1] == 3:
        conn[:, [1, 2]] = conn[:, [2, 1]]
    elif conn.shape[1] == 6:
        conn[:, [1, 2, 3, 4, 5]] = conn[:, [5, 4, 3, 2, 1]]
    return conn


# ---------------------------------------------------------------------------
# Parameters (the CtrlVar fields that change hot-path arithmetic)
# ---------------------------------------------------------------------------


@dataclass
class Params:
    """Subset of CtrlVar; defaults from Ua2D_DefaultParameters.m (line given)."""
    kH: float = 1.0                  # :2288
    Hh0: float = 0.0                 # :2295
    SpeedZero: float = 1e-4          # :412
    EpsZero: float = 1e-10           # :413
    etaZero: float = 10.0            # :415
    Czero: float = 0.0               # :441
    Cmin: float = 1e-20              # :456-460 (SSTREAM)
    AGlenmin: float = 1e-20          # :463
    Picard: int = 0                  # :593
    NRviscosity: float = 1.0         # :594
    NRitmax: int = 50                # :597
    NRitmin: int = 1                 # :600
    NewtonAcceptRatio: float = 0.5   # :601
    BacktrackingGammaMin: float = 1e-10  # :604
    LineSearchAllowedToUseExtrapolation: bool = False  # :603
    BackTrackBeta: float = 0.1       # :616
    BackTrackMaxIterations: int = 50  # :617
    BackTrackMaxExtrapolations: int = 50  # :618
    BackTrackExtrapolationRatio: float = 2.5  # :619
    BackTrackMinXfrac: float = 1e-10  # :620
    BackTrackMaxFuncSame: int = 3    # :621
    BackTrackGuardLower: float = 0.25  # :625
    BackTrackGuardUpper: float = 0.95  # :626
    uvDesiredWorkAndForceTolerances: tuple = (math.inf, 1e-15)   # :508
    uvDesiredWorkOrForceTolerances: tuple = (math.inf, 1e-15)    # :509
    uvExitBackTrackingStepLength: float = 1e-10                  # :510
    uvAcceptableWorkAndForceTolerances: tuple = (math.inf, 1e-15)  # :511
    uvAcceptableWorkOrForceTolerances: tuple = (math.inf, 1e-15)   # :512
    ModifiedNRuvIntervalCriterion: int = 1       # :582
    ModifiedNRuvReductionCriterion: float = 0.5  # :583
    # uvh
    theta: float = 0.5               # :377
    SUPG_beta0: float = 1.0          # :376
    uvh_SUPG_tau: str = "taus"       # :551
    uvh_SUPG_tauMultiplier: float = 1.0  # :555
    uvhDesiredWorkAndForceTolerances: tuple = (math.inf, 1e-15)    # :496
    uvhDesiredWorkOrForceTolerances: tuple = (math.inf, 1e-15)     # :498
    uvhExitBackTrackingStepLength: float = 1e-3                    # :502
    uvhAcceptableWorkAndForceTolerances: tuple = (math.inf, 1e-6)  # :504
    uvhAcceptableWorkOrForceTolerances: tuple = (1.0, 1e-8)        # :505
    ThicknessConstraints: int = 1                  # :1478 (active-set method)
    ThickMin: float = 1.0                          # :1469
    ThicknessConstraintsItMax: int = 10            # :1479
    MaxNumberOfNewlyIntroducedActiveThicknessConstraints: int = 1000  # :1500
    MinNumberOfNewlyIntroducedActiveThicknessConstraints: int = 0     # :1502
    ModifiedNRuvhIntervalCriterion: int = 1        # :584
    ModifiedNRuvhReductionCriterion: float = 0.5   # :585
    NLtol: float = 1e-15             # BackTracking.m:125-127 default
    SlidingLaw: str = "Weertman"     # :171
    Nzero: float = 1e-20             # :445
    IncludeMelangeModelPhysics: bool = False

    def set_force_tolerance(self, tol):
        """Set every force tolerance (desired and acceptable) to ``tol``."""
        self.uvDesiredWorkAndForceTolerances = (math.inf, tol)
        self.uvDesiredWorkOrForceTolerances = (math.inf, tol)
        self.uvAcceptableWorkAndForceTolerances = (math.inf, tol)
        self.uvAcceptableWorkOrForceTolerances = (math.inf, tol)


@dataclass
class Fields:
    """UaFields.m subset: nodal column vectors plus scalars."""
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
    s: np.ndarray = None
    b: np.ndarray = None
    GF: np.ndarray = None
    # uvh
    as_: np.ndarray = None
    ab: np.ndarray = None
    dasdh: np.ndarray = None
    dabdh: np.ndarray = None
    # other sliding laws (BasalDrag.m): Budd exponent q, Coulomb friction muk, Joughin V0
    q: np.ndarray = None
    muk: np.ndarray = None
    V0: np.ndarray = None
    # melange / ocean and atmosphere drag (CtrlVar.IncludeMelangeModelPhysics)
    uo: np.ndarray = None
    vo: np.ndarray = None
    Co: np.ndarray = None
    mo: np.ndarray = None
    ua: np.ndarray = None
    va: np.ndarray = None
    Ca: np.ndarray = None
    ma: np.ndarray = None

    def copy(self):
        out = Fields(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()})
        return out


@dataclass
class BCs:
    """BoundaryConditions subset (fixed and tied nodes, 0-based)."""
    ubFixedNode: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    ubFixedValue: np.ndarray = field(default_factory=lambda: np.zeros(0))
    vbFixedNode: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    vbFixedValue: np.ndarray = field(default_factory=lambda: np.zeros(0))
    ubTiedNodeA: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    ubTiedNodeB: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    vbTiedNodeA: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    vbTiedNodeB: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    hFixedNode: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    hFixedValue: np.ndarray = field(default_factory=lambda: np.zeros(0))
    ubvbFixedNormalNode: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    ubvbFixedNormalValue: np.ndarray = field(default_factory=lambda: np.zeros(0))


# ---------------------------------------------------------------------------
# Physics (EffectiveViscositySSTREAM.m, BasalDrag.m, HeavisideApprox.m,
# DiracDelta.m, Calc_bs_From_hBS.m)
# ---------------------------------------------------------------------------


def heaviside_approx(k, x, x0):
    """HeavisideApprox.m:86: 0.5 + 0.5 tanh(k (x-x0))."""
    return 0.5 + 0.5 * np.tanh(k * (x - x0))


def dirac_delta(k, x, x0):
    """DiracDelta.m:29: 0.5 k sech^2(k (x-x0))."""
    with np.errstate(over="ignore"):
        return 0.5 * k * (1.0 / np.cosh(k * (x - x0))) ** 2


def calc_bs_from_hBS(p: Params, h, S, B, rho, rhow):
    """Calc_bs_From_hBS.m:71-79,109 (Enforce_bAboveB=false, no thickness reset)."""
    hf = rhow * (S - B) / rho
    GF = heaviside_approx(p.kH, h - hf, p.Hh0)
    bfloat = S - rho * h / rhow
    b = GF * B + (1 - GF) * bfloat
    s = b + h
    return b, s, GF


def effective_viscosity(p: Params, A, n, exx, eyy, exy):
    """EffectiveViscositySSTREAM.m:7-9."""
    e = np.sqrt(p.EpsZero ** 2 + exx ** 2 + eyy ** 2 + exx * eyy + exy ** 2)
    eta = 0.5 * A ** (-1.0 / n) * e ** ((1 - n) / n) + p.etaZero
    E = (1 - n) / (4 * n) * A ** (-1.0 / n) * e ** ((1 - 3 * n) / n)
    return eta, E


def effective_pressure_n0(p, h, H, rho, rhow, g):
    """N0 inside BasalDrag.m (zeroth-order hydrology): N = rho g max(h-hf, 0) + Nzero,
    dN/dh = rho g where h > hf (else 0)."""
    hf = rhow * H / rho
    hf = np.where(hf < EPS, 0.0, hf)
    Dh = h - hf
    I = Dh < EPS
    Dh = np.where(I, 0.0, Dh)
    N = rho * g * Dh + p.Nzero
    dNdh = np.where(I, 0.0, rho * g + 0 * Dh)
    return N, dNdh


def _isotropic(T_over_U, Bcoef, ub, vb):
    """Drag of an isotropic law |tau| = T(U), tau = T(U) (u, v)/U with U = sqrt(u^2+v^2+u0^2):
    tau_x = A u, d tau_x/du = A + B u^2, d tau_x/dv = B u v, d tau_y/dv = A + B v^2, where
    A = T/U and B = (T' - T/U)/U^2."""
    A, B = T_over_U, Bcoef
    return A * ub, A * vb, A + B * ub * ub, B * ub * vb, B * ub * vb, A + B * vb * vb


def basal_drag(p: Params, He, delta, h, H, rho, rhow, g, ub, vb, C, m, q=None, muk=None, V0=None, melange=None):
    """BasalDrag.m:44-363 for CtrlVar.SlidingLaw (p.SlidingLaw) and the melange terms.

    Weertman/W (:184-186, Weertman :410-446), Budd/W-N0 (:188-191, Budd :448-490), Coulomb/C
    (:193-205, Coulomb :365-408), Tsai/minCW-N0 (:207-244: the smaller of the Weertman and
    Coulomb stresses), Cornford/rpCW-N0 (:246-252, rpCWN0.m), Umbi/rCW-N0 (:254-263, rCWN0.m),
    Joughin/rCW-V0 (:265-272, rCWV0.m).  The velocity derivatives of the last three follow from
    their stresses |tau| = mu N W/((mu N)^m + W^m)^(1/m), mu N W/(mu N + W) and
    W (U+V0)^(-1/m) with W = He (C+C0)^(-1/m) U^(1/m); their thickness derivatives are the
    reference's expressions.  ``melange`` = (uo, vo, Co, mo, ua, va, Ca, ma) adds the ocean and
    atmosphere drag on the floating part (:275-343).
    Returns taux, tauy, dtauxdu, dtauxdv, dtauydu, dtauydv, dtauxdh, dtauydh.
    """
    law = p.SlidingLaw
    delta = np.where(delta < 0, 0.0, delta)  # :48-49
    He = np.where(He < 0, 0.0, He)
    C0, u0 = p.Czero, p.SpeedZero
    speed = np.sqrt(ub * ub + vb * vb + u0 ** 2)  # :71-77
    Um = speed ** (1.0 / m - 1)
    beta2 = (C + C0) ** (-1.0 / m) * Um
    Dbeta2 = (1.0 / m - 1) * (C + C0) ** (-1.0 / m) * (ub ** 2 + vb ** 2 + u0 ** 2) ** ((1 - 3 * m) / (2 * m))
    zero = 0 * ub

    def weertman():
        return (He * beta2 * ub, He * beta2 * vb, He * (beta2 + Dbeta2 * ub * ub), He * Dbeta2 * ub * vb,
                He * Dbeta2 * ub * vb, He * (beta2 + Dbeta2 * vb * vb), delta * beta2 * ub, delta * beta2 * vb)

    def coulomb(N, dNdh, Dh):  # Coulomb :365-408
        Tau = muk * N
        tx, ty = Tau * ub / speed, Tau * vb / speed
        temp = speed ** 3
        dxu = Tau * (1 / speed - ub ** 2 / temp)
        dyv = Tau * (1 / speed - vb ** 2 / temp)
        dxv = -Tau * ub * vb / temp
        E = np.where(Dh < EPS, 0.0, muk * dNdh / speed)
        return tx, ty, dxu, dxv, dxv, dyv, E * ub, E * vb

    if law in ("Weertman", "W"):
        out = weertman()
    elif law in ("Budd", "W-N0"):  # Budd :448-490
        N, dNdh = effective_pressure_n0(p, h, H, rho, rhow, g)
        qm = q / m
        Nqm = N ** qm
        T = He * Nqm * beta2
        E = delta * T + He * qm * N ** (qm - 1) * dNdh * beta2
        out = (T * ub, T * vb, He * Nqm * (beta2 + Dbeta2 * ub * ub), He * Nqm * Dbeta2 * ub * vb,
               He * Nqm * Dbeta2 * ub * vb, He * Nqm * (beta2 + Dbeta2 * vb * vb), E * ub, E * vb)
    elif law in ("Coulomb", "C"):
        N, dNdh = effective_pressure_n0(p, h, H, rho, rhow, g)
        hf = rhow * H / rho
        hf = np.where(hf < EPS, 0.0, hf)
        Dh = h - hf
        Dh = np.where(Dh < EPS, 0.0, Dh)
        out = coulomb(N, dNdh, Dh)
    elif law in ("Tsai", "minCW-N0"):
        hf = rhow * H / rho
        hf = np.where(hf < EPS, 0.0, hf)
        Dh = h - hf
        Dh = np.where(Dh < EPS, 0.0, Dh)
        N, dNdh = effective_pressure_n0(p, h, H, rho, rhow, g)
        W = weertman()
        Cc = coulomb(N, dNdh, Dh)
        isC = Cc[0] * Cc[0] + Cc[1] * Cc[1] < W[0] * W[0] + W[1] * W[1]
        out = tuple(np.where(isC, c, w) for w, c in zip(W, Cc))
        out = out[:4] + (out[3],) + out[5:]  # dtauydu = dtauxdv
    elif law in ("Cornford", "rpCW-N0"):
        N, dNdh = effective_pressure_n0(p, h, H, rho, rhow, g)
        c = (C + C0) ** (-1.0 / m)
        W = He * c * speed ** (1.0 / m)
        muN = muk * N
        S = muN ** m + W ** m
        T_U = muN * He * c * speed ** (1.0 / m - 1) * S ** (-1.0 / m)
        Tp = muN * (W / (m * speed)) * muN ** m * S ** (-1.0 / m - 1)
        out = _isotropic(T_U, (Tp - T_U) / speed ** 2, ub, vb)
        Wm = (c * speed ** (1.0 / m)) ** m
        Eh = (2.0 ** (m + 1) * muN ** (m + 1) * delta * c * speed ** (1.0 / m - 1)
              * (2.0 ** m * muN ** m + Wm) ** (-(m + 1) / m)
              + muk * dNdh * He ** (m + 1) * c * speed ** (1.0 / m - 1) * Wm * S ** (-(m + 1) / m))
        out = out + (Eh * ub, Eh * vb)
    elif law in ("Umbi", "rCW-N0"):
        N, dNdh = effective_pressure_n0(p, h, H, rho, rhow, g)
        c1 = (C + C0) ** (1.0 / m)
        muN = muk * N
        den = muN * c1 + He * speed ** (1.0 / m)
        T_U = muN * He * speed ** (1.0 / m - 1) / den
        W = He * speed ** (1.0 / m) / c1
        Tp = muN ** 2 * W / (m * speed * (muN + W) ** 2)
        out = _isotropic(T_U, (Tp - T_U) / speed ** 2, ub, vb)
        Eh = (muk * dNdh * He * speed ** (2.0 / m - 1) / den ** 2
              + 4.0 * muk ** 2 * N ** 2 * delta * c1 * speed ** (1.0 / m - 1) / (2 * muN * c1 + speed ** (1.0 / m)) ** 2)
        out = out + (Eh * ub, Eh * vb)
    elif law in ("Joughin", "rCW-V0"):
        c = (C + C0) ** (-1.0 / m)
        T_U = He * c * (V0 + speed) ** (-1.0 / m) * speed ** (1.0 / m - 1)
        Tp = T_U * speed * V0 / (m * speed * (speed + V0))
        out = _isotropic(T_U, (Tp - T_U) / speed ** 2, ub, vb)
        Eh = delta * c * (V0 + speed) ** (-1.0 / m) * speed ** (1.0 / m - 1)
        out = out + (Eh * ub, Eh * vb)
    else:
        raise ValueError("BasalDrag:CaseNotFound")
    out = [o + zero for o in out]
    if melange is not None:  # :275-343
        uo, vo, Co, mo, ua_, va_, Ca, ma = melange
        for (uw, vw, Cw, mw) in ((uo, vo, Co, mo), (ua_, va_, Ca, ma)):
            U, V = ub - uw, vb - vw
            b2 = (Cw + C0) ** (-1.0 / mw) * np.sqrt(U * U + V * V + u0 ** 2) ** (1.0 / mw - 1)
            Db2 = (1.0 / mw - 1) * (Cw + C0) ** (-1.0 / mw) * (U ** 2 + V ** 2 + u0 ** 2) ** ((1 - 3 * mw) / (2 * mw))
            add = ((1 - He) * b2 * U, (1 - He) * b2 * V, (1 - He) * (b2 + Db2 * U * U), (1 - He) * (Db2 * U * V),
                   (1 - He) * (Db2 * U * V), (1 - He) * (b2 + Db2 * V * V), -delta * b2 * U, -delta * b2 * V)
            out = [a + b for a, b in zip(out, add)]
    return tuple(out)


def _drag_extras(p: Params, F: Fields, conn, fun):
    """Integration-point values of the sliding-law fields (uvMatrixAssemblySSTREAM.m:210-254):
    q, muk and V0 where the law uses them, and the melange fields when
    CtrlVar.IncludeMelangeModelPhysics is on."""
    at = lambda v: None if v is None else np.asarray(v, dtype=float)[conn] @ fun
    out = {"q": at(F.q), "muk": at(F.muk), "V0": at(F.V0)}
    if p.IncludeMelangeModelPhysics:
        out["melange"] = tuple(at(getattr(F, k)) for k in ("uo", "vo", "Co", "mo", "ua", "va", "Ca", "ma"))
    return out


def basal_drag_weertman(p: Params, He, delta, ub, vb, C, m):
    """BasalDrag.m:54-77 (clamps, β², Dβ²), :184-186 dispatch, Weertman :410-446.

    Returns taux, tauy, dtauxdu, dtauxdv, dtauydu, dtauydv, dtauxdh, dtauydh.
    """
    delta = np.where(delta < 0, 0.0, delta)
    He = np.where(He < 0, 0.0, He)
    C0 = p.Czero
    u0 = p.SpeedZero
    speed = np.sqrt(ub * ub + vb * vb + u0 ** 2)
    Um = speed ** (1.0 / m - 1)
    beta2 = (C + C0) ** (-1.0 / m) * Um
    Dbeta2 = (1.0 / m - 1) * (C + C0) ** (-1.0 / m) * (ub ** 2 + vb ** 2 + u0 ** 2) ** ((1 - 3 * m) / (2 * m))
    taux = He * beta2 * ub
    tauy = He * beta2 * vb
    dtauxdu = He * (beta2 + Dbeta2 * ub * ub)
    dtauydv = He * (beta2 + Dbeta2 * vb * vb)
    dtauxdv = He * Dbeta2 * ub * vb
    dtauydu = dtauxdv
    dtauxdh = delta * beta2 * ub
    dtauydh = delta * beta2 * vb
    return taux, tauy, dtauxdu, dtauxdv, dtauydu, dtauydv, dtauxdh, dtauydh


# ---------------------------------------------------------------------------
# uv assembly — UaMain/uvMatrixAssemblySSTREAM.m
# ---------------------------------------------------------------------------


_COMPILED = {"lib": None, "threads": 1}


def use_compiled_element_loop(enable=True, threads=1):
    """Run uv_matrix_assembly's element loop in the C++ restatement (oracle/ua_ref_asm.cpp,
    built by oracle/Makefile) on ``threads`` host threads, or back in numpy (the default)."""
    import ctypes
    import os
    if not enable:
        _COMPILED["lib"] = None
        return
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libua_ref_asm.so")
    lib = ctypes.CDLL(path)
    lib.uvref_element_loop.restype = ctypes.c_int
    _COMPILED["lib"] = lib
    _COMPILED["threads"] = int(threads)


def _compiled_element_loop(mua, funs, F, ub, vb, par, Ronly, K, T):
    import ctypes
    lib = _COMPILED["lib"]
    c = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    keep = [np.ascontiguousarray(mua.connectivity, dtype=np.int64), c(mua.Deriv), c(mua.DetJ), c(mua.weights),
            c(funs), c(F.h), c(F.s), c(ub), c(vb), c(F.C), c(F.m), c(F.AGlen), c(F.n), c(F.S), c(F.B), c(F.rho),
            c(par)]
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a is not None else None
    outs = list(K) if K is not None else [None] * 4
    outs += list(T)
    rc = lib.uvref_element_loop(ctypes.c_int64(mua.Nele), ctypes.c_int(mua.nod), ctypes.c_int(mua.nip),
                                *[ptr(a) for a in keep], ctypes.c_int(1 if Ronly else 0),
                                ctypes.c_int(_COMPILED["threads"]), *[ptr(a) for a in outs])
    if rc != 0:
        raise RuntimeError("uvref_element_loop failed")


def _matlab_sparse(I, J, V, m, n):
    """MATLAB ``sparse(I,J,V,m,n)``: sum duplicates, keep non-zeros only (CSC)."""
    A = sp.coo_matrix((V, (I, J)), shape=(m, n)).tocsc()
    A.sum_duplicates()
    A.eliminate_zeros()
    A.sort_indices()
    return A


def uv_matrix_assembly(p: Params, mua: MUA, F: Fields, bcs: BCs = None, Ronly=False, ZeroFields=False,
                       return_parts=False):
    """uvMatrixAssemblySSTREAM.m:6-553 (post-2025 default, no melange, Weertman).

    Returns (R, K) with R a dense 2Nn vector (Tint-Fext) and K the symmetrised
    CSC tangent ``(K+K.')/2`` (None when Ronly).  ``return_parts`` also returns
    Tint and Fext.
    """
    ub, vb = F.ub, F.vb
    if ZeroFields:  # :24-28
        ub = np.zeros_like(ub)
        vb = np.zeros_like(vb)
        if bcs is not None:
            ub[bcs.ubFixedNode] = bcs.ubFixedValue
            vb[bcs.vbFixedNode] = bcs.vbFixedValue
    if np.any(np.isnan(ub)) or np.any(np.isnan(vb)):  # :63-64
        raise FloatingPointError("uvMatrixAssembly:NaN")
    Dvisk = 0.0 if p.Picard else p.NRviscosity  # :67-71
    g = F.g
    Nele, nod, Nn = mua.Nele, mua.nod, mua.Nnodes
    neq = 2 * Nn
    conn = mua.connectivity
    hnod = F.h[conn]; snod = F.s[conn]
    ubnod = ub[conn]; vbnod = vb[conn]
    Cnod = F.C[conn]; mnod = F.m[conn]
    AGlennod = F.AGlen[conn]; nnod = F.n[conn]
    Snod = F.S[conn]; Bnod = F.B[conn]
    rhonod = F.rho[conn]
    ca, sa = math.cos(F.alpha), math.sin(F.alpha)

    if not Ronly:
        d1d1 = np.zeros((Nele, nod, nod)); d2d2 = np.zeros((Nele, nod, nod))
        d1d2 = np.zeros((Nele, nod, nod)); d2d1 = np.zeros((Nele, nod, nod))
    Tx = np.zeros((Nele, nod)); Ty = np.zeros((Nele, nod))
    Fx = np.zeros((Nele, nod)); Fy = np.zeros((Nele, nod))

    compiled = (_COMPILED["lib"] is not None and p.SlidingLaw in ("Weertman", "W")
                and not p.IncludeMelangeModelPhysics)
    if compiled:  # the same element loop in C++ (oracle/ua_ref_asm.cpp), Weertman drag
        par = np.array([p.kH, p.Hh0, p.SpeedZero, p.EpsZero, p.etaZero, p.Czero, p.Cmin, p.AGlenmin, Dvisk,
                        F.rhow, g, ca, sa])
        funs = np.array([shape_fun(nod, mua.points[i]) for i in range(mua.nip)])
        _compiled_element_loop(mua, funs, F, ub, vb, par, Ronly, None if Ronly else (d1d1, d2d2, d1d2, d2d1),
                               (Tx, Fx, Ty, Fy))
    for Iint in (range(mua.nip) if not compiled else ()):  # :168
        fun = shape_fun(nod, mua.points[Iint])
        Deriv = mua.Deriv[:, :, :, Iint]
        detJ = mua.DetJ[:, Iint]
        hint = hnod @ fun; sint = snod @ fun
        uint = ubnod @ fun; vint = vbnod @ fun
        Cint = Cnod @ fun
        Cint = np.where(Cint < p.Cmin, p.Cmin, Cint)  # :205
        mint = mnod @ fun
        AGlenint = AGlennod @ fun
        AGlenint = np.where(AGlenint < p.AGlenmin, p.AGlenmin, AGlenint)  # :243
        nint = nnod @ fun
        Bint = Bnod @ fun; Sint = Snod @ fun
        Hint = Sint - Bint
        rhoint = rhonod @ fun
        # post-2025 flotation at integration points :300-310
        hfint = F.rhow * Hint / rhoint
        Heint = heaviside_approx(p.kH, hint - hfint, p.Hh0)
        HEint = heaviside_approx(p.kH, hfint - hint, p.Hh0)
        deltaint = dirac_delta(p.kH, hint - hfint, p.Hh0)
        Hposint = heaviside_approx(p.kH, Hint, p.Hh0) * Hint
        dint = HEint * rhoint * hint / F.rhow + Heint * Hposint
        # nodal-derivative sums :322-347
        dsdx = np.zeros(Nele); dhdx = np.zeros(Nele); dsdy = np.zeros(Nele); dhdy = np.zeros(Nele)
        exx = np.zeros(Nele); eyy = np.zeros(Nele); exy = np.zeros(Nele)
        for Inod in range(nod):
            dsdx = dsdx + Deriv[:, 0, Inod] * snod[:, Inod]
            dhdx = dhdx + Deriv[:, 0, Inod] * hnod[:, Inod]
            dsdy = dsdy + Deriv[:, 1, Inod] * snod[:, Inod]
            dhdy = dhdy + Deriv[:, 1, Inod] * hnod[:, Inod]
            exx = exx + Deriv[:, 0, Inod] * ubnod[:, Inod]
            eyy = eyy + Deriv[:, 1, Inod] * vbnod[:, Inod]
            exy = exy + 0.5 * (Deriv[:, 0, Inod] * vbnod[:, Inod] + Deriv[:, 1, Inod] * ubnod[:, Inod])
        taux, tauy, dtauxdu, dtauxdv, dtauydu, dtauydv, _, _ = basal_drag(
            p, Heint, deltaint, hint, Hint, rhoint, F.rhow, g, uint, vint, Cint, mint,
            **_drag_extras(p, F, conn, fun))  # :351-352
        etaint, Eint = effective_viscosity(p, AGlenint, nint, exx, eyy, exy)  # :353
        dbdx = dsdx - dhdx; dbdy = dsdy - dhdy  # :357
        detJw = detJ * mua.weights[Iint]  # :359
        for Inod in range(nod):  # :362
            if not Ronly:
                for Jnod in range(nod):
                    d1d1[:, Inod, Jnod] += (4 * hint * etaint * Deriv[:, 0, Inod] * Deriv[:, 0, Jnod]
                                            + hint * etaint * Deriv[:, 1, Inod] * Deriv[:, 1, Jnod]
                                            + dtauxdu * fun[Jnod] * fun[Inod]) * detJw
                    d2d2[:, Inod, Jnod] += (4 * hint * etaint * Deriv[:, 1, Inod] * Deriv[:, 1, Jnod]
                                            + hint * etaint * Deriv[:, 0, Inod] * Deriv[:, 0, Jnod]
                                            + dtauydv * fun[Jnod] * fun[Inod]) * detJw
                    d1d2[:, Inod, Jnod] += (etaint * hint * (2 * Deriv[:, 0, Inod] * Deriv[:, 1, Jnod]
                                                             + Deriv[:, 1, Inod] * Deriv[:, 0, Jnod])
                                            + dtauxdv * fun[Jnod] * fun[Inod]) * detJw
                    d2d1[:, Inod, Jnod] += (etaint * hint * (2 * Deriv[:, 1, Inod] * Deriv[:, 0, Jnod]
                                                             + Deriv[:, 0, Inod] * Deriv[:, 1, Jnod])
                                            + dtauydu * fun[Jnod] * fun[Inod]) * detJw
                    Deu = Eint * ((2 * exx + eyy) * Deriv[:, 0, Jnod] + exy * Deriv[:, 1, Jnod])  # :398
                    Dev = Eint * ((2 * eyy + exx) * Deriv[:, 1, Jnod] + exy * Deriv[:, 0, Jnod])
                    E11 = hint * (4 * exx + 2 * eyy) * Deu * Deriv[:, 0, Inod] + 2 * hint * exy * Deu * Deriv[:, 1, Inod]
                    E12 = hint * (4 * exx + 2 * eyy) * Dev * Deriv[:, 0, Inod] + 2 * hint * exy * Dev * Deriv[:, 1, Inod]
                    E22 = hint * (4 * eyy + 2 * exx) * Dev * Deriv[:, 1, Inod] + 2 * hint * exy * Dev * Deriv[:, 0, Inod]
                    E21 = hint * (4 * eyy + 2 * exx) * Deu * Deriv[:, 1, Inod] + 2 * hint * exy * Deu * Deriv[:, 0, Inod]
                    d1d1[:, Inod, Jnod] += Dvisk * E11 * detJw  # :421-424
                    d2d2[:, Inod, Jnod] += Dvisk * E22 * detJw
                    d1d2[:, Inod, Jnod] += Dvisk * E12 * detJw
                    d2d1[:, Inod, Jnod] += Dvisk * E21 * detJw
            # residual terms :431-449
            t1 = -g * (rhoint * hint - F.rhow * dint) * dbdx * fun[Inod] * ca + rhoint * g * hint * sa * fun[Inod]
            t2 = 0.5 * g * ca * (rhoint * hint ** 2 - F.rhow * dint ** 2) * Deriv[:, 0, Inod]
            t3 = hint * etaint * (4 * exx + 2 * eyy) * Deriv[:, 0, Inod]
            t4 = hint * etaint * 2 * exy * Deriv[:, 1, Inod]
            t5 = taux * fun[Inod]
            Tx[:, Inod] += (t3 + t4 + t5) * detJw
            Fx[:, Inod] += (t1 + t2) * detJw
            t1 = -g * (rhoint * hint - F.rhow * dint) * dbdy * fun[Inod] * ca
            t2 = 0.5 * ca * g * (rhoint * hint ** 2 - F.rhow * dint ** 2) * Deriv[:, 1, Inod]
            t3 = hint * etaint * (4 * eyy + 2 * exx) * Deriv[:, 1, Inod]
            t4 = hint * etaint * 2 * exy * Deriv[:, 0, Inod]
            t5 = tauy * fun[Inod]
            Ty[:, Inod] += (t3 + t4 + t5) * detJw
            Fy[:, Inod] += (t1 + t2) * detJw

    # R scatter :462-488 (sparse accumulate, here dense bincount)
    iR = np.concatenate([np.concatenate([conn[:, I], conn[:, I] + Nn]) for I in range(nod)])
    Tval = np.concatenate([np.concatenate([Tx[:, I], Ty[:, I]]) for I in range(nod)])
    Fval = np.concatenate([np.concatenate([Fx[:, I], Fy[:, I]]) for I in range(nod)])
    Tint = np.bincount(iR, weights=Tval, minlength=neq)
    Fext = np.bincount(iR, weights=Fval, minlength=neq)
    R = Tint - Fext
    K = None
    if not Ronly:  # :490-534
        Ii, Jj, Xv = [], [], []
        for Inod in range(nod):
            for Jnod in range(nod):
                Ii += [conn[:, Inod], conn[:, Inod] + Nn, conn[:, Inod], conn[:, Inod] + Nn]
                Jj += [conn[:, Jnod], conn[:, Jnod] + Nn, conn[:, Jnod] + Nn, conn[:, Jnod]]
                Xv += [d1d1[:, Inod, Jnod], d2d2[:, Inod, Jnod], d1d2[:, Inod, Jnod], d2d1[:, Inod, Jnod]]
        K = _matlab_sparse(np.concatenate(Ii), np.concatenate(Jj), np.concatenate(Xv), neq, neq)
        K = (K + K.T) / 2  # :530-531
        K = K.tocsc()
        K.eliminate_zeros()
        K.sort_indices()
    if return_parts:
        return R, K, Tint, Fext
    return R, K


def structural_pattern(mua: MUA, ndof: int):
    """Structural (connectivity-implied) pattern of the ndof-block tangent, CSR with sorted columns."""
    conn = mua.connectivity
    Nn, nod = mua.Nnodes, mua.nod
    I = np.repeat(conn, nod, axis=1).ravel()
    J = np.tile(conn, (1, nod)).ravel()
    rows, cols = [], []
    for a in range(ndof):
        for b in range(ndof):
            rows.append(I + a * Nn)
            cols.append(J + b * Nn)
    A = sp.coo_matrix((np.ones(len(I) * ndof * ndof), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(ndof * Nn, ndof * Nn)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    return A.indptr.copy(), A.indices.copy()


# ---------------------------------------------------------------------------
# Constraints — CreateLuv.m:2-78, ScaleL.m:28-33, BCs2MLC.m:19-20,49
# ---------------------------------------------------------------------------


def boundary_edges(connectivity, Nnodes):
    """The boundary edges of the mesh (FindBoundary.m: the element edges that belong to one
    element), each as [start, (mid,) end] in its element's node order."""
    nod = connectivity.shape[1]
    corners = [0, 1, 2] if nod == 3 else [0, 2, 4]
    edges = []
    for k in range(3):
        a = connectivity[:, corners[k]]
        b = connectivity[:, corners[(k + 1) % 3]]
        if nod == 6:
            edges.append(np.stack([a, connectivity[:, corners[k] + 1], b], axis=1))
        else:
            edges.append(np.stack([a, b], axis=1))
    E = np.concatenate(edges)
    key = np.minimum(E[:, 0], E[:, -1]) * Nnodes + np.maximum(E[:, 0], E[:, -1])
    _, inv, cnt = np.unique(key, return_inverse=True, return_counts=True)
    return E[cnt[inv] == 1]


def nodal_normals(coordinates, connectivity):
    """CalcEdgeAndNodalNormals.m:9-40: unit edge normals (-dy, dx)/l of the boundary edges and the
    nodal normals (start node: the edge's normal, end node: plus the edge's normal, P2 mid node:
    the mean of its two sub-edges), normalised.  Returns (Nx, Ny) over all nodes."""
    Nn = coordinates.shape[0]
    E = boundary_edges(connectivity, Nn)
    nsub = E.shape[1] - 1
    x, y = coordinates[:, 0], coordinates[:, 1]
    nx = np.zeros((E.shape[0], nsub)); ny = np.zeros((E.shape[0], nsub))
    for I in range(nsub):
        dx = x[E[:, I + 1]] - x[E[:, I]]
        dy = y[E[:, I + 1]] - y[E[:, I]]
        l = np.sqrt(dy * dy + dx * dx)
        nx[:, I] = -dy / l
        ny[:, I] = dx / l
    Nx = np.zeros(Nn); Ny = np.zeros(Nn)
    Nx[E[:, 0]] = nx[:, 0]; Ny[E[:, 0]] = ny[:, 0]
    Nx[E[:, -1]] = Nx[E[:, -1]] + nx[:, nsub - 1]
    Ny[E[:, -1]] = Ny[E[:, -1]] + ny[:, nsub - 1]
    for I in range(1, nsub):
        Nx[E[:, I]] = Nx[E[:, I]] + (nx[:, I - 1] + nx[:, I]) / 2
        Ny[E[:, I]] = Ny[E[:, I]] + (ny[:, I - 1] + ny[:, I]) / 2
    with np.errstate(invalid="ignore", divide="ignore"):
        l = np.sqrt(Nx * Nx + Ny * Ny)
        return Nx / l, Ny / l


def create_Luv(Nnodes, bcs: BCs, mua: MUA = None):
    """BCs2MLC.m:19-29 + CreateLuv.m:28-76 + ScaleL.m:28-33 (u ties, v ties, fixed u, fixed v,
    fixed normal velocities Nx u + Ny v = -value with the nodal normals of the mesh)."""
    ufn, ui = np.unique(bcs.ubFixedNode, return_index=True)
    ufv = np.asarray(bcs.ubFixedValue, dtype=float)[ui]
    vfn, vi = np.unique(bcs.vbFixedNode, return_index=True)
    vfv = np.asarray(bcs.vbFixedValue, dtype=float)[vi]
    ia, ib, xv, b = [], [], [], []
    JJ = 0
    for A_, B_ in zip(bcs.ubTiedNodeA, bcs.ubTiedNodeB):
        ia += [JJ, JJ]; ib += [A_, B_]; xv += [1.0, -1.0]; b.append(0.0); JJ += 1
    for A_, B_ in zip(bcs.vbTiedNodeA, bcs.vbTiedNodeB):
        ia += [JJ, JJ]; ib += [A_ + Nnodes, B_ + Nnodes]; xv += [1.0, -1.0]; b.append(0.0); JJ += 1
    for nI, val in zip(ufn, ufv):
        ia.append(JJ); ib.append(nI); xv.append(1.0); b.append(val); JJ += 1
    for nI, val in zip(vfn, vfv):
        ia.append(JJ); ib.append(nI + Nnodes); xv.append(1.0); b.append(val); JJ += 1
    if len(bcs.ubvbFixedNormalNode):
        Nx, Ny = nodal_normals(mua.coordinates, mua.connectivity)
        for nI, val in zip(bcs.ubvbFixedNormalNode, bcs.ubvbFixedNormalValue):
            ia += [JJ, JJ]; ib += [nI, nI + Nnodes]; xv += [Nx[nI], Ny[nI]]; b.append(-val); JJ += 1
    if JJ == 0:
        return None, None
    L = _matlab_sparse(np.array(ia), np.array(ib), np.array(xv), JJ, 2 * Nnodes).tocsr()
    c = np.array(b)
    Lscale = np.sqrt(np.asarray(L.multiply(L).sum(axis=1)).ravel())  # ScaleL.m:29
    S = sp.diags(1.0 / Lscale)
    return (S @ L).tocsr(), S @ c


# ---------------------------------------------------------------------------
# Linear solve — ABfgPreEliminate.m:29-160
# ---------------------------------------------------------------------------


def _splu(A):
    """Sparse LU with UMFPACK's symmetric strategy, which MATLAB's ``decomposition`` applies to a
    matrix of (nearly) symmetric pattern with a non-zero diagonal: a minimum-degree ordering of
    A+A' and diagonal pivots unless an entry falls below 0.001 of its column's largest
    (UMFPACK's default symmetric pivot tolerance)."""
    return spla.splu(A, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.001, options=dict(SymmetricMode=True))


def abfg_pre_eliminate(A, B, f, g):
    """ABfgPreEliminate.m:29-160 with SuperLU in place of MATLAB ``decomposition``."""
    A = sp.csc_matrix(A)
    if B is None or B.shape[0] == 0:
        return spla.spsolve(A, f), np.zeros(0)
    B = sp.csr_matrix(B)
    BBT = (B @ B.T).toarray()
    if not np.allclose(BBT, np.diag(np.diag(BBT)), atol=0, rtol=0):
        raise ValueError("ABfgPreEliminate:B B*B^T not diagonal")
    Scale = np.ones(B.shape[0])
    if not np.all(np.abs(np.diag(BBT) - 1) < 1000 * EPS):  # :38-45
        Lscale = np.sqrt(np.diag(BBT))
        Scale = 1.0 / Lscale
        B = sp.diags(Scale) @ B
        g = Scale * g
    dA = np.abs(A.diagonal())
    factor = 1.0 / np.mean(dA) if np.mean(dA) != 0 else 1.0  # :49-53
    if not np.isfinite(factor):
        factor = 1.0
    BtB = (B.T @ B).tocsc()
    As = factor * A
    fs = factor * f
    Q = sp.identity(A.shape[0], format="csc") - BtB  # :61
    Atilde = (Q @ As + BtB).tocsc()  # :62
    btilde = Q @ fs + B.T @ g  # :63
    # :110-115 decomposition(Atilde) and solve.  MATLAB factors a square sparse
    # unsymmetric matrix with UMFPACK, which applies iterative refinement
    # (UMFPACK_IRSTEP, default 2 steps); SuperLU is used here with the same
    # number of refinement steps.
    lu = _splu(Atilde)
    x = lu.solve(btilde)
    for _ in range(2):
        x = x + lu.solve(btilde - Atilde @ x)
    y = B @ (fs - As @ x)  # :138
    y = y / factor  # :142
    y = Scale * y  # :159
    return x, y


# ---------------------------------------------------------------------------
# Cost function and convergence tests
# ---------------------------------------------------------------------------


def calc_cost_function_nr(p, mua, gamma, F, fext0, L, lubvb, cuv, dub, dvb, dl, bcs=None):
    """CalcCostFunctionNR.m:14-47.  Returns (r, rForce, rWork, D2, frhs, grhs)."""
    if gamma != gamma:
        raise ValueError("gamma is nan")
    Fg = F.copy()
    Fg.ub = F.ub + gamma * dub
    Fg.vb = F.vb + gamma * dvb
    lg = lubvb + gamma * dl if L is not None else None
    R, _ = uv_matrix_assembly(p, mua, Fg, bcs, Ronly=True)
    if L is not None:
        frhs = -R - L.T @ lg
        grhs = cuv - L @ np.concatenate([Fg.ub, Fg.vb])
        fg = np.concatenate([frhs, grhs])
        dd = np.concatenate([dub, dvb, dl])
    else:
        frhs = -R
        grhs = np.zeros(0)
        fg = frhs
        dd = np.concatenate([dub, dvb])
    Normalisation = fext0 @ fext0 + 1000 * EPS
    rForce = (fg @ fg) / Normalisation
    D2 = fg @ dd
    rWork = D2 ** 2
    return rForce, rForce, rWork, D2, frhs, grhs


def uv_residuals_criteria(p: Params, rForce, rWork, iteration, gamma):
    """uvResidualsCriteria.m:1-23."""
    if gamma > max(p.uvExitBackTrackingStepLength, p.BacktrackingGammaMin):
        a, o = p.uvDesiredWorkAndForceTolerances, p.uvDesiredWorkOrForceTolerances
    else:
        a, o = p.uvAcceptableWorkAndForceTolerances, p.uvAcceptableWorkOrForceTolerances
    return ((rWork < a[0] and rForce < a[1]) and (rWork < o[0] or rForce < o[1])
            and iteration >= p.NRitmin)


# ---------------------------------------------------------------------------
# Line search — BackTracking.m, CubicFit.m, parabolamin.m, rLineminUa.m
# ---------------------------------------------------------------------------


def parabolamin(a, b, c, fa, fb, fc):
    """parabolamin.m (3-point parabola minimum with non-convex fallbacks)."""
    if c < b:
        b, c, fb, fc = c, b, fc, fb
    if not (a < b < c):
        return math.nan, 1
    if math.isinf(fa) and math.isinf(fb) and math.isinf(fc):
        return a / 100, 1
    if math.isinf(fb) and math.isinf(fc):
        return (b / 100 if b == b else 1e-5), 1
    t1 = (b - a) ** 2 * (fb - fc)
    t2 = (b - c) ** 2 * (fb - fa)
    t3 = (b - a) * (fb - fc)
    t4 = (b - c) * (fb - fa)
    status = 0
    if t3 != t4:
        xmin = b - 0.5 * (t1 - t2) / (t3 - t4)
    else:
        xmin, status = math.nan, 1
    if xmin != xmin or (fa + (b - a) * (fc - fa) / (c - a) < fb):
        if fc < fb < fa:
            xmin = 5 * c
        elif fc > fb > fa:
            xmin = a + b / 10
        elif fc > fa and fb > fa:
            xmin = a + b / 100
        else:
            xmin = (a + b) / 3
    return xmin, status


def cubic_fit(slope, y0, y1, y2, x1, x2):
    """CubicFit.m: minimum of the cubic through (0,y0) with slope, (x1,y1), (x2,y2)."""
    if any(v != v for v in (y0, y1, y2, x1, x2)):
        raise ValueError("CubicFit:nanOnInput")
    if x1 > x2:
        x1, x2, y1, y2 = x2, x1, y2, y1
    status = 0
    if x1 == x2:
        D = (y1 - y0) / x1 - slope
        xmin = -x1 * slope / 2 / D if D != 0 else x1 * 0.9
    else:
        M = np.array([[1 / x1 ** 2, -1 / x2 ** 2], [-x2 / x1 ** 2, x1 / x2 ** 2]])
        ab = (M @ np.array([y1 - slope * x1 - y0, y2 - slope * x2 - y0])) / (x1 - x2)
        disc = ab[1] ** 2 - 3 * ab[0] * slope
        if ab[0] == 0 or disc < 0:
            xmin = math.nan
        else:
            xmin = (-ab[1] + math.sqrt(disc)) / 3 / ab[0]
        if ab[0] == 0 or xmin != xmin:
            if slope == slope:
                D = (y1 - y0) / x1 - slope
                xmin = -x1 * slope / 2 / D if D != 0 else math.nan
            else:
                xmin, status = parabolamin(0, x1, x2, y0, y1, y2)
    if xmin != xmin:
        if y0 < y1 < y2:
            xmin = x1 / 2
        elif y0 > y1 > y2:
            xmin = x1 + (x2 - x1) / 2
        elif y0 < y1 and y1 > y2:
            xmin = x1 + (x2 - x1) / 2 if y2 < y0 else x1 / 2
    return xmin, status


@dataclass
class BackTrackInfo:
    Converged: int = 0
    iarm: int = 0
    nFuncEval: int = 0
    nExtrapolationSteps: int = 0
    Infovector: list = field(default_factory=list)


def backtracking(slope0, b, fa, fb, func, p: Params, GammaMin=None, AcceptRatio=None, AllowExtrapolation=None):
    """BackTracking.m:54-759 (no plotting).  ``func(gamma) -> f``.

    ``GammaMin``/``AcceptRatio``/``AllowExtrapolation`` are the CtrlVar
    overrides rLineminUa.m sets before calling (e.g. :87, :241-243).
    """
    beta = p.BackTrackBeta
    MaxIterations = p.BackTrackMaxIterations
    MaxExtrapolations = p.BackTrackMaxExtrapolations
    ExtrapolationRatio = p.BackTrackExtrapolationRatio
    MinXfrac = p.BackTrackMinXfrac * b
    MaxFuncSame = p.BackTrackMaxFuncSame
    BacktrackingGammaMin = p.BacktrackingGammaMin if GammaMin is None else GammaMin
    NewtonAcceptRatio = p.NewtonAcceptRatio if AcceptRatio is None else AcceptRatio
    allow_ext = p.LineSearchAllowedToUseExtrapolation if AllowExtrapolation is None else AllowExtrapolation
    GL, GU = p.BackTrackGuardLower, p.BackTrackGuardUpper
    ContinueRatio = 0.5  # :147
    info = BackTrackInfo()
    nfe = 0
    NoSlope = slope0 is None or slope0 != slope0
    if not NoSlope and slope0 > 0:
        return math.nan, math.nan, info
    target = max(NewtonAcceptRatio * fa, p.NLtol)  # :160
    if not NoSlope:
        tws = min(fa + beta * slope0 * b, NewtonAcceptRatio * fa)
        target = max(target, tws)
        if target < 0:
            target = max(NewtonAcceptRatio * fa, p.NLtol)
    xfrac = 1e10
    iMinSame = 0
    iMinSameWB = 0
    iarm = 0
    a = 0.0
    if fa is None or fa != fa:
        fa = func(a); nfe += 1
    f0 = fa
    if fb is None or fb != fb:
        if b is None or b != b:
            b = 1.0
        fb = func(b); nfe += 1
    Info = [[a, fa], [b, fb]]

    def cur_min():
        fm = min(v[1] for v in Info)
        for v in Info:
            if v[1] == fm:
                return v[0], fm

    gmin, fmin = cur_min()
    if fb < target:  # :239-265
        info.Converged = 1
        info.nFuncEval = nfe
        info.Infovector = Info
        return gmin, fmin, info
    if not NoSlope:
        gamma = -b * slope0 / 2 / ((fb - fa) / b - slope0)  # :268
    else:
        gamma = a + 0.9 * (b - a)
    if gamma > GU * b:
        gamma = GU * b
    elif gamma < GL * b:
        gamma = GL * b
    if fmin > target:  # :282
        iarm = 1
        fgamma = func(gamma); nfe += 1
        gammaOld = gamma
        Info.append([gamma, fgamma])
    else:
        gammaOld = gamma; gamma = b; fgamma = fb
    gmin, fmin = cur_min()
    c = b; fc = fb; b = gamma; fb = fgamma  # :306
    Extrapolation = 0
    fbOld = bOld = None
    if allow_ext:
        while fb < fa and fc < fb and fmin > target:
            Extrapolation += 1
            gamma = ExtrapolationRatio * c
            gammaOld = gamma
            fgamma = func(gamma); nfe += 1
            Info.append([gamma, fgamma]); gmin, fmin = cur_min()
            fbOld, bOld = fb, b
            fb, b = fc, c
            fc, c = fgamma, gamma
            if Extrapolation > MaxExtrapolations:
                break
    if Extrapolation > 0:  # :388-405
        a, fa = bOld, fbOld
        b = (a + c) / 2
        NoSlope = True
        fb = func(b); nfe += 1
        Info.append([b, fb]); gmin, fmin = cur_min()
    fLastReduction = 1.0
    while fgamma > target or fLastReduction < ContinueRatio:  # :408
        iarm += 1
        if NoSlope:
            gamma, _ = parabolamin(a, b, c, fa, fb, fc)
            if gamma != gamma:
                raise ValueError("BackTrack:nan")
        else:
            gamma, _ = cubic_fit(slope0, fa, fb, fc, b, c)
            if gamma != gamma:
                raise ValueError("BackTrack:nan")
        if iarm == 2 and Extrapolation > 0:  # :433-470
            if gamma > b + 0.95 * (c - b):
                gamma = b + 0.95 * (c - b)
            elif gamma < a + 0.25 * (b - a):
                gamma = a + 0.25 * (b - a)
            fgamma = func(gamma); nfe += 1
            if gamma < b and fgamma < fb:
                c, fc = b, fb
                b, fb = gamma, fgamma
            elif gamma > b and fgamma < fb:
                b, fb = c, fc
                c, fc = gamma, fgamma
        else:
            if b < gamma < c:  # :479-502
                if gamma < (b + GU * (c - a)):
                    gamma = b + GU * (c - a)
                elif gamma > (c - GL * (c - b)):
                    gamma = c - GL * (c - b)
                fgamma = func(gamma); nfe += 1
                b, fb = gamma, fgamma
            else:  # :503-534
                if gamma > (a + GU * (b - a)):
                    gamma = a + GU * (b - a)
                elif gamma < (a + GL * (b - a)):
                    gamma = a + GL * (b - a)
                fgamma = func(gamma); nfe += 1
                c, fc, b, fb = b, fb, gamma, fgamma
        fminOld, gminOld = fmin, gmin
        Info.append([gamma, fgamma]); gmin, fmin = cur_min()
        fLastReduction = fmin / fminOld
        if gmin != gminOld:
            xfrac = abs(gmin - gminOld)
            MinXfrac = gmin * 1e-10
        iMinSame = iMinSame + 1 if fmin == fminOld else 0
        iMinSameWB = iMinSameWB + 1 if (gamma < gammaOld and fmin == fminOld) else 0
        gammaOld = gamma
        if not NoSlope:
            target = fa + beta * slope0 * b  # :567
            if target < 0:
                target = max(NewtonAcceptRatio * fa, p.NLtol)
        if iMinSame > MaxFuncSame and fmin < f0:
            break
        if iarm > 5 and iMinSameWB > 2 and fmin < f0:
            break
        if xfrac < MinXfrac and fmin < f0:
            break
        if b < BacktrackingGammaMin:
            break
        if iarm > MaxIterations:
            break
    if fgamma < (target - EPS):  # :626-633
        info.Converged = 1
    elif abs(fmin - fa) / fa > 1e-5 and gamma > BacktrackingGammaMin:
        info.Converged = 1
    else:
        info.Converged = 0
    Info.sort(key=lambda v: v[0])  # :646-649 (sorted copy for the record only)
    info.Infovector = Info
    info.nExtrapolationSteps = Extrapolation
    info.iarm = iarm
    info.nFuncEval = nfe
    return gmin, fmin, info


@dataclass
class LineSearchResult:
    gamma: float
    r: float
    du: np.ndarray
    dv: np.ndarray
    dl: np.ndarray
    info: BackTrackInfo
    rForce: float
    rWork: float
    D2: float
    needs_cauchy: bool = False


def rlinemin_newton(p: Params, func, r0, r1, du0, dv0, dl0):
    """rLineminUa.m:57-135: Newton-direction backtracking (the '-Auto-' first stage).

    ``func(gamma) -> (r, rForce, rWork, D2)``.  ``needs_cauchy`` reports the
    :96 condition under which the reference continues with the mass-matrix
    Cauchy step (:159-322); that continuation is not restated here.
    """
    rmin = r0
    out = LineSearchResult(0.0, r0, du0 * 0, dv0 * 0, dl0 * 0, BackTrackInfo(), r0, math.nan, math.nan)
    fN = lambda gm: func(gm)[0]
    gN, rN, info = backtracking(-2 * r0, 1.0, r0, r1, fN, p, GammaMin=0.001)  # :84-89
    out.info = info
    if gN < 0.75 and rN / r0 > 0.7:  # :94-104
        out.needs_cauchy = True
    if rN < rmin:  # :108-133
        out.du, out.dv, out.dl = gN * du0, gN * dv0, gN * dl0
        out.gamma, out.r = gN, rN
        rT, rF, rW, D2 = func(gN)
        out.rForce, out.rWork, out.D2 = rF, rW, D2
        if abs(rT - rN) > 1000 * EPS:
            raise ValueError("rLineMinUa:inconsistent")
    return out


# ---------------------------------------------------------------------------
# uv Newton driver — SSTREAM2dNR2.m:3-431 (+ uv.m:34-51)
# ---------------------------------------------------------------------------


@dataclass
class NewtonRecord:
    iteration: int
    gamma: float
    r0: float
    r: float
    rForce: float
    rWork: float
    iarm: int
    update: np.ndarray = None  # the accepted update [du; dv; (dh;) dl] (SSTREAM2dNR2.m:367-369)


@dataclass
class UvResult:
    ub: np.ndarray
    vb: np.ndarray
    lubvb: np.ndarray
    converged: bool
    iterations: int
    records: list
    K: object = None
    R: np.ndarray = None
    L: object = None
    cauchy_needed: int = 0


def prepare_fields(p: Params, F: Fields):
    """uv.m:34-51: expand scalar m,n, then Calc_bs_From_hBS."""
    F = F.copy()
    Nn = F.h.shape[0]
    for name in ("m", "n"):
        v = getattr(F, name)
        if np.isscalar(v) or np.ndim(v) == 0:
            setattr(F, name, np.zeros(Nn) + float(v))
    F.b, F.s, F.GF = calc_bs_from_hBS(p, F.h, F.S, F.B, F.rho, F.rhow)
    return F


def sstream2dnr2(p: Params, mua: MUA, bcs: BCs, F: Fields, lubvb=None, solver=None, verbose=False):
    """SSTREAM2dNR2.m:3-431 (full-Newton default, interval criterion 1).

    ``solver(K, L, frhs, grhs) -> (dx, dl)`` defaults to ABfgPreEliminate.
    """
    if solver is None:
        solver = abfg_pre_eliminate
    F = F.copy()
    Nn = mua.Nnodes
    L, cuv = create_Luv(Nn, bcs, mua)  # :32
    nc = 0 if cuv is None else cuv.shape[0]
    if lubvb is None or lubvb.shape[0] != nc:
        lubvb = np.zeros(nc)
    if np.any(np.isnan(F.C)) or np.any(np.isnan(F.AGlen)):  # :42-56
        return UvResult(F.ub + np.nan, F.vb + np.nan, lubvb, False, 0, [])
    F.ub = F.ub.copy(); F.vb = F.vb.copy()
    F.ub[bcs.ubFixedNode] = bcs.ubFixedValue  # :101-104
    F.vb[bcs.vbFixedNode] = bcs.vbFixedValue
    dub = np.zeros(Nn); dvb = np.zeros(Nn); dl = np.zeros(nc)
    fext0, _ = uv_matrix_assembly(p, mua, F, bcs, Ronly=True, ZeroFields=True)  # :122-124
    Ruv, _ = uv_matrix_assembly(p, mua, F, bcs, Ronly=True)  # :138-140

    def Func(gamma, Du, Dv, Dl):
        r, rF, rW, D2, fr, gr = calc_cost_function_nr(p, mua, gamma, F, fext0, L, lubvb, cuv, Du, Dv, Dl, bcs)
        return r, rF, rW, D2

    r, rForce, _, _ = Func(0.0, dub, dvb, dl)  # :149-150
    rWork = 0.0
    gamma = 1.0
    iteration = 0
    ResidualReduction = 1e10
    records = []
    converged = True
    Kuv = None
    cauchy = 0
    while True:
        if uv_residuals_criteria(p, rForce, rWork, iteration, gamma):  # :160-174
            converged = True
            break
        if iteration > p.NRitmax:  # :177-187
            converged = False
            break
        iteration += 1
        if (iteration - 1) % p.ModifiedNRuvIntervalCriterion == 0 or ResidualReduction > p.ModifiedNRuvReductionCriterion:
            Ruv, Kuv = uv_matrix_assembly(p, mua, F, bcs, Ronly=False)  # :200-203
        else:
            Ruv, _ = uv_matrix_assembly(p, mua, F, bcs, Ronly=True)
        if L is not None:  # :234-240
            frhs = -Ruv - L.T @ lubvb
            grhs = cuv - L @ np.concatenate([F.ub, F.vb])
        else:
            frhs = -Ruv
            grhs = np.zeros(0)
        sol, dl = solver(Kuv, L, frhs, grhs)  # :245
        dub = sol[:Nn].copy(); dvb = sol[Nn:2 * Nn].copy()
        if dl is None:
            dl = np.zeros(nc)
        r0, rForce0, rWork0, D20 = Func(0.0, dub, dvb, dl)  # :260-261
        if iteration == 1 and uv_residuals_criteria(p, rForce0, rWork0, iteration, 1.0):  # :263-283
            iteration -= 1
            converged = True
            break
        r1, rForce1, rWork1, D21 = Func(1.0, dub, dvb, dl)  # :288
        if r1 / r0 < p.NewtonAcceptRatio:  # :290-296
            r, rForce, rWork = r1, rForce1, rWork1
            du, dv, dlu = dub, dvb, dl
            gamma = 1.0
            iarm = 0
            bt_conv = 1
        else:  # :300-308
            ls = rlinemin_newton(p, lambda gm: Func(gm, dub, dvb, dl), r0, r1, dub, dvb, dl)
            gamma, r, du, dv, dlu = ls.gamma, ls.r, ls.du, ls.dv, ls.dl
            rForce, rWork = ls.rForce, ls.rWork
            iarm = ls.info.iarm
            bt_conv = ls.info.Converged
            cauchy += int(ls.needs_cauchy)
        records.append(NewtonRecord(iteration, gamma, r0, r, rForce, rWork, iarm, np.concatenate([du, dv, dlu])))
        if verbose:
            print(f"NR-SSTREAM(uv):{iteration:3d}/{iarm:<2d} g={gamma:<14.7g} r/r0={r / r0:<14.7g} "
                  f"r0={r0:<14.7g} r={r:<14.7g} rForce={rForce:<14.7g} rWork={rWork:<14.7g}")
        if bt_conv == 0:  # :322-327
            converged = False
            break
        F.ub = F.ub + du  # :367-369
        F.vb = F.vb + dv
        lubvb = lubvb + dlu
        ResidualReduction = r / r0  # :371
    return UvResult(F.ub, F.vb, lubvb, converged, iteration, records, Kuv, Ruv, L, cauchy)


def uv(p: Params, mua: MUA, bcs: BCs, F: Fields, lubvb=None, solver=None, verbose=False):
    """uv.m:34-112: prepare fields, Newton solve, one reset-and-retry on failure."""
    F = prepare_fields(p, F)
    res = sstream2dnr2(p, mua, bcs, F, lubvb, solver, verbose)
    if not res.converged:  # uv.m:107-112
        F2 = F.copy()
        F2.ub = F2.ub * 0; F2.vb = F2.vb * 0
        l0 = res.lubvb * 0 if res.lubvb is not None else None
        res = sstream2dnr2(p, mua, bcs, F2, l0, solver, verbose)
    return res


# ---------------------------------------------------------------------------
# uvh implicit transient step — uvhMatrixAssembly.m, uvhAssemblyIntPointImplicitSUPG.m,
# uvhNodalLoopSSTREAM.m, SUPGtau.m, CalcCostFunctionNRuvh.m, AssembleLuvhSSTREAM.m,
# SSTREAM_TransientImplicit.m
# ---------------------------------------------------------------------------


def tri_area_fe(coordinates, connectivity):
    """TriAreaFE.m / TriArea.m: area from the three corner nodes."""
    nod = connectivity.shape[1]
    c = connectivity if nod == 3 else connectivity[:, [0, 2, 4]]
    x = coordinates[c, 0]; y = coordinates[c, 1]
    return 0.5 * np.abs((x[:, 0] - x[:, 2]) * (y[:, 1] - y[:, 0]) - (x[:, 0] - x[:, 1]) * (y[:, 2] - y[:, 0]))


def supg_tau(p: Params, v, l, dt):
    """SUPGtau.m:7-111 for the configured option (default "taus", :61-62)."""
    taut = dt / 2 + EPS
    taus = l / (2 * v + p.SpeedZero)
    if p.uvh_SUPG_tau == "taus":
        tau = taus
    elif p.uvh_SUPG_tau == "taut":
        tau = taut + 0 * v
    elif p.uvh_SUPG_tau == "tau2":
        ECN = taut / taus
        tau = (dt / 2) / (1 + ECN)
    elif p.uvh_SUPG_tau == "tau1":
        ECN = taut / taus
        with np.errstate(divide="ignore", invalid="ignore"):
            K = 1 / np.tanh(ECN) - 1 / ECN
        K = np.where(ECN < 1e-6, ECN / 3, K)
        tau = K * taus
    else:
        raise ValueError(p.uvh_SUPG_tau)
    return p.uvh_SUPG_tauMultiplier * tau


@dataclass
class UvhState:
    """Fields of the two time levels (F0 at t, F1 at t+dt), UaFields.m subset."""
    h: np.ndarray
    ub: np.ndarray
    vb: np.ndarray
    as_: np.ndarray
    ab: np.ndarray

    def copy(self):
        return UvhState(self.h.copy(), self.ub.copy(), self.vb.copy(), self.as_.copy(), self.ab.copy())


def uvh_matrix_assembly(p: Params, mua: MUA, F: Fields, S0: UvhState, S1: UvhState, dt, Ronly=False,
                        ZeroFields=False):
    """uvhMatrixAssembly.m:6-585 (sequential; no level set, no thickness penalty or
    barrier, MassBalanceGeometryFeedback=0 so dadh=0; post-2025 Kxh/Kyh).

    F carries the time-independent fields (S, B, rho, AGlen, n, C, m, rhow, g,
    alpha).  Returns (R, K) with R = Tint-Fext (3Nn) and K the unsymmetrised CSC.
    """
    S0 = S0.copy(); S1 = S1.copy()
    if ZeroFields:  # :9-15
        S1.ub = S1.ub * 0; S1.vb = S1.vb * 0
        S0.ub = S0.ub * 0; S0.vb = S0.vb * 0
        S1.h = S0.h.copy()
        S1.as_ = np.abs(S1.ab) + 1; S1.ab = np.abs(S1.ab)
        S0.as_ = np.abs(S0.ab) + 1; S0.ab = np.abs(S0.ab)
    g = F.g; rhow = F.rhow; theta = p.theta
    ca, sa = math.cos(F.alpha), math.sin(F.alpha)
    b1, s1, _ = calc_bs_from_hBS(p, S1.h, F.S, F.B, F.rho, rhow)  # :36
    Nele, nod, Nn = mua.Nele, mua.nod, mua.Nnodes
    neq = 3 * Nn
    conn = mua.connectivity
    G = lambda v: v[conn]
    hnod, unod, vnod = G(S1.h), G(S1.ub), G(S1.vb)
    Cnod, mnod, Anod, nnod = G(F.C), G(F.m), G(F.AGlen), G(F.n)
    Snod, Bnod, rhonod, bnod = G(F.S), G(F.B), G(F.rho), G(b1)
    h0nod, u0nod, v0nod = G(S0.h), G(S0.ub), G(S0.vb)
    as0nod, ab0nod, as1nod, ab1nod = G(S0.as_), G(S0.ab), G(S1.as_), G(S1.ab)
    dadhnod = np.zeros((Nele, nod))
    if not Ronly:
        Kb = {k: np.zeros((Nele, nod, nod)) for k in ("xu", "xv", "xh", "yu", "yv", "yh", "hu", "hv", "hh")}
    Tx = np.zeros((Nele, nod)); Ty = np.zeros((Nele, nod)); Th = np.zeros((Nele, nod))
    Fx = np.zeros((Nele, nod)); Fy = np.zeros((Nele, nod)); Fh = np.zeros((Nele, nod))
    areas = tri_area_fe(mua.coordinates, conn)
    for Iint in range(mua.nip):  # :356-383 -> uvhAssemblyIntPointImplicitSUPG.m
        fun = shape_fun(nod, mua.points[Iint])
        Deriv = mua.Deriv[:, :, :, Iint]
        detJ = mua.DetJ[:, Iint]
        hint = hnod @ fun; uint = unod @ fun; vint = vnod @ fun
        Cint = Cnod @ fun; mint = mnod @ fun
        AGlenint = Anod @ fun; nint = nnod @ fun
        h0int = h0nod @ fun; u0int = u0nod @ fun; v0int = v0nod @ fun
        a1int = as1nod @ fun + ab1nod @ fun  # :64-66 (as1int+ab1int)
        a0int = as0nod @ fun + ab0nod @ fun
        dadhint = dadhnod @ fun
        h1barr = 0.0; h0barr = 0.0; lambda_h = 1.0  # :77
        Bint = Bnod @ fun; Sint = Snod @ fun; rhoint = rhonod @ fun
        Hint = Sint - Bint
        hfint = rhow * Hint / rhoint  # :106
        Heint = heaviside_approx(p.kH, hint - hfint, p.Hh0)  # :114-120
        HEint = heaviside_approx(p.kH, hfint - hint, p.Hh0)
        deltaint = dirac_delta(p.kH, hint - hfint, p.Hh0)
        Deltaint = dirac_delta(p.kH, hfint - hint, p.Hh0)
        Hposint = heaviside_approx(p.kH, Hint, p.Hh0) * Hint
        dint = HEint * rhoint * hint / rhow + Heint * Hposint
        Dddhint = HEint * rhoint / rhow - Deltaint * hint * rhoint / rhow + deltaint * Hposint
        z = lambda: np.zeros(Nele)
        dhdx, dhdy, dh0dx, dh0dy = z(), z(), z(), z()
        exx0, eyy0, exx, eyy, exy = z(), z(), z(), z(), z()
        dbdx, dbdy, drhodx, drhody = z(), z(), z(), z()
        for Inod in range(nod):  # :132-148
            Dx = Deriv[:, 0, Inod]; Dy = Deriv[:, 1, Inod]
            dhdx = dhdx + Dx * hnod[:, Inod]; dhdy = dhdy + Dy * hnod[:, Inod]
            dh0dx = dh0dx + Dx * h0nod[:, Inod]; dh0dy = dh0dy + Dy * h0nod[:, Inod]
            exx0 = exx0 + Dx * u0nod[:, Inod]; eyy0 = eyy0 + Dy * v0nod[:, Inod]
            dbdx = dbdx + Dx * bnod[:, Inod]; dbdy = dbdy + Dy * bnod[:, Inod]
            drhodx = drhodx + Dx * rhonod[:, Inod]; drhody = drhody + Dy * rhonod[:, Inod]
            exx = exx + Dx * unod[:, Inod]; eyy = eyy + Dy * vnod[:, Inod]
            exy = exy + 0.5 * (Dx * vnod[:, Inod] + Dy * unod[:, Inod])
        etaint, Eint = effective_viscosity(p, AGlenint, nint, exx, eyy, exy)  # :149
        taux, tauy, dtauxdu, dtauxdv, dtauydu, dtauydv, dtauxdh, dtauydh = basal_drag(
            p, Heint, deltaint, hint, Hint, rhoint, rhow, g, uint, vint, Cint, mint,
            **_drag_extras(p, F, conn, fun))  # :150-151
        l = np.sqrt(2 * areas)  # :156
        speed0 = np.sqrt(u0int * u0int + v0int * v0int + p.SpeedZero ** 2)  # :157
        tau0 = p.SUPG_beta0 * supg_tau(p, speed0, l, dt)  # :158-159
        detJw = detJ * mua.weights[Iint]
        # uvhNodalLoopSSTREAM.m
        qx1dx = rhoint * exx * hint + rhoint * uint * dhdx + drhodx * uint * hint  # :39
        qy1dy = rhoint * eyy * hint + rhoint * vint * dhdy + drhody * vint * hint
        qx0dx = rhoint * exx0 * h0int + rhoint * u0int * dh0dx + drhodx * u0int * h0int
        qy0dy = rhoint * eyy0 * h0int + rhoint * v0int * dh0dy + drhody * v0int * h0int
        for Inod in range(nod):
            DxI = Deriv[:, 0, Inod]; DyI = Deriv[:, 1, Inod]
            SUPG = fun[Inod] + 0.5 * tau0 * (u0int * DxI + v0int * DyI)  # :55
            funI = fun[Inod]
            if not Ronly:
                for Jnod in range(nod):
                    DxJ = Deriv[:, 0, Jnod]; DyJ = Deriv[:, 1, Jnod]; fJ = fun[Jnod]
                    Deu = Eint * ((2 * exx + eyy) * DxJ + exy * DyJ)
                    Dev = Eint * ((2 * eyy + exx) * DyJ + exy * DxJ)
                    E11 = hint * (4 * exx + 2 * eyy) * Deu * DxI + 2 * hint * exy * Deu * DyI
                    E12 = hint * (4 * exx + 2 * eyy) * Dev * DxI + 2 * hint * exy * Dev * DyI
                    E22 = hint * (4 * eyy + 2 * exx) * Dev * DyI + 2 * hint * exy * Dev * DxI
                    E21 = hint * (4 * eyy + 2 * exx) * Deu * DyI + 2 * hint * exy * Deu * DxI
                    Kb["xu"][:, Inod, Jnod] += (4 * hint * etaint * DxI * DxJ + hint * etaint * DyI * DyJ + E11
                                                + dtauxdu * fJ * funI) * detJw
                    Kb["yv"][:, Inod, Jnod] += (4 * hint * etaint * DyI * DyJ + hint * etaint * DxI * DxJ + E22
                                                + dtauydv * fJ * funI) * detJw
                    Kb["xv"][:, Inod, Jnod] += (etaint * hint * (2 * DxI * DyJ + DyI * DxJ) + E12
                                                + dtauxdv * fJ * funI) * detJw
                    Kb["yu"][:, Inod, Jnod] += (etaint * hint * (2 * DyI * DxJ + DxI * DyJ) + E21
                                                + dtauydu * fJ * funI) * detJw
                    Kb["xh"][:, Inod, Jnod] += (etaint * (4 * exx + 2 * eyy) * DxI * fJ
                                                + etaint * 2 * exy * DyI * fJ
                                                + dtauxdh * funI * fJ
                                                + ca * g * (rhoint - rhow * Dddhint) * dbdx * funI * fJ
                                                - sa * g * rhoint * funI * fJ
                                                - ca * g * (rhoint * hint - rhow * dint * Dddhint) * DxI * fJ) * detJw
                    Kb["yh"][:, Inod, Jnod] += (etaint * (4 * eyy + 2 * exx) * DyI * fJ
                                                + etaint * 2 * exy * DxI * fJ
                                                + dtauydh * funI * fJ
                                                + ca * g * (rhoint - rhow * Dddhint) * dbdy * funI * fJ
                                                - ca * g * (rhoint * hint - rhow * dint * Dddhint) * DyI * fJ) * detJw
                    Kb["hu"][:, Inod, Jnod] += theta * (rhoint * dhdx * fJ + drhodx * hint * fJ
                                                        + rhoint * hint * DxJ) * SUPG * detJw * dt
                    Kb["hv"][:, Inod, Jnod] += theta * (rhoint * dhdy * fJ + drhody * hint * fJ
                                                        + rhoint * hint * DyJ) * SUPG * detJw * dt
                    Kb["hh"][:, Inod, Jnod] += (rhoint * fJ - dt * theta * rhoint * dadhint * fJ
                                                + dt * theta * rhoint * fJ * h1barr / lambda_h
                                                + dt * theta * (rhoint * exx * fJ + drhodx * uint * fJ + rhoint * uint * DxJ
                                                                + rhoint * eyy * fJ + drhody * vint * fJ
                                                                + rhoint * vint * DyJ)) * SUPG * detJw
            t1 = -ca * g * (rhoint * hint - rhow * dint) * dbdx * funI + rhoint * g * hint * sa * funI  # :189
            t2 = 0.5 * ca * g * (rhoint * hint ** 2 - rhow * dint ** 2) * DxI
            t3 = hint * etaint * (4 * exx + 2 * eyy) * DxI
            t4 = hint * etaint * 2 * exy * DyI
            t5 = taux * funI
            Tx[:, Inod] += (t3 + t4 + t5) * detJw
            Fx[:, Inod] += (t1 + t2) * detJw
            t1 = -ca * g * (rhoint * hint - rhow * dint) * dbdy * funI
            t2 = 0.5 * ca * g * (rhoint * hint ** 2 - rhow * dint ** 2) * DyI
            t3 = hint * etaint * (4 * eyy + 2 * exx) * DyI
            t4 = hint * etaint * 2 * exy * DxI
            t5 = tauy * funI
            Ty[:, Inod] += (t3 + t4 + t5) * detJw
            Fy[:, Inod] += (t1 + t2) * detJw
            qterm = dt * (theta * qx1dx + (1 - theta) * qx0dx + theta * qy1dy + (1 - theta) * qy0dy) * SUPG  # :212
            dhdt = rhoint * (h0int - hint + dt * (1 - theta) * h0barr + dt * theta * h1barr) * SUPG
            accterm = dt * rhoint * ((1 - theta) * a0int + theta * a1int) * SUPG
            th = -dhdt
            fh = accterm - qterm
            Th[:, Inod] += th * detJw
            Fh[:, Inod] += fh * detJw
    iR = np.concatenate([np.concatenate([conn[:, I], conn[:, I] + Nn, conn[:, I] + 2 * Nn]) for I in range(nod)])
    Tval = np.concatenate([np.concatenate([Tx[:, I], Ty[:, I], Th[:, I]]) for I in range(nod)])
    Fval = np.concatenate([np.concatenate([Fx[:, I], Fy[:, I], Fh[:, I]]) for I in range(nod)])
    R = np.bincount(iR, weights=Tval, minlength=neq) - np.bincount(iR, weights=Fval, minlength=neq)  # :238
    if any(np.isnan(R)):
        raise FloatingPointError("uvhMatrixAssembly:NaNinR")
    K = None
    if not Ronly:  # :241-297
        off = {"x": 0, "y": Nn, "h": 2 * Nn}
        Ii, Jj, Xv = [], [], []
        for Inod in range(nod):
            for Jnod in range(nod):
                for key in ("xu", "xv", "xh", "yu", "yv", "yh", "hu", "hv", "hh"):
                    Ii.append(conn[:, Inod] + off[key[0]])
                    Jj.append(conn[:, Jnod] + {"u": 0, "v": Nn, "h": 2 * Nn}[key[1]])
                    Xv.append(Kb[key][:, Inod, Jnod])
        K = _matlab_sparse(np.concatenate(Ii), np.concatenate(Jj), np.concatenate(Xv), neq, neq)
    return R, K


def create_Luvh(Nnodes, bcs: BCs, mua: MUA = None):
    """AssembleLuvhSSTREAM.m:5-72 with BCs2MLC.m (Luv as create_Luv; Lh from
    createLh.m: ties, then fixed h nodes in the given order), rows scaled by ScaleL."""
    Luv, cuv = create_Luv(Nnodes, bcs, mua)
    hn = np.asarray(bcs.hFixedNode, dtype=np.int64)
    if hn.size:
        Lh = _matlab_sparse(np.arange(hn.size), hn, np.ones(hn.size), hn.size, Nnodes).tocsr()
        ch = np.asarray(bcs.hFixedValue, dtype=float)
    else:
        Lh, ch = None, None
    blocks, rhs = [], []
    if Luv is not None:
        blocks.append(sp.hstack([Luv, sp.csr_matrix((Luv.shape[0], Nnodes))]))
        rhs.append(cuv)
    if Lh is not None:
        blocks.append(sp.hstack([sp.csr_matrix((Lh.shape[0], 2 * Nnodes)), Lh]))
        rhs.append(ch)
    if not blocks:
        return None, None
    return sp.vstack(blocks).tocsr(), np.concatenate(rhs)


def calc_cost_function_nr_uvh(p, mua, F, S0, S1, dt, dub, dvb, dh, dl, L, luvh, cuvh, gamma, fext0):
    """CalcCostFunctionNRuvh.m:12-105.  Returns (r, rForce, rWork, D2)."""
    if gamma != gamma:
        raise ValueError("CalcCostFunctionNRuvh:nan")
    S1g = S1.copy()
    S1g.ub = S1.ub + gamma * dub; S1g.vb = S1.vb + gamma * dvb; S1g.h = S1.h + gamma * dh
    R, _ = uvh_matrix_assembly(p, mua, F, S0, S1g, dt, Ronly=True)
    if L is not None:
        lg = luvh + gamma * dl
        frhs = -R - L.T @ lg
        grhs = cuvh - L @ np.concatenate([S1g.ub, S1g.vb, S1g.h])
        fg = np.concatenate([frhs, grhs]); dd = np.concatenate([dub, dvb, dh, dl])
    else:
        fg = -R; dd = np.concatenate([dub, dvb, dh])
    D2 = fg @ dd
    rWork = D2 ** 2
    rForce = (fg @ fg) / (fext0 @ fext0 + 1000 * EPS)
    return rForce, rForce, rWork, D2


def uvh_criteria(p: Params, rForce, rWork, iteration, gamma):
    """SSTREAM_TransientImplicit.m:81-89."""
    if gamma > max(p.uvhExitBackTrackingStepLength, p.BacktrackingGammaMin):
        a, o = p.uvhDesiredWorkAndForceTolerances, p.uvhDesiredWorkOrForceTolerances
    else:
        a, o = p.uvhAcceptableWorkAndForceTolerances, p.uvhAcceptableWorkOrForceTolerances
    return ((rWork < a[0] and rForce < a[1]) and (rWork < o[0] or rForce < o[1]) and iteration >= p.NRitmin)


@dataclass
class UvhResult:
    ub: np.ndarray
    vb: np.ndarray
    h: np.ndarray
    luvh: np.ndarray
    converged: bool
    iterations: int
    records: list


def sstream_transient_implicit(p: Params, mua: MUA, bcs: BCs, F: Fields, S0: UvhState, S1: UvhState, dt,
                               luvh=None, verbose=False, solver=None):
    """SSTREAM_TransientImplicit.m:6-717 (uvh2D.m:20), NRitmin>=1 branch, no mass-balance
    geometry feedback, GuardAgainstWildExtrapolation off."""
    if solver is None:
        solver = abfg_pre_eliminate
    Nn = mua.Nnodes
    S1 = S1.copy()
    L, cuvh = create_Luvh(Nn, bcs, mua)  # :35
    nc = 0 if cuvh is None else cuvh.size
    luvh = np.zeros(nc) if luvh is None or len(luvh) != nc else luvh.copy()
    dl = np.zeros(nc)
    # uvhMakeInitialIterateFeasible (:37-41)
    S1.ub = S1.ub.copy(); S1.vb = S1.vb.copy(); S1.h = S1.h.copy()
    S1.ub[bcs.ubFixedNode] = bcs.ubFixedValue
    S1.vb[bcs.vbFixedNode] = bcs.vbFixedValue
    if len(bcs.hFixedNode):
        S1.h[bcs.hFixedNode] = bcs.hFixedValue
    fext0, _ = uvh_matrix_assembly(p, mua, F, S0, S1, dt, Ronly=True, ZeroFields=True)  # :53-56
    rWork = math.nan; rForce = math.inf; r = math.inf; r0 = math.inf  # :66-71
    iteration = 0
    converged = False
    bt_conv = 1
    gamma = 1.0
    rRatioVector = np.zeros(3)
    records = []
    while True:
        if rWork != rWork:
            rWork = 0.0
        if uvh_criteria(p, rForce, rWork, iteration, gamma):
            converged = True
            break
        if iteration > p.NRitmax:
            converged = False
            break
        if bt_conv == 0 or gamma == 0:  # :104-110
            converged = False
            break
        with np.errstate(invalid="ignore"):
            rRatio = r / r0
        rRatioVector[iteration % 3] = rRatio  # :111-124
        if np.all(rRatioVector > 0.98):
            converged = rWork < 1e-14
            break
        iteration += 1
        Ruvh, K = uvh_matrix_assembly(p, mua, F, S0, S1, dt)  # :127
        if L is not None:
            frhs = -Ruvh - L.T @ luvh
            grhs = cuvh - L @ np.concatenate([S1.ub, S1.vb, S1.h])
        else:
            frhs = -Ruvh; grhs = np.zeros(0)
        duvh, dl = solver(K, L, frhs, grhs)  # :136 solveKApe -> ABfgPreEliminate
        dub = duvh[:Nn].copy(); dvb = duvh[Nn:2 * Nn].copy(); dh = duvh[2 * Nn:].copy()
        if dl is None:
            dl = np.zeros(nc)
        func = lambda gm: calc_cost_function_nr_uvh(p, mua, F, S0, S1, dt, dub, dvb, dh, dl, L, luvh, cuvh, gm, fext0)
        r0 = func(0.0)[0]
        r1 = func(1.0)[0]
        ls = rlinemin_newton(p, func, r0, r1, dub, dvb, dl)  # :157 (rLineminUa)
        gamma, r = ls.gamma, ls.r
        rForce, rWork = ls.rForce, ls.rWork
        bt_conv = ls.info.Converged
        S1.ub = S1.ub + gamma * dub  # :191-194
        S1.vb = S1.vb + gamma * dvb
        S1.h = S1.h + gamma * dh
        luvh = luvh + gamma * dl
        records.append(NewtonRecord(iteration, gamma, r0, r, rForce, rWork, ls.info.iarm,
                                    np.concatenate([gamma * dub, gamma * dvb, gamma * dh, gamma * dl])))
        if verbose:
            print(f"NR-SSTREAM(uvh):{iteration:3d}/{ls.info.iarm:<2d} g={gamma:<14.7g} r/r0={r / r0:<14.7g} "
                  f"r0={r0:<14.7g} r={r:<14.7g} rForce={rForce:<14.7g} rWork={rWork:<14.7g}")
    return UvhResult(S1.ub, S1.vb, S1.h, luvh, converged, iteration, records)


# ---------------------------------------------------------------------------
# Adjoint gradient of the velocity misfit with respect to C — Misfit.m ("-uv-", adjoint branch),
# dIdCq.m, BasalDrag.m (dFuvdClambda), MassMatrix2D1dof.m, ApplyAdjointGradientPreMultiplier.m
# ---------------------------------------------------------------------------


def mass_matrix(mua: MUA):
    """MassMatrix2D1dof.m: consistent mass matrix, symmetrised as (M+M.')/2."""
    Nele, nod = mua.Nele, mua.nod
    d1d1 = np.zeros((Nele, nod, nod))
    for Iint in range(mua.nip):
        fun = shape_fun(nod, mua.points[Iint])
        detJw = mua.DetJ[:, Iint] * mua.weights[Iint]
        for I in range(nod):
            for J in range(nod):
                d1d1[:, I, J] += fun[J] * fun[I] * detJw
    conn = mua.connectivity
    Ii = np.concatenate([conn[:, I] for I in range(nod) for J in range(nod)])
    Jj = np.concatenate([conn[:, J] for I in range(nod) for J in range(nod)])
    Xv = np.concatenate([d1d1[:, I, J] for I in range(nod) for J in range(nod)])
    M = _matlab_sparse(Ii, Jj, Xv, mua.Nnodes, mua.Nnodes)
    return ((M + M.T) / 2).tocsc()


def mesh_area(mua: MUA):
    """CreateMUA.m:97-98: total area, the sum of the element areas (TriAreaFE.m)."""
    return float(np.sum(tri_area_fe(mua.coordinates, mua.connectivity)))


def misfit_uv(mua: MUA, F: Fields, us, vs, usErr, vsErr, M=None):
    """Misfit.m:38-131 with CtrlVar.Inverse.Measurements "-uv-" (ud = vd = 0 for SSTREAM):
    residuals (u - us)/uErr, I = (r_u' M r_u + r_v' M r_v)/2/Area and dI/d(u,v) = [M r_u ./ uErr;
    M r_v ./ vErr]/Area.  Returns (I, dIduv)."""
    if M is None:
        M = mass_matrix(mua)
    A = mesh_area(mua)
    ru = (F.ub - us) / usErr
    rv = (F.vb - vs) / vsErr
    duIdu = (M @ ru) / usErr / A
    dvIdv = (M @ rv) / vsErr / A
    I = float(ru @ (M @ ru) + rv @ (M @ rv)) / 2 / A
    return I, np.concatenate([duIdu, dvIdv])


def dFuvdC(p: Params, He, h, H, rho, rhow, g, u, v, C, m, q=None, muk=None, V0=None):
    """BasalDrag.m:80-160 (CtrlVar.Inverse.dFuvdClambda): the derivative of the drag magnitude over
    speed with respect to C, per sliding law.  The Coulomb law has none (the reference stops)."""
    law = p.SlidingLaw
    He = np.where(He < 0, 0.0, He)
    C0, u0 = p.Czero, p.SpeedZero
    speed = np.sqrt(u * u + v * v + u0 ** 2)
    Um = speed ** (1.0 / m - 1)
    if law in ("Weertman", "W"):
        return He * (1.0 / m) * (C + C0) ** (-1.0 / m - 1) * Um
    if law in ("Budd", "W-N0"):
        hf = rhow * H / rho
        hf = np.where(hf < EPS, 0.0, hf)
        Dh = h - hf
        Dh = np.where(Dh < EPS, 0.0, Dh)
        N = rho * g * Dh
        Nqm = N ** (q / m)
        return He * Nqm * (1.0 / m) * (C + C0) ** (-1.0 / m - 1) * Um
    if law in ("Cornford", "rpCW-N0"):
        N, _ = effective_pressure_n0(p, h, H, rho, rhow, g)
        U = speed
        return (U ** (1.0 / m - 1) * muk ** (m + 1) * N ** (m + 1) * He
                * (muk ** m * N ** m + U * (He * (C + C0) ** (-1.0 / m)) ** m) ** (-1.0 / m - 1)
                * (C + C0) ** (-1.0 / m - 1)) / m
    if law in ("Umbi", "rCW-N0"):
        N, _ = effective_pressure_n0(p, h, H, rho, rhow, g)
        U = speed
        return (U ** (1.0 / m) * muk ** 2 * N ** 2 * He / (U ** (1.0 / m) * He + muk * N * (C + C0) ** (1.0 / m)) ** 2
                * (C + C0) ** (1.0 / m - 1)) / (U * m)
    if law in ("Tsai", "minCW-N0"):
        out = He * (1.0 / m) * (C + C0) ** (-1.0 / m - 1) * Um
        N, dNdh = effective_pressure_n0(p, h, H, rho, rhow, g)
        beta2 = (C + C0) ** (-1.0 / m) * Um
        tW2 = (He * beta2 * u) ** 2 + (He * beta2 * v) ** 2
        Tau = muk * N
        tC2 = (Tau * u / speed) ** 2 + (Tau * v / speed) ** 2
        return np.where(tC2 < tW2, 0.0, out)
    if law in ("Joughin", "rCW-V0"):
        U = speed
        return (U ** (1.0 / m - 1) * He * (U + V0) ** (-1.0 / m) * (C + C0) ** (-1.0 / m - 1)) / m
    raise ValueError("BasalDrag:InvalidCase inversion for C with this sliding law is not implemented")


def dIdCq(p: Params, mua: MUA, F: Fields, uAdjoint, vAdjoint):
    """dIdCq.m:1-163 (before the logC scaling and the pre-multiplier): the nodal integral
    int dFuvdC (u uAdj + v vAdj) N_I, with He from the interpolated nodal flotation thickness."""
    conn = mua.connectivity
    G = lambda a: np.asarray(a, dtype=float)[conn]
    hnod, unod, vnod, Cnod, mnod = G(F.h), G(F.ub), G(F.vb), G(F.C), G(F.m)
    qnod = G(F.q) if (p.SlidingLaw in ("Budd", "W-N0") and F.q is not None) else mnod * 0
    muknod = G(F.muk) if F.muk is not None else mnod * 0
    V0nod = G(F.V0) if F.V0 is not None else mnod * 0
    Bnod, Snod, rhonod = G(F.B), G(F.S), G(F.rho)
    hfnod = F.rhow * (Snod - Bnod) / rhonod
    uAn, vAn = G(uAdjoint), G(vAdjoint)
    T = np.zeros((mua.Nele, mua.nod))
    for Iint in range(mua.nip):
        fun = shape_fun(mua.nod, mua.points[Iint])
        detJ = mua.DetJ[:, Iint]
        hint, uint, vint = hnod @ fun, unod @ fun, vnod @ fun
        Cint = Cnod @ fun
        Cint = np.where(Cint < p.Cmin, p.Cmin, Cint)
        mint, qint, mukint, V0int = mnod @ fun, qnod @ fun, muknod @ fun, V0nod @ fun
        Bint, Sint = Bnod @ fun, Snod @ fun
        Hint = Sint - Bint
        rhoint = rhonod @ fun
        uAi, vAi = uAn @ fun, vAn @ fun
        hfint = hfnod @ fun
        Heint = heaviside_approx(p.kH, hint - hfint, p.Hh0)
        Ctemp = dFuvdC(p, Heint, hint, Hint, rhoint, F.rhow, F.g, uint, vint, Cint, mint, qint, mukint, V0int)
        detJw = detJ * mua.weights[Iint]
        for I in range(mua.nod):
            T[:, I] += Ctemp * (uint * uAi + vint * vAi) * fun[I] * detJw
    return np.bincount(conn.ravel(order="F"), weights=T.ravel(order="F"), minlength=mua.Nnodes)


def adjoint_gradient_C(p: Params, mua: MUA, F: Fields, bcs_adjoint: BCs, us, vs, usErr, vsErr, logC=True,
                       premultiplier="M"):
    """The adjoint gradient of the "-uv-" misfit with respect to C at the solved state F
    (Misfit.m:160-260): the last Newton tangent K at (ub, vb), the adjoint system
    [K L'; L 0][lambda; mu] = [dI/duv; 0] with L of the adjoint BCs (solveKApeSymmetric),
    dIdCq at lambda, log(10) C dIdC for "logC" (dIdCq.m:153-156), and (M/Area)\\dIdC for the
    pre-multiplier "M" (ApplyAdjointGradientPreMultiplier.m).  Returns (I, dIduv, lambda, dIdC)."""
    Fp = prepare_fields(p, F)
    _, K = uv_matrix_assembly(p, mua, Fp)
    M = mass_matrix(mua)
    I, dIduv = misfit_uv(mua, Fp, us, vs, usErr, vsErr, M)
    L, c = create_Luv(mua.Nnodes, bcs_adjoint, mua)
    lam, _ = abfg_pre_eliminate(K, L, dIduv, np.zeros(0 if c is None else c.size))
    N = mua.Nnodes
    g = dIdCq(p, mua, Fp, lam[:N], lam[N:2 * N])
    if logC:
        g = math.log(10) * Fp.C * g
    if premultiplier == "M":
        g = spla.spsolve((M / mesh_area(mua)).tocsc(), g)
    return I, dIduv, lam, g


# ---------------------------------------------------------------------------
# uvh active-set thickness constraints — uvh.m:64-212, ActiveSetInitialisation.m,
# ActiveSetUpdate.m, CalculateReactions.m
# ---------------------------------------------------------------------------


@dataclass
class ActiveSetResult:
    res: UvhResult
    hPosNode: np.ndarray
    iterations: int
    cyclical: bool
    converged: bool


def _setdiff(a, b):
    """MATLAB setdiff: the sorted unique values of a that are not in b."""
    return np.setdiff1d(np.asarray(a, dtype=np.int64), np.asarray(b, dtype=np.int64))


def uvh_active_set(p: Params, mua: MUA, bcs: BCs, F: Fields, S0: UvhState, S1: UvhState, dt, hPosNode=None,
                   solver=None):
    """uvh.m:64-212: the implicit step with the active set of minimum-thickness constraints.

    hPos constraints fix h = ThickMin at their nodes (rows appended after the fixed-h rows,
    createLh.m).  After each solve, constraints whose mass-flux reaction
    ah = -Reactions.h/(rho dt) is negative are released (Reactions.h = M^-1 Lh' l.h,
    CalculateReactions.m) and nodes with h < ThickMin are activated (at most
    MaxNumberOfNewlyIntroducedActiveThicknessConstraints, the thinnest ones); the loop ends when
    the set is unchanged, cyclical, or after ThicknessConstraintsItMax iterations.
    """
    hfixed = np.asarray(bcs.hFixedNode, dtype=np.int64)
    hfixv = np.asarray(bcs.hFixedValue, dtype=float)
    tmin = p.ThickMin
    S1 = S1.copy()
    # ActiveSetInitialisation.m
    hpos = _setdiff([] if hPosNode is None else hPosNode, hfixed)
    last_active = hpos.copy()
    if np.min(S1.h) > 1.1 * tmin:
        hpos = np.zeros(0, np.int64)
    if hpos.size == 0:
        hpos = _setdiff(np.flatnonzero(S1.h < tmin), hfixed)
    deact = _setdiff(last_active, hpos)
    act = _setdiff(hpos, last_active)
    if (deact.size or act.size) and deact.size < p.MinNumberOfNewlyIntroducedActiveThicknessConstraints \
            and act.size < p.MinNumberOfNewlyIntroducedActiveThicknessConstraints:
        hpos, act, deact = last_active, np.zeros(0, np.int64), np.zeros(0, np.int64)
    last_released, last_activated = deact, act
    M = mass_matrix(mua)
    it = 1
    cyclical = False
    as_converged = True
    while True:
        S1.h = S1.h.copy()
        S1.h[hpos] = tmin
        b = BCs(ubFixedNode=bcs.ubFixedNode, ubFixedValue=bcs.ubFixedValue, vbFixedNode=bcs.vbFixedNode,
                vbFixedValue=bcs.vbFixedValue, hFixedNode=np.concatenate([hfixed, hpos]),
                hFixedValue=np.concatenate([hfixv, np.full(hpos.size, tmin)]))
        res = sstream_transient_implicit(p, mua, b, F, S0, S1, dt, solver=solver)
        if not res.converged:
            return ActiveSetResult(res, hpos, it, cyclical, False)
        S1 = UvhState(res.h.copy(), res.ub, res.vb, S1.as_, S1.ab)
        if np.any(S1.h[hpos] < tmin):
            S1.h[hpos] = tmin
        # ActiveSetUpdate.m
        hpos = _setdiff(hpos, hfixed)
        last_set = hpos.copy()
        nuv = res.luvh.size - hfixed.size - last_set.size
        lh = res.luvh[nuv:]
        if hpos.size:
            rhs = np.zeros(mua.Nnodes)
            np.add.at(rhs, np.concatenate([hfixed, last_set]), lh)  # Lh' l.h (unit rows)
            Rh = spla.spsolve(M.tocsc(), rhs)
            ah = (-Rh / (F.rho * dt))[hpos]
            isneg = ah < -0.0 * tmin / dt
            newinactive = np.flatnonzero(isneg)
            hpos = hpos[~isneg]
        else:
            newinactive = np.zeros(0, np.int64)
        released = last_set[newinactive]
        new_active = np.flatnonzero(S1.h < tmin)
        new_active = _setdiff(_setdiff(_setdiff(new_active, hfixed), hpos), released)
        if new_active.size > p.MaxNumberOfNewlyIntroducedActiveThicknessConstraints:
            order = np.argsort(S1.h, kind="stable")
            new_active = order[:p.MaxNumberOfNewlyIntroducedActiveThicknessConstraints]
        if new_active.size:
            hpos = np.concatenate([hpos, new_active])
        deact = _setdiff(last_set, hpos)
        act = _setdiff(hpos, last_set)
        cyclical = False
        if act.size or deact.size:
            if np.setxor1d(act, last_released).size == 0 and np.setxor1d(deact, last_activated).size == 0:
                cyclical = True
        if cyclical:
            hpos = np.concatenate([hpos, deact])
        if (deact.size or act.size) and deact.size < p.MinNumberOfNewlyIntroducedActiveThicknessConstraints \
                and act.size < p.MinNumberOfNewlyIntroducedActiveThicknessConstraints:
            hpos, act, deact = last_set, np.zeros(0, np.int64), np.zeros(0, np.int64)
        modified = np.setxor1d(hpos, last_set).size > 0
        last_released, last_activated = deact, act
        it += 1
        if not modified or cyclical:
            break
        if it > p.ThicknessConstraintsItMax:
            as_converged = False
            break
    res = UvhResult(S1.ub, S1.vb, S1.h, res.luvh, res.converged, res.iterations, res.records)
    return ActiveSetResult(res, hpos, it - 1, cyclical, as_converged)
