"""Known-answer problems from the reference's own analytic solutions.

* ``ice_shelf_problem`` — UaUtilities/AnalyticalOneDimentionalIceShelf.m:36-63:
  steady floating shelf, Glen n=3, accumulation a; thickness h(x) given, the
  velocity u(x) = (a x + q_gl)/h(x) is the answer.
* ``ice_stream_problem`` — UaMain/Simple1dIceStreamSolution.m:5-78: grounded
  slab of uniform thickness on a bed sloping at alpha, n=m=1;
  u(x) = C tau + K sinh(kappa x)/(kappa cosh(kappa L)).

Both are 1-D, posed on a 2-D strip with v=0 on the lateral sides.  These
builders are shared by the CPU oracle tests and the GPU tests.
"""
import numpy as np

from uasource_b200 import synth


def _strip(L, W, nx, ny, nod):
    coords, conn = synth.rect_mesh(L, W, nx, ny, nod)
    tol = 1e-9 * L
    left = np.flatnonzero(coords[:, 0] < tol)
    sides = np.flatnonzero((coords[:, 1] < tol) | (coords[:, 1] > W - tol))
    return coords, conn, left, np.unique(np.concatenate([left, sides]))


def ice_shelf_problem(nx=81, ny=5, nod=3, L=100e3, W=10e3, A=2e-10):
    """Floating shelf: AnalyticalOneDimentionalIceShelf.m defaults (a=0.3, n=3,
    rho=910, rhow=1030, g=9.81e-3, hgl=1000, ugl=300); A defaults to 2e-10 so that
    the thinning near the grounding line is resolved by coarse test meshes."""
    a, n, rho, rhow, g, A, hgl, ugl = 0.3, 3.0, 910.0, 1030.0, 9.81 / 1000, A, 1000.0, 300.0
    coords, conn, left, vfix = _strip(L, W, nx, ny, nod)
    x = coords[:, 0]
    qgl = hgl * ugl
    gamm = A * (rho * (1 - rho / rhow) * g) ** n / 4 ** n
    K = qgl ** (n + 1) * (a / hgl ** (n + 1) - gamm)
    h = ((gamm + K / (qgl + a * x) ** (n + 1)) / a) ** (-1.0 / (n + 1))
    u_exact = (a * x + qgl) / h
    Nn = coords.shape[0]
    prob = dict(coordinates=coords, connectivity=conn, h=h, S=np.zeros(Nn), B=np.full(Nn, -5000.0),
                rho=np.full(Nn, rho), AGlen=np.full(Nn, A), n=np.full(Nn, n), C=np.full(Nn, 1.0),
                m=np.full(Nn, 3.0), ub=np.zeros(Nn), vb=np.zeros(Nn), rhow=rhow, g=g,
                ubFixedNode=left, ubFixedValue=np.full(left.size, ugl),
                vbFixedNode=vfix, vbFixedValue=np.zeros(vfix.size))
    return prob, u_exact


def ice_stream_problem(nx=101, ny=5, nod=3, L=25e3, W=5e3):
    """Grounded stream: Simple1dIceStreamSolution.m:5-20 defaults (n=m=1, h=1000,
    alpha=0.001, rho=900, rhow=1000, ud=0.1, SlipRatio=10)."""
    h0, alpha, g, rho, rhow = 1000.0, 0.001, 9.81 / 1000, 900.0, 1000.0
    ud, slip = 0.1, 10.0
    tau = rho * g * h0 * alpha
    A = ud / (2 * tau * h0 / 2)
    C = slip * ud / tau
    coords, conn, left, vfix = _strip(L, W, nx, ny, nod)
    x = coords[:, 0]
    Nn = coords.shape[0]
    B = -np.tan(alpha) * x
    dl = np.tan(alpha) * L                       # draft at the front (S=0, B(0)=0)
    kappa = np.sqrt(A / (2 * h0 * C))
    K = A * (g * (rho * h0 ** 2 - rhow * dl ** 2) / 4 / h0)
    u_exact = C * tau + K * np.sinh(kappa * x) / (kappa * np.cosh(kappa * L))
    prob = dict(coordinates=coords, connectivity=conn, h=np.full(Nn, h0), S=np.zeros(Nn), B=B,
                rho=np.full(Nn, rho), AGlen=np.full(Nn, A), n=np.full(Nn, 1.0), C=np.full(Nn, C),
                m=np.full(Nn, 1.0), ub=np.zeros(Nn), vb=np.zeros(Nn), rhow=rhow, g=g,
                ubFixedNode=left, ubFixedValue=np.full(left.size, C * tau),
                vbFixedNode=vfix, vbFixedValue=np.zeros(vfix.size))
    return prob, u_exact
