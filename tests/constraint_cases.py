"""Tied-node and fixed-normal-velocity constraints on the ice-stream/shelf problem (CreateLuv.m).

ties: u at the y = 0 nodes tied to u at the y = Ly nodes with the same x (u is free there: it is
fixed only at x = 0, whose nodes are left out), so the lateral sides are periodic in u.
normal: the interior calving-front nodes (x = Lx, not on y = 0 or y = Ly, where v is fixed) get
Nx u + Ny v = -value with the boundary's nodal normals.
"""
import numpy as np

from uasource_b200 import synth


def problem(nx=21, ny=11, nod=3, angle=0.0):
    """The synthetic problem with its mesh rotated by `angle` (radians) about the origin: the
    nodal fields stay, so the flow is the same problem turned, and the boundary normals mix the
    u and v components."""
    P = synth.ice_stream_shelf(nx, ny, nod=nod, seed=0)
    if angle:
        c, s = np.cos(angle), np.sin(angle)
        x, y = P.coordinates[:, 0].copy(), P.coordinates[:, 1].copy()
        P.coordinates = np.stack([c * x - s * y, s * x + c * y], axis=1)
        P.unrotated = np.stack([x, y], axis=1)
    return P


def _xy(P):
    c = getattr(P, "unrotated", P.coordinates)
    return c[:, 0], c[:, 1]


def tie_nodes(P):
    x, y = _xy(P)
    tol = 1e-6 * (x.max() - x.min())
    bottom = np.flatnonzero((np.abs(y - y.min()) < tol) & (x > x.min() + tol))
    top = np.flatnonzero((np.abs(y - y.max()) < tol) & (x > x.min() + tol))
    bottom = bottom[np.argsort(x[bottom])]
    top = top[np.argsort(x[top])]
    assert np.allclose(x[bottom], x[top])
    return bottom.astype(np.int64), top.astype(np.int64)


def front_nodes(P):
    x, y = _xy(P)
    tol = 1e-6 * (x.max() - x.min())
    f = np.flatnonzero((np.abs(x - x.max()) < tol) & (y > y.min() + tol) & (y < y.max() - tol))
    return f[np.argsort(y[f])].astype(np.int64)
