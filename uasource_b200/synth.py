"""Seeded synthetic SSA problems (meshes, fields, boundary conditions).

The reference publishes no benchmark meshes for this path, so the workloads
are synthetic, generated here with fixed seeds:

* ``ice_stream_shelf`` — the rectangular ice stream / shelf of the
  diagnostic-solve workload: bed ``B=-200-0.006x``, thickness
  ``h=1200-0.009x`` plus five seeded +-50 m Gaussian bumps (sigma 3 km),
  ``S=0``, rho=917, rhow=1030, g=9.81e-3 (Úa's kPa/m/a units,
  ``DefineGeometryAndDensities.m``), Glen ``A=1e-8 exp(0.3 z)`` and Weertman
  ``C=1e-2 exp(0.5 z)`` with z an i.i.d. nodal N(0,1) field smoothed over
  5 km and rescaled to unit variance, ``n=m=3``; u=v=0 on x=0, v=0 on the
  lateral sides (free slip), ocean-pressure calving front at x=xmax.
  Larger domains evaluate the same fields at coordinates scaled back onto the
  100 km x 50 km reference rectangle.

Triangles use Úa's node order: P1 nodes are ordered so that the Jacobian of
the map from the reference triangle (shape_fun.m: N=[xi, 1-xi-eta, eta]) is
positive; P2 elements list corners at local positions 1,3,5 and edge
mid-points at 2,4,6 (tri3to6.m:22-47).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Problem:
    """Host arrays of one SSA problem (0-based connectivity)."""
    coordinates: np.ndarray      # Nnodes x 2 (float64)
    connectivity: np.ndarray     # Nele x nod (int32)
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
    ubFixedNode: np.ndarray
    ubFixedValue: np.ndarray
    vbFixedNode: np.ndarray
    vbFixedValue: np.ndarray
    rhow: float = 1030.0
    g: float = 9.81 / 1000
    alpha: float = 0.0
    # transient (uvh) extras
    as_: np.ndarray = None
    ab: np.ndarray = None
    h0: np.ndarray = None
    u0: np.ndarray = None
    v0: np.ndarray = None
    hFixedNode: np.ndarray = None
    hFixedValue: np.ndarray = None
    name: str = ""

    @property
    def Nnodes(self):
        return self.coordinates.shape[0]

    @property
    def Nele(self):
        return self.connectivity.shape[0]

    @property
    def nod(self):
        return self.connectivity.shape[1]


def rect_mesh(Lx: float, Ly: float, nx: int, ny: int, nod: int = 3):
    """Structured triangulation of [0,Lx]x[0,Ly] with nx x ny vertices.

    Cells are split along alternating diagonals.  Vertices are numbered with
    y fastest (column-major in x), which keeps the matrix bandwidth at ~ny.
    Returns (coordinates, connectivity) in Úa orientation.
    """
    xs = np.linspace(0.0, Lx, nx)
    ys = np.linspace(0.0, Ly, ny)
    X, Y = np.meshgrid(xs, ys, indexing="ij")           # [nx, ny]
    coords = np.stack([X.ravel(), Y.ravel()], axis=1)
    vid = np.arange(nx * ny).reshape(nx, ny)
    i, j = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), indexing="ij")
    i = i.ravel(); j = j.ravel()
    v00 = vid[i, j]; v10 = vid[i + 1, j]; v01 = vid[i, j + 1]; v11 = vid[i + 1, j + 1]
    alt = ((i + j) % 2) == 0
    # counter-clockwise triangles per cell
    t1 = np.where(alt[:, None], np.stack([v00, v10, v11], 1), np.stack([v00, v10, v01], 1))
    t2 = np.where(alt[:, None], np.stack([v00, v11, v01], 1), np.stack([v10, v11, v01], 1))
    tri = np.empty((2 * len(i), 3), dtype=np.int64)
    tri[0::2] = t1
    tri[1::2] = t2
    # Úa's P1 order (N1 at xi=1, N2 at origin, N3 at eta=1) has positive
    # Jacobian for clockwise triangles: reverse the counter-clockwise ones.
    tri = tri[:, [0, 2, 1]]
    if nod == 3:
        return coords, tri.astype(np.int32)
    if nod == 6:
        return tri3to6(coords, tri)
    raise ValueError("nod must be 3 or 6")


def tri3to6(coords, tri):
    """Add one mid-node per unique edge; corners at 1,3,5 and mids at 2,4,6."""
    Nn = coords.shape[0]
    edges = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    ekey = np.sort(edges, axis=1)
    uniq, inv = np.unique(ekey[:, 0] * np.int64(Nn) + ekey[:, 1], return_inverse=True)
    a = uniq // Nn
    b = uniq % Nn
    mid = 0.5 * (coords[a] + coords[b])
    coords6 = np.concatenate([coords, mid])
    Ne = tri.shape[0]
    m01 = Nn + inv[:Ne]; m12 = Nn + inv[Ne:2 * Ne]; m20 = Nn + inv[2 * Ne:]
    conn6 = np.stack([tri[:, 0], m01, tri[:, 1], m12, tri[:, 2], m20], axis=1)
    # renumber nodes by x then y so mid-nodes sit next to their corners
    order = np.lexsort((coords6[:, 1], coords6[:, 0]))
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    return coords6[order], rank[conn6].astype(np.int32)


def _smooth_normal(rng, coords, Lx, Ly, sigma, ngrid=(141, 71)):
    """i.i.d. N(0,1) on a regular grid, Gaussian-smoothed (sigma in m), unit variance,
    bilinearly sampled at the given (reference-domain) coordinates."""
    from scipy.ndimage import gaussian_filter
    gx, gy = ngrid
    z = rng.standard_normal((gx, gy))
    dx = Lx / (gx - 1); dy = Ly / (gy - 1)
    z = gaussian_filter(z, sigma=(sigma / dx, sigma / dy), mode="nearest")
    z = (z - z.mean()) / z.std()
    fx = np.clip(coords[:, 0] / dx, 0, gx - 1 - 1e-12)
    fy = np.clip(coords[:, 1] / dy, 0, gy - 1 - 1e-12)
    i0 = np.floor(fx).astype(int); j0 = np.floor(fy).astype(int)
    tx = fx - i0; ty = fy - j0
    return ((1 - tx) * (1 - ty) * z[i0, j0] + tx * (1 - ty) * z[i0 + 1, j0]
            + (1 - tx) * ty * z[i0, j0 + 1] + tx * ty * z[i0 + 1, j0 + 1])


def ice_stream_shelf(nx=141, ny=71, Lx=100e3, Ly=50e3, nod=3, seed=0, transient=False):
    """Ice stream flowing into a floating shelf; see the module docstring."""
    rng = np.random.Generator(np.random.PCG64(seed))
    coords, conn = rect_mesh(Lx, Ly, nx, ny, nod)
    # evaluate fields on the 100 km x 50 km reference rectangle
    sx, sy = 100e3 / Lx, 50e3 / Ly
    ref = coords * np.array([sx, sy])
    x = ref[:, 0]; y = ref[:, 1]
    Nn = coords.shape[0]
    B = -200.0 - 0.006 * x
    h = 1200.0 - 0.009 * x
    cx = rng.uniform(10e3, 90e3, 5)
    cy = rng.uniform(5e3, 45e3, 5)
    sgn = rng.choice([-1.0, 1.0], 5)
    for k in range(5):
        r2 = (x - cx[k]) ** 2 + (y - cy[k]) ** 2
        h = h + sgn[k] * 50.0 * np.exp(-r2 / (2 * 3000.0 ** 2))
    zA = _smooth_normal(rng, ref, 100e3, 50e3, 5e3)
    zC = _smooth_normal(rng, ref, 100e3, 50e3, 5e3)
    AGlen = 1e-8 * np.exp(0.3 * zA)
    C = 1e-2 * np.exp(0.5 * zC)
    tol = 1e-6 * max(Lx, Ly)
    left = np.flatnonzero(coords[:, 0] < tol)
    bottom = np.flatnonzero(coords[:, 1] < tol)
    top = np.flatnonzero(coords[:, 1] > Ly - tol)
    vfix = np.unique(np.concatenate([left, bottom, top]))
    prob = Problem(
        coordinates=coords, connectivity=conn,
        h=h, S=np.zeros(Nn), B=B, rho=np.full(Nn, 917.0),
        AGlen=AGlen, n=np.full(Nn, 3.0), C=C, m=np.full(Nn, 3.0),
        ub=np.zeros(Nn), vb=np.zeros(Nn),
        ubFixedNode=left.astype(np.int32), ubFixedValue=np.zeros(left.size),
        vbFixedNode=vfix.astype(np.int32), vbFixedValue=np.zeros(vfix.size),
        name=f"ice_stream_shelf_{'P1' if nod == 3 else 'P2'}_{nx}x{ny}_seed{seed}")
    if transient:
        zA2 = rng.standard_normal(Nn)
        prob.as_ = 0.3 + 0.1 * zA2
        prob.ab = np.zeros(Nn)
        prob.h0 = prob.h.copy()
        prob.u0 = np.zeros(Nn)
        prob.v0 = np.zeros(Nn)
        prob.hFixedNode = np.zeros(0, np.int32)
        prob.hFixedValue = np.zeros(0)
    return prob


def elements_to_grid(nele_target: int, aspect: float = 2.0):
    """Vertex grid (nx, ny) of a 2:1 rectangle with about ``nele_target`` P1 triangles."""
    # Nele = 2 (nx-1)(ny-1), nx-1 = aspect (ny-1)
    ny1 = max(1, int(round(math.sqrt(nele_target / (2.0 * aspect)))))
    nx1 = max(1, int(round(aspect * ny1)))
    return nx1 + 1, ny1 + 1


def batch_sizes(count=256, lo=2e3, hi=2e5, seed=12345):
    """Element counts of the batched workload: log-uniform in [lo, hi] (seeded)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.exp(rng.uniform(np.log(lo), np.log(hi), count))


def batch_problem(k, count=256, lo=2e3, hi=2e5, seed=12345):
    """Problem k of the batched workload (see ``batch_problems``)."""
    ne = batch_sizes(count, lo, hi, seed)[k]
    nx, ny = elements_to_grid(int(ne), aspect=2.0)
    return ice_stream_shelf(nx, ny, nod=3, seed=1000 + k)


def batch_problems(count=256, lo=2e3, hi=2e5, seed=12345):
    """256 independent ice-stream/shelf problems on 100 km x 50 km rectangles of
    log-uniform size (P1), each with its own seed for bumps, A and C."""
    return [batch_problem(k, count, lo, hi, seed) for k in range(count)]


def serve_templates(count=16, lo=5e3, hi=5e5, seed=777):
    """Resident mesh templates of the served workload: ``count`` ice-stream/shelf
    problems (P1) of log-uniform size in [lo, hi] elements, each with its own seed."""
    out = []
    for k, ne in enumerate(batch_sizes(count, lo, hi, seed)):
        nx, ny = elements_to_grid(int(ne), aspect=2.0)
        out.append(ice_stream_shelf(nx, ny, nod=3, seed=5000 + k))
    return out
