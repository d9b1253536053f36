"""Implicit-step cases for the minimum-thickness active set (uvh.m:64-212): a thin,
strongly ablating grounded patch that drives the thickness below ThickMin, and the same
with a seeded active set whose thick nodes must be released."""
import numpy as np

from uasource_b200 import synth


def thin_patch_problem(nod=3, nx=21, ny=11):
    """(problem, start thickness, surface mass balance): 4 m of ice with as = -40 m/a on an
    8 km disc of the grounded part, so dt = 0.1 a would take it below ThickMin = 1 m."""
    P = synth.ice_stream_shelf(nx, ny, nod=nod, seed=0, transient=True)
    x, y = P.coordinates[:, 0], P.coordinates[:, 1]
    thin = (x - 30e3) ** 2 + (y - 25e3) ** 2 < 8e3 ** 2
    h = P.h.copy()
    h[thin] = 4.0
    as_ = P.as_.copy()
    as_[thin] = -40.0
    return P, h, as_


SEED_NODES = np.array([71, 100, 150, 160])
SEED_THIN_NODE = 100  # set to 1.05 m so that min(h) <= 1.1 ThickMin keeps the seeded set
