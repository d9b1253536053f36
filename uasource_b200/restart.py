"""Restart files into resident handles: the MUA, BCs, F and l of an Úa forward-run restart file
(WriteForwardRunRestartFile.m:25 saves CtrlVarInRestartFile, UserVarInRestartFile, MUA, BCs, F,
GF, l, RunInfo) read into the host objects the solvers and the serving loop take.

Úa writes restart files as MAT v7.3 (HDF5), where F (UaFields) and RunInfo (UaRunInfo) are
MATLAB classdef objects stored as opaque MCOS references that only MATLAB can decode.  The
bridge is therefore a MAT v5/v7 file with the same variable names in which F and l are plain
structs: ``mex/UaRestartToV7.m`` writes one from a restart file inside MATLAB, and
:func:`save_restart` writes one from Python (for tests, and to hand meshes between runs).
:func:`load_restart` reads either into a :class:`~uasource_b200.synth.Problem` (0-based
connectivity and BC node lists), with the warm start F.ub, F.vb and the multipliers l.ubvb.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .synth import Problem

# the F fields the uv and uvh paths read (UaFields.m names; "as" is a Python keyword: as_)
_F_NODAL = ("h", "S", "B", "rho", "AGlen", "n", "C", "m", "ub", "vb", "as", "ab")
_BC_LISTS = (("ubFixedNode", "ubFixedValue"), ("vbFixedNode", "vbFixedValue"), ("hFixedNode", "hFixedValue"))


@dataclass
class Restart:
    problem: Problem          # mesh, fields, fixed-node BCs, warm start (ub, vb)
    lubvb: np.ndarray         # l.ubvb (may be empty)
    time: float = 0.0         # CtrlVarInRestartFile.time, if present
    dt: float = 0.0           # CtrlVarInRestartFile.dt, if present


def _get(s, name, default=None):
    if s is None:
        return default
    if isinstance(s, dict):
        return s.get(name, default)
    return getattr(s, name, default)


def _vec(v, n=None, name=""):
    a = np.atleast_1d(np.asarray(v, dtype=np.float64)).ravel(order="F")
    if n is not None and a.size == 1 and n > 1:
        a = np.full(n, a[0])  # a scalar field (F.n = 3) as a nodal vector
    if n is not None and a.size != n:
        raise ValueError(f"restart: F.{name} has {a.size} entries for {n} nodes")
    return a


def _nodes(v):
    if v is None:
        return np.zeros(0, np.int32)
    a = np.atleast_1d(np.asarray(v, dtype=np.float64)).ravel(order="F")
    if a.size and (np.any(a != np.round(a)) or a.min() < 1):
        raise ValueError("restart: node lists are 1-based integers")
    return (a.astype(np.int64) - 1).astype(np.int32)


def load_restart(path) -> Restart:
    """Reads a MAT v5/v7 restart file (variables MUA, BCs, F, l and optionally
    CtrlVarInRestartFile) into a Restart.  MUA.connectivity and the BC node lists are 1-based
    in the file, as Úa writes them."""
    import scipy.io as sio
    try:
        d = sio.loadmat(path, squeeze_me=True, struct_as_record=False)
    except NotImplementedError as e:  # scipy refuses MAT v7.3 (HDF5)
        raise ValueError(f"{path} is a MAT v7.3 file: convert it with mex/UaRestartToV7.m inside MATLAB") from e
    for v in ("MUA", "F"):
        if v not in d:
            raise ValueError(f"restart: {path} has no variable {v}")
    MUA, F, BCs, l = d["MUA"], d["F"], d.get("BCs"), d.get("l")
    coords = np.asarray(_get(MUA, "coordinates"), dtype=np.float64)
    conn = np.asarray(_get(MUA, "connectivity"), dtype=np.float64)
    if coords.ndim != 2 or coords.shape[1] != 2 or conn.ndim != 2 or conn.shape[1] not in (3, 6):
        raise ValueError("restart: MUA.coordinates must be Nnodes x 2, MUA.connectivity Nele x 3 or x 6")
    if np.any(conn != np.round(conn)) or conn.min() < 1 or conn.max() > coords.shape[0]:
        raise ValueError("restart: MUA.connectivity must hold 1-based node numbers")
    nn = coords.shape[0]
    f = {k: (None if _get(F, k) is None else _vec(_get(F, k), nn, k)) for k in _F_NODAL}
    for k in ("h", "S", "B", "rho", "AGlen", "n", "C", "m"):
        if f[k] is None:
            raise ValueError(f"restart: F.{k} is missing")
    bc = {}
    for node, val in _BC_LISTS:
        nodes = _nodes(_get(BCs, node))
        vals = _get(BCs, val)
        vals = np.zeros(nodes.size) if vals is None else _vec(vals, None, val)
        if vals.size != nodes.size:
            raise ValueError(f"restart: BCs.{val} has {vals.size} entries for {nodes.size} nodes")
        bc[node], bc[val] = nodes, vals
    P = Problem(coordinates=np.ascontiguousarray(coords), connectivity=(conn.astype(np.int64) - 1).astype(np.int32),
                h=f["h"], S=f["S"], B=f["B"], rho=f["rho"], AGlen=f["AGlen"], n=f["n"], C=f["C"], m=f["m"],
                ub=np.zeros(nn) if f["ub"] is None else f["ub"], vb=np.zeros(nn) if f["vb"] is None else f["vb"],
                ubFixedNode=bc["ubFixedNode"], ubFixedValue=bc["ubFixedValue"],
                vbFixedNode=bc["vbFixedNode"], vbFixedValue=bc["vbFixedValue"],
                rhow=float(_get(F, "rhow", 1030.0)), g=float(_get(F, "g", 9.81 / 1000)),
                alpha=float(_get(F, "alpha", 0.0)), as_=f["as"], ab=f["ab"],
                hFixedNode=bc["hFixedNode"] if bc["hFixedNode"].size else None,
                hFixedValue=bc["hFixedValue"] if bc["hFixedNode"].size else None, name=str(path))
    lubvb = np.zeros(0) if _get(l, "ubvb") is None else _vec(_get(l, "ubvb"))
    C = d.get("CtrlVarInRestartFile")
    return Restart(P, lubvb, float(_get(C, "time", 0.0)), float(_get(C, "dt", 0.0)))


def save_restart(path, P: Problem, lubvb=None, time=0.0, dt=0.0):
    """Writes P (and l.ubvb) in the restart layout as a MAT v5 file (1-based connectivity and
    BC node lists, F and l as structs)."""
    import scipy.io as sio
    col = lambda a: np.asarray(a, dtype=np.float64).reshape(-1, 1)  # noqa: E731
    F = {k: col(getattr(P, k)) for k in ("h", "S", "B", "rho", "AGlen", "n", "C", "m", "ub", "vb")}
    if P.as_ is not None:
        F["as"] = col(P.as_)
    if P.ab is not None:
        F["ab"] = col(P.ab)
    F.update(rhow=float(P.rhow), g=float(P.g), alpha=float(P.alpha))
    B = {"ubFixedNode": col(np.asarray(P.ubFixedNode) + 1), "ubFixedValue": col(P.ubFixedValue),
         "vbFixedNode": col(np.asarray(P.vbFixedNode) + 1), "vbFixedValue": col(P.vbFixedValue)}
    if P.hFixedNode is not None and len(P.hFixedNode):
        B.update(hFixedNode=col(np.asarray(P.hFixedNode) + 1), hFixedValue=col(P.hFixedValue))
    sio.savemat(path, {"MUA": {"coordinates": np.asarray(P.coordinates, dtype=np.float64),
                               "connectivity": np.asarray(P.connectivity, dtype=np.float64) + 1},
                       "BCs": B, "F": F, "l": {"ubvb": col(np.zeros(0) if lubvb is None else lubvb)},
                       "CtrlVarInRestartFile": {"time": float(time), "dt": float(dt)}},
                do_compression=True)
