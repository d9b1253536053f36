"""Restart files into host problems (WriteForwardRunRestartFile.m:25 layout, MAT v7 with F and l
as structs): a synthetic problem written and read back is the same problem, 1-based lists come
back 0-based, and malformed files are refused with a message naming the field."""
import numpy as np
import pytest
import scipy.io as sio

from uasource_b200 import synth
from uasource_b200.restart import load_restart, save_restart


def _same(P, Q):
    for k in ("coordinates", "h", "S", "B", "rho", "AGlen", "n", "C", "m", "ub", "vb", "ubFixedValue",
              "vbFixedValue"):
        assert np.array_equal(np.asarray(getattr(P, k), dtype=np.float64), getattr(Q, k)), k
    assert np.array_equal(P.connectivity, Q.connectivity) and Q.connectivity.dtype == np.int32
    assert np.array_equal(P.ubFixedNode, Q.ubFixedNode) and np.array_equal(P.vbFixedNode, Q.vbFixedNode)
    assert (P.rhow, P.g, P.alpha) == (Q.rhow, Q.g, Q.alpha)


@pytest.mark.parametrize("nod,transient", [(3, False), (6, True)], ids=["P1", "P2-transient"])
def test_round_trip(tmp_path, nod, transient):
    P = synth.ice_stream_shelf(15, 8, nod=nod, seed=3, transient=transient)
    rng = np.random.default_rng(0)
    P.ub = rng.random(P.Nnodes)
    P.vb = rng.random(P.Nnodes)
    lam = rng.standard_normal(7)
    f = tmp_path / "restart.mat"
    save_restart(f, P, lam, time=12.5, dt=0.1)
    r = load_restart(f)
    _same(P, r.problem)
    if transient:
        assert np.array_equal(P.as_, r.problem.as_) and np.array_equal(P.ab, r.problem.ab)
    assert np.array_equal(r.lubvb, lam) and r.time == 12.5 and r.dt == 0.1
    # on disk the lists are 1-based, as Ua writes them
    raw = sio.loadmat(f, squeeze_me=True, struct_as_record=False)
    assert raw["MUA"].connectivity.min() == 1
    assert np.array_equal(np.atleast_1d(raw["BCs"].ubFixedNode), P.ubFixedNode + 1)


def test_scalar_field_is_expanded(tmp_path):
    P = synth.ice_stream_shelf(9, 6, seed=1)
    f = tmp_path / "r.mat"
    save_restart(f, P)
    d = sio.loadmat(f)
    d["F"] = {**{k: d["F"][k][0, 0] for k in d["F"].dtype.names}, "n": 3.0}
    sio.savemat(f, {k: v for k, v in d.items() if not k.startswith("__")})
    assert np.array_equal(load_restart(f).problem.n, np.full(P.Nnodes, 3.0))


def test_malformed_files_are_refused(tmp_path):
    P = synth.ice_stream_shelf(9, 6, seed=1)
    f = tmp_path / "bad.mat"
    save_restart(f, P)
    d = {k: v for k, v in sio.loadmat(f).items() if not k.startswith("__")}
    bad = dict(d)
    bad["MUA"] = {"coordinates": d["MUA"]["coordinates"][0, 0], "connectivity": d["MUA"]["connectivity"][0, 0] - 1}
    sio.savemat(f, bad)
    with pytest.raises(ValueError, match="1-based"):
        load_restart(f)
    bad = dict(d)
    bad["F"] = {k: d["F"][k][0, 0] for k in d["F"].dtype.names if k != "AGlen"}
    sio.savemat(f, bad)
    with pytest.raises(ValueError, match="F.AGlen"):
        load_restart(f)
    # a MAT v7.3 (HDF5) header: the file has to go through mex/UaRestartToV7.m first
    g = tmp_path / "v73.mat"
    hdr = b"MATLAB 7.3 MAT-file, Platform: GLNXA64".ljust(116, b" ") + b"\0" * 8 + b"\x00\x02IM"
    g.write_bytes(hdr + b"\0" * 512)
    with pytest.raises(ValueError, match="v7.3"):
        load_restart(g)
