"""The oracle reproduces the committed golden fixtures (no GPU)."""
import glob
import os

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ua_ref as R

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "uv_*.npz")))


def load_case(path):
    z = np.load(path)
    mua = R.create_mua(z["coordinates"], z["connectivity"])
    F = R.Fields(h=z["h"], S=z["S"], B=z["B"], rho=z["rho"], AGlen=z["AGlen"], n=z["n"], C=z["C"], m=z["m"],
                 ub=np.zeros(mua.Nnodes), vb=np.zeros(mua.Nnodes), rhow=float(z["rhow"]), g=float(z["g"]))
    bcs = R.BCs(ubFixedNode=z["ubFixedNode"], ubFixedValue=z["ubFixedValue"], vbFixedNode=z["vbFixedNode"],
                vbFixedValue=z["vbFixedValue"])
    return z, mua, F, bcs


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_reproduces_fixture(path):
    z, mua, F, bcs = load_case(path)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    Fs = R.prepare_fields(p, F)
    Fs.ub, Fs.vb = z["state_ub"], z["state_vb"]
    Rv, K = R.uv_matrix_assembly(p, mua, Fs)
    Kz = sp.coo_matrix((z["K_val"], (z["K_row"], z["K_col"])), shape=K.shape).tocsc()
    assert abs(K - Kz).max() <= 1e-13 * abs(Kz).max()
    assert np.max(np.abs(Rv - z["R"])) <= 1e-13 * np.max(np.abs(z["R"]))
    res = R.uv(p, mua, bcs, F)
    assert res.converged
    u_ref = np.concatenate([z["sol_ub"], z["sol_vb"]])
    u = np.concatenate([res.ub, res.vb])
    assert np.linalg.norm(u - u_ref) <= 1e-10 * np.linalg.norm(u_ref)


UVH_FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "uvh_*.npz")))


@pytest.mark.parametrize("path", UVH_FIXTURES, ids=[os.path.basename(p) for p in UVH_FIXTURES])
def test_oracle_reproduces_uvh_fixture(path):
    z = np.load(path)
    mua = R.create_mua(z["coordinates"], z["connectivity"])
    F = R.Fields(h=z["h0"], S=z["S"], B=z["B"], rho=z["rho"], AGlen=z["AGlen"], n=z["n"], C=z["C"], m=z["m"],
                 ub=z["u0"], vb=z["v0"], rhow=float(z["rhow"]), g=float(z["g"]))
    S0 = R.UvhState(z["h0"], z["u0"], z["v0"], z["as_"], z["ab"])
    S1 = R.UvhState(z["state_h"], z["state_ub"], z["state_vb"], z["as_"], z["ab"])
    p = R.Params()
    Rv, K = R.uvh_matrix_assembly(p, mua, F, S0, S1, float(z["dt"]))
    Kz = sp.coo_matrix((z["K_val"], (z["K_row"], z["K_col"])), shape=K.shape).tocsc()
    assert abs(K - Kz).max() <= 1e-13 * abs(Kz).max()
    assert np.max(np.abs(Rv - z["R"])) <= 1e-13 * np.max(np.abs(z["R"]))
