"""Generate the golden fixtures for the GPU parity tests from the CPU oracle.

    python tests/golden/make_golden.py          # uv fixtures
    python tests/golden/make_golden.py --uvh    # uvh fixtures

The reference (MATLAB) cannot run on this machine, so the fixtures hold the
oracle's outputs (oracle/ua_ref.py, itself pinned by the analytic
known-answer tests in tests/test_oracle_kat.py) on seeded synthetic inputs:

* ``uv_<P>_<nx>x<ny>.npz`` — inputs of ``synth.ice_stream_shelf``, the
  residual and tangent at a perturbed velocity state (R, K as COO of the
  symmetrised CSC), and the converged Newton solution (rForce < 1e-20).

tests/test_golden.py checks that the oracle still reproduces these files.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ua_ref as R  # noqa: E402
from uasource_b200 import synth  # noqa: E402

CASES = [("P1", 3, 21, 11, 0), ("P2", 6, 9, 6, 0)]


def fixture_state(P, mua, res):
    """Perturbed velocity state used for the assembly comparison."""
    rng = np.random.default_rng(7)
    ub = res.ub * (1 + 0.1 * rng.standard_normal(mua.Nnodes)) + 5 * rng.standard_normal(mua.Nnodes)
    vb = res.vb * (1 + 0.1 * rng.standard_normal(mua.Nnodes)) + 5 * rng.standard_normal(mua.Nnodes)
    return ub, vb


def make(name, nod, nx, ny, seed):
    P = synth.ice_stream_shelf(nx, ny, nod=nod, seed=seed)
    mua = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    F = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    res = R.uv(p, mua, bcs, F)
    assert res.converged
    ub, vb = fixture_state(P, mua, res)
    Fs = R.prepare_fields(p, F)
    Fs.ub, Fs.vb = ub, vb
    Rv, K = R.uv_matrix_assembly(p, mua, Fs)
    K = K.tocoo()
    out = os.path.join(HERE, f"uv_{name}_{nx}x{ny}.npz")
    np.savez_compressed(
        out, coordinates=P.coordinates, connectivity=P.connectivity, h=P.h, S=P.S, B=P.B, rho=P.rho,
        AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue,
        vbFixedNode=P.vbFixedNode, vbFixedValue=P.vbFixedValue, rhow=P.rhow, g=P.g,
        state_ub=ub, state_vb=vb, R=Rv, K_row=K.row, K_col=K.col, K_val=K.data,
        sol_ub=res.ub, sol_vb=res.vb, sol_l=res.lubvb, sol_iterations=res.iterations)
    print(out, "Nele", mua.Nele, "iterations", res.iterations)


if __name__ == "__main__" and "--uvh" not in sys.argv:
    for c in CASES:
        make(*c)


UVH_CASES = [("P1", 3, 21, 11, 0), ("P2", 6, 9, 6, 0)]
UVH_DT = 0.1


def uvh_params():
    p = R.Params()
    p.set_force_tolerance(1e-20)
    p.uvhDesiredWorkAndForceTolerances = (np.inf, 1e-20)
    p.uvhDesiredWorkOrForceTolerances = (np.inf, 1e-20)
    return p


def make_uvh(name, nod, nx, ny, seed):
    """Implicit uvh step of dt=0.1 a starting from the converged diagnostic state."""
    P = synth.ice_stream_shelf(nx, ny, nod=nod, seed=seed, transient=True)
    mua = R.create_mua(P.coordinates, P.connectivity)
    p = uvh_params()
    F = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    uv = R.uv(p, mua, bcs, F)
    assert uv.converged
    S0 = R.UvhState(P.h.copy(), uv.ub.copy(), uv.vb.copy(), P.as_.copy(), P.ab.copy())
    res = R.sstream_transient_implicit(p, mua, bcs, F, S0, S0.copy(), UVH_DT)
    assert res.converged
    rng = np.random.default_rng(5)
    S1 = R.UvhState(res.h + 2 * rng.standard_normal(mua.Nnodes), res.ub * (1 + 0.05 * rng.standard_normal(mua.Nnodes)),
                    res.vb * (1 + 0.05 * rng.standard_normal(mua.Nnodes)), P.as_.copy(), P.ab.copy())
    Rv, K = R.uvh_matrix_assembly(p, mua, F, S0, S1, UVH_DT)
    K = K.tocoo()
    out = os.path.join(HERE, f"uvh_{name}_{nx}x{ny}.npz")
    np.savez_compressed(
        out, coordinates=P.coordinates, connectivity=P.connectivity, S=P.S, B=P.B, rho=P.rho,
        AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue,
        vbFixedNode=P.vbFixedNode, vbFixedValue=P.vbFixedValue, rhow=P.rhow, g=P.g, dt=UVH_DT,
        h0=S0.h, u0=S0.ub, v0=S0.vb, as_=P.as_, ab=P.ab,
        state_h=S1.h, state_ub=S1.ub, state_vb=S1.vb, R=Rv, K_row=K.row, K_col=K.col, K_val=K.data,
        sol_ub=res.ub, sol_vb=res.vb, sol_h=res.h, sol_l=res.luvh, sol_iterations=res.iterations)
    print(out, "Nele", mua.Nele, "iterations", res.iterations)


if __name__ == "__main__" and "--uvh" in sys.argv:
    for c in UVH_CASES:
        make_uvh(*c)
