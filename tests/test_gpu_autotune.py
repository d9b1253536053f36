"""The assembly autotuner (ua_autotune) and the schedules it chooses between: patch shapes
(patch_nodes), P1 CTA sizes (asm_threads) and register budgets (asm_regs) change where and how
the element work runs, not what is
summed in which order, so the tangent, the residual and whole Newton solves are bit-identical
under every schedule; the tuner times every candidate and keeps the fastest."""
import numpy as np
import pytest

import uasource_b200 as ua
from uasource_b200 import lib as L
from uasource_b200 import synth

pytestmark = pytest.mark.gpu


def _state(P, seed=2):
    rng = np.random.default_rng(seed)
    return 100 + 200 * rng.random(P.Nnodes), 30 * rng.standard_normal(P.Nnodes)


@pytest.mark.parametrize("nod,nx,ny", [(3, 61, 31), (6, 21, 11)], ids=["P1", "P2"])
@pytest.mark.parametrize("precision", [L.UA_PREC_FP64, L.UA_PREC_MIXED], ids=["fp64", "mixed"])
def test_assembly_is_bit_identical_under_every_schedule(nod, nx, ny, precision):
    P = synth.ice_stream_shelf(nx, ny, nod=nod, seed=1)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)
    F.ub, F.vb = _state(P)
    out = []
    scheds = ((256, 128), (128, 128), (128, 96), (256, 80), (128, 80)) if nod == 3 else ((0, 0),)
    for pn in (0, 16, 37, 128):
        for t, rg in scheds:
            ctrl = ua.CtrlVar(precision=precision, patch_nodes=pn, asm_threads=t, asm_regs=rg)
            R, K = ua.uvMatrixAssembly(ctrl, mua, F)
            Rr, _ = ua.uvMatrixAssembly(ctrl, mua, F, Ronly=True)
            assert np.array_equal(Rr, R)  # the residual-only pass computes R with the same instructions
            out.append((R, K.data.copy()))
    for R, Kd in out[1:]:
        assert np.array_equal(R, out[0][0]) and np.array_equal(Kd, out[0][1])


def test_autotune_times_every_candidate_and_keeps_the_fastest():
    probs = [synth.ice_stream_shelf(41, 21, seed=0), synth.ice_stream_shelf(81, 41, seed=3),
             synth.ice_stream_shelf(25, 13, seed=7)]
    mua = ua.CreateMUABatch([(P.coordinates, P.connectivity) for P in probs])
    Fs = [ua.Fields.from_problem(P) for P in probs]
    bcs = [ua.BCs.from_problem(P) for P in probs]
    ctrl = ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20)
    before = ua.uv_batch(ctrl, mua, [F.copy() for F in Fs], bcs)
    t = ua.autotune(ctrl, mua, Fs, reps=2)
    c = t["candidates"]
    assert len(c) == 35  # seven patch shapes x five (CTA size, register budget) schedules (P1)
    assert {x["threads"] for x in c} == {128, 256} and {x["regs"] for x in c} == {128, 96, 80}
    assert all(x["ms"] > 0 for x in c)
    assert t["chosen"]["ms"] == min(x["ms"] for x in c)
    assert t["default_ms"] == c[0]["ms"] and (c[0]["div"], c[0]["cap"], c[0]["threads"], c[0]["regs"]) == \
        (600, 128, 256, 128)
    after = ua.uv_batch(ctrl, mua, [F.copy() for F in Fs], bcs)  # now on the tuned schedule
    for (ua_, va, ia), (ub_, vb_, ib) in zip(before, after):
        assert ia.converged and ib.converged and ia.iterations == ib.iterations
        assert np.array_equal(ua_, ub_) and np.array_equal(va, vb_)
    # a new handle takes the tuned schedule too, with the same results
    m2 = ua.CreateMUABatch([(P.coordinates, P.connectivity) for P in probs])
    again = ua.uv_batch(ctrl, m2, [F.copy() for F in Fs], bcs)
    for (ua_, va, _), (ub_, vb_, _) in zip(before, again):
        assert np.array_equal(ua_, ub_) and np.array_equal(va, vb_)


def test_bad_schedule_is_refused():
    P = synth.ice_stream_shelf(9, 6, seed=0)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    for kw in (dict(patch_nodes=-1), dict(patch_nodes=5000), dict(asm_threads=96), dict(asm_regs=64),
               dict(asm_threads=256, asm_regs=96)):
        with pytest.raises(L.UaError) as ei:
            ua.uvMatrixAssembly(ua.CtrlVar(**kw), mua, ua.Fields.from_problem(P))
        assert ei.value.code == L.UA_ERR_INVALID
