"""Serving form: continuous batching gives the same result per request alone
and in the mix, and requests that arrive while others iterate overlap."""
import numpy as np
import pytest

import uasource_b200 as ua
from uasource_b200 import lib as L
from uasource_b200 import synth
from uasource_b200.serve import Request, SsaServer, perturbed_C

pytestmark = pytest.mark.gpu


def _templates():
    return [synth.ice_stream_shelf(15, 8, seed=21), synth.ice_stream_shelf(21, 11, seed=22),
            synth.ice_stream_shelf(31, 16, seed=23)]


def _requests(templates, n, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        k = i % len(templates)
        P = templates[k]
        reqs.append(Request(rid=i, template=k, C=perturbed_C(P, rng), ub0=np.zeros(P.Nnodes), vb0=np.zeros(P.Nnodes),
                            arrival=0.0))
    return reqs


@pytest.mark.parametrize("precision,rtol", [(L.UA_PREC_MIXED, 1e-6), (L.UA_PREC_FP64, 1e-12)])
def test_served_results_equal_alone(precision, rtol):
    tpl = _templates()
    ctrl = ua.CtrlVar(precision=precision, krylov_rtol=rtol).set_force_tolerance(1e-20)
    srv = SsaServer(tpl, ctrl, replicas=2)
    reqs = _requests(tpl, 9, seed=4)
    # staggered joins: requests enter between Newton iterations of earlier ones
    for i, r in enumerate(reqs):
        r.arrival = 0.002 * i
    stats = srv.run(reqs, realtime=True)
    assert stats.completed == len(reqs)
    assert stats.max_active > 1
    for r in reqs:
        assert r.info.converged
        P = tpl[r.template]
        mua = ua.CreateMUA(P.coordinates, P.connectivity)
        F = ua.Fields.from_problem(P)
        F.C = r.C
        Fo, _, _, _, info = ua.uv(ctrl, mua, ua.BCs.from_problem(P), F)
        assert np.array_equal(Fo.ub, r.ub) and np.array_equal(Fo.vb, r.vb)
        assert info.iterations == r.info.iterations
        mua.close()
    srv.close()


def test_mixed_served_within_tolerance_of_plain_fp64():
    tpl = _templates()
    srv = SsaServer(tpl, ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20),
                    replicas=1)
    reqs = _requests(tpl, 3, seed=9)
    srv.run(reqs, realtime=False)
    ctrl64 = ua.CtrlVar().set_force_tolerance(1e-20)
    for r in reqs:
        P = tpl[r.template]
        mua = ua.CreateMUA(P.coordinates, P.connectivity)
        F = ua.Fields.from_problem(P)
        F.C = r.C
        Fo, _, _, _, _ = ua.uv(ctrl64, mua, ua.BCs.from_problem(P), F)
        u64 = np.concatenate([Fo.ub, Fo.vb])
        u = np.concatenate([r.ub, r.vb])
        assert np.linalg.norm(u - u64) <= 1e-8 * np.linalg.norm(u64)
        mua.close()
    srv.close()


def _solve_alone(ctrl, P, C):
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    F = ua.Fields.from_problem(P)
    F.C = C
    Fo, _, _, _, info = ua.uv(ctrl, mua, ua.BCs.from_problem(P), F)
    mua.close()
    return Fo, info


def test_cancel_leaves_the_other_slots_bit_identical():
    """A request cancelled from another thread between steps (one active, one still queued)
    frees its slot; every other request's result is the one it gets alone, bit for bit."""
    import threading
    tpl = _templates()
    ctrl = ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20)
    srv = SsaServer(tpl, ctrl, replicas=1)
    reqs = _requests(tpl, 7, seed=12)
    for i, r in enumerate(reqs):
        r.arrival = 0.0 if i < 3 else 10.0  # the last four wait in the queue (offline run)
    cancelled = {1, 5}

    def on_step(step, server):
        if step == 2:  # from a host thread, as a client would
            t = threading.Thread(target=lambda: [server.cancel(rid) for rid in cancelled])
            t.start()
            t.join()

    srv.run(reqs, realtime=False, on_step=on_step)
    for r in reqs:
        if r.rid in cancelled:
            assert r.status == "cancelled" and r.info is None
            continue
        assert r.status == "done" and r.info.converged
        Fo, info = _solve_alone(ctrl, tpl[r.template], r.C)
        assert np.array_equal(Fo.ub, r.ub) and np.array_equal(Fo.vb, r.vb)
        assert info.iterations == r.info.iterations
    srv.close()


def test_own_mesh_request_is_admitted_by_its_memory_estimate():
    """A mesh that is not a template is admitted on its device-memory estimate, solved with the
    resident slots in the same loop, and gives the result it gets alone."""
    tpl = _templates()
    ctrl = ua.CtrlVar(precision=L.UA_PREC_FP64, krylov_rtol=1e-12).set_force_tolerance(1e-20)
    srv = SsaServer(tpl, ctrl, replicas=1)
    reqs = _requests(tpl, 3, seed=3)
    P = synth.ice_stream_shelf(27, 14, seed=31)
    rng = np.random.default_rng(5)
    own = Request(rid=99, template=None, problem=P, C=perturbed_C(P, rng), ub0=np.zeros(P.Nnodes),
                  vb0=np.zeros(P.Nnodes))
    stats = srv.run(reqs + [own], realtime=False)
    assert stats.completed == 4 and stats.max_active == 4
    assert own.status == "done" and own.info.converged
    assert 0 < own.estimate_bytes < srv.free_bytes()
    Fo, info = _solve_alone(ctrl, P, own.C)
    assert np.array_equal(Fo.ub, own.ub) and np.array_equal(Fo.vb, own.vb)
    srv.close()


def test_own_mesh_request_is_refused_when_its_estimate_exceeds_free_hbm():
    tpl = _templates()
    ctrl = ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20)
    srv = SsaServer(tpl, ctrl, replicas=1)
    P = synth.ice_stream_shelf(21, 11, seed=32)
    own = Request(rid=7, template=None, problem=P, C=P.C, ub0=np.zeros(P.Nnodes), vb0=np.zeros(P.Nnodes))
    srv.reserve_bytes = srv.free_bytes()  # nothing left for a new handle
    reqs = _requests(tpl, 2, seed=8)
    stats = srv.run(reqs + [own], realtime=False)
    assert own.status == "refused" and own.error == L.UA_ERR_OOM and own.info is None
    assert stats.completed == 2 and all(r.status == "done" for r in reqs)
    srv.close()
