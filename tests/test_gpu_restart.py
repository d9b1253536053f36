"""Restart files feed the resident handles: a problem read from a restart file solves to the same
result as the problem itself, a restart written at a converged state restarts at that state
(warm start F.ub, F.vb and l.ubvb), and restart files serve as the templates of the serving loop."""
import numpy as np
import pytest

import uasource_b200 as ua
from uasource_b200 import lib as L
from uasource_b200 import synth
from uasource_b200.restart import load_restart, save_restart
from uasource_b200.serve import Request, SsaServer

pytestmark = pytest.mark.gpu


def test_restart_problem_solves_like_the_original(tmp_path):
    P = synth.ice_stream_shelf(31, 16, seed=2)
    ctrl = ua.CtrlVar().set_force_tolerance(1e-20)
    mua = ua.CreateMUA(P.coordinates, P.connectivity)
    Fa, lam, _, _, ia = ua.uv(ctrl, mua, ua.BCs.from_problem(P), ua.Fields.from_problem(P))
    assert ia.converged
    f = tmp_path / "r.mat"
    save_restart(f, P)
    Q = load_restart(f).problem
    mq = ua.CreateMUA(Q.coordinates, Q.connectivity)
    Fb, _, _, _, ib = ua.uv(ctrl, mq, ua.BCs.from_problem(Q), ua.Fields.from_problem(Q))
    assert np.array_equal(Fa.ub, Fb.ub) and np.array_equal(Fa.vb, Fb.vb) and ia.iterations == ib.iterations
    # restart at the converged state: the warm start is already a solution
    P.ub, P.vb = Fa.ub, Fa.vb
    save_restart(f, P, lam)
    r = load_restart(f)
    Fc, lc, _, _, ic = ua.uv(ctrl, mq, ua.BCs.from_problem(r.problem), ua.Fields.from_problem(r.problem), l=r.lubvb)
    assert ic.converged and ic.iterations <= 1
    u = np.concatenate([Fa.ub, Fa.vb])
    assert np.linalg.norm(np.concatenate([Fc.ub, Fc.vb]) - u) <= 1e-12 * np.linalg.norm(u)


def test_restart_files_as_serving_templates(tmp_path):
    tpl = []
    for k, (nx, ny) in enumerate(((15, 8), (21, 11))):
        f = tmp_path / f"t{k}.mat"
        save_restart(f, synth.ice_stream_shelf(nx, ny, seed=40 + k))
        tpl.append(load_restart(f).problem)
    ctrl = ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20)
    srv = SsaServer(tpl, ctrl, replicas=1)
    reqs = [Request(rid=i, template=i % 2, C=tpl[i % 2].C, ub0=np.zeros(tpl[i % 2].Nnodes),
                    vb0=np.zeros(tpl[i % 2].Nnodes)) for i in range(4)]
    st = srv.run(reqs, realtime=False)
    assert st.completed == 4 and all(r.info.converged for r in reqs)
    srv.close()
