"""Serving form: continuous batching of SSA uv solves over resident mesh templates.

Each template (mesh, boundary conditions, base fields) is resident on the
device in one or more *slots* (systems of a batch handle), sized from free
HBM when the server starts.  A request names a template and carries its own
slipperiness C (a lognormal perturbation of the template's) and a warm-start
velocity.  The loop admits arrived requests into free slots of their template
between Newton iterations, while the other slots keep iterating
(``ua_serve_begin`` / ``ua_serve_step``), so work of requests that arrive
while others are on the GPU overlaps on the device.  Each slot's arithmetic
is independent of the other slots (per-system reductions and line searches),
so a result is the same alone and in the mix.

A request may also carry a mesh that is not a template (``problem``).  It is
admitted by its own device-memory estimate (bytes per node measured on the
resident template set, times its node count, with a margin) against the free
HBM less a reserve: admitted, it gets a handle of its own that is stepped with
the resident slots and released when it finishes; refused, it ends with status
"refused" and ``UA_ERR_OOM``.  ``cancel(rid)`` may be called from any thread:
between two Newton iterations a queued request is dropped and an active one
leaves its slot (``ua_serve_cancel``), without touching the other slots.
"""
from __future__ import annotations

import collections
import ctypes as C
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import lib as L
from .ua import BCs, CtrlVar, Fields, MUA, _c_bcs, _c_fields, _Keep, _report


@dataclass
class Request:
    rid: int
    template: int
    C: np.ndarray                 # slipperiness of this request
    ub0: np.ndarray               # warm start
    vb0: np.ndarray
    arrival: float = 0.0          # seconds after the start of the run
    problem: object = None        # a mesh that is not a template (template is then None)
    # filled by the server
    admitted: float = None
    finished: float = None
    slot: int = None
    ub: np.ndarray = None
    vb: np.ndarray = None
    info: object = None
    status: str = None            # "done", "cancelled" or "refused"
    error: int = 0                # UA_ERR_OOM for a request refused by its memory estimate
    estimate_bytes: int = None

    @property
    def latency(self):
        return None if self.finished is None else self.finished - self.arrival


@dataclass
class ServeStats:
    completed: int
    makespan_s: float
    solves_per_s: float
    p50_ms: float
    p99_ms: float
    mean_queue_ms: float
    slots: int
    steps: int
    max_active: int
    latencies_ms: list = field(default_factory=list)


class SsaServer:
    """Resident templates x replicas slots on one device."""

    def __init__(self, templates, ctrl: CtrlVar, device=0, replicas=None, hbm_fraction=0.5, max_replicas=8,
                 reserve_bytes=1 << 30, margin=1.25):
        self.templates = list(templates)
        self.ctrl = ctrl
        self.device = device
        self.reserve_bytes = int(reserve_bytes)
        self.margin = float(margin)
        self._cancel = set()
        self._lock = threading.Lock()
        lib = L.load()
        if replicas is None:
            replicas = self._replicas_from_hbm(hbm_fraction, max_replicas)
        self.replicas = max(1, int(replicas))
        self.slot_template = []
        meshes = []
        for r in range(self.replicas):
            for k, P in enumerate(self.templates):
                meshes.append((P.coordinates, P.connectivity))
                self.slot_template.append(k)
        self.mua = MUA(meshes, ndof=2, device=device)
        keep = _Keep()
        nb = len(meshes)
        cbs = (L.ua_bcs * nb)()
        for s in range(nb):
            cbs[s] = _c_bcs(BCs.from_problem(self.templates[self.slot_template[s]]), keep)
        self._p = ctrl.to_c()
        L.check(lib.ua_serve_setup(self.mua.handle, C.byref(self._p), cbs))
        self.free = collections.defaultdict(collections.deque)
        for s, k in enumerate(self.slot_template):
            self.free[k].append(s)
        # device bytes per node of a resident, set-up slot: the memory model of admission
        self.bytes_per_node = self.mua.device_bytes() / max(1, sum(self.templates[k].Nnodes
                                                                   for k in self.slot_template))

    # -- admission of a mesh that is not a template, by its memory estimate --------------
    def estimate_bytes(self, P):
        """Device bytes a handle for problem P is expected to take (set up for serving)."""
        return int(self.margin * self.bytes_per_node * P.Nnodes)

    def free_bytes(self):
        free = C.c_int64()
        total = C.c_int64()
        L.check(L.load().ua_mem_info(self.device, C.byref(free), C.byref(total)))
        return free.value

    def cancel(self, rid):
        """Cancels request rid (queued or active); safe from any thread, applied between steps."""
        with self._lock:
            self._cancel.add(rid)

    # -- admission by free HBM ---------------------------------------------------------
    def _replicas_from_hbm(self, fraction, max_replicas):
        """Replicas of the template set that fit in `fraction` of the free device memory,
        measured with one resident copy of every template."""
        lib = L.load()
        probe = MUA([(P.coordinates, P.connectivity) for P in self.templates], ndof=2, device=self.device)
        keep = _Keep()
        nb = len(self.templates)
        cbs = (L.ua_bcs * nb)()
        for s, P in enumerate(self.templates):
            cbs[s] = _c_bcs(BCs.from_problem(P), keep)
        p = self.ctrl.to_c()
        L.check(lib.ua_serve_setup(probe.handle, C.byref(p), cbs))
        per_set = probe.device_bytes()
        probe.close()
        free = C.c_int64()
        total = C.c_int64()
        L.check(lib.ua_mem_info(self.device, C.byref(free), C.byref(total)))
        return int(max(1, min(max_replicas, (fraction * free.value) // max(per_set, 1))))

    @property
    def nslots(self):
        return len(self.slot_template)

    def _fields(self, req: Request, keep: _Keep):
        P = self.templates[req.template] if req.problem is None else req.problem
        F = Fields.from_problem(P)
        F.C = req.C
        F.ub = req.ub0
        F.vb = req.vb0
        cf, _, _ = _c_fields(F, keep, P.Nnodes)
        return cf

    def _result(self, mua, slot, r, P, tnow):
        lib = L.load()
        r.ub = np.zeros(P.Nnodes)
        r.vb = np.zeros(P.Nnodes)
        rep = L.ua_newton_report()
        cap = 2 * (self.ctrl.NRitmax + 2)
        recs = (L.ua_newton_iter * cap)()
        rep.iters = C.cast(recs, C.POINTER(L.ua_newton_iter))
        rep.iters_capacity = cap
        L.check(lib.ua_serve_result(mua.handle, int(slot), L.dptr(r.ub), L.dptr(r.vb), C.byref(rep)))
        r.info = _report(rep, recs)
        r.finished = tnow
        r.status = "done"

    def _admit_own(self, r, now):
        """A request with its own mesh: admitted on its memory estimate into a handle of its own,
        else refused with UA_ERR_OOM.  Returns the handle or None."""
        lib = L.load()
        P = r.problem
        r.estimate_bytes = self.estimate_bytes(P)
        if r.estimate_bytes > self.free_bytes() - self.reserve_bytes:
            r.status, r.error, r.admitted, r.finished = "refused", L.UA_ERR_OOM, now, now
            return None
        mua = MUA([(P.coordinates, P.connectivity)], ndof=2, device=self.device)
        keep = _Keep()
        cbs = (L.ua_bcs * 1)()
        cbs[0] = _c_bcs(BCs.from_problem(P), keep)
        L.check(lib.ua_serve_setup(mua.handle, C.byref(self._p), cbs))
        cfs = (L.ua_fields * 1)()
        cfs[0] = self._fields(r, keep)
        sys_ids = np.zeros(1, np.int32)
        L.check(lib.ua_serve_begin(mua.handle, C.byref(self._p), 1, L.iptr(sys_ids), cfs))
        r.slot, r.admitted = 0, now
        return mua

    def run(self, requests, realtime=True, sleep=time.sleep, on_step=None):
        """Serve `requests` (sorted by arrival time).  With realtime=False the
        arrivals are taken as already due when the loop reaches them (offline batch).
        on_step(step, server), if given, runs after every step (for instance to cancel)."""
        lib = L.load()
        queue = collections.deque(sorted(requests, key=lambda r: r.arrival))
        pending = collections.deque()
        active = {}
        own = {}  # rid -> (handle, request): requests with their own mesh
        nslots = self.nslots
        finished = np.zeros(nslots, np.int32)
        fin1 = np.zeros(1, np.int32)
        nact = C.c_int32()
        t0 = time.perf_counter()
        steps = 0
        max_active = 0
        done = []
        while queue or pending or active or own:
            now = time.perf_counter() - t0
            while queue and (queue[0].arrival <= now or not realtime):
                pending.append(queue.popleft())
            # cancellations (from any thread): queued requests are dropped, active ones leave
            with self._lock:
                cancel, self._cancel = self._cancel, set()
            if cancel:
                for dq in (queue, pending):
                    for r in [x for x in dq if x.rid in cancel]:
                        dq.remove(r)
                        r.status, r.finished = "cancelled", now
                        done.append(r)
                slots = [s for s, r in active.items() if r.rid in cancel]
                if slots:
                    L.check(lib.ua_serve_cancel(self.mua.handle, len(slots), L.iptr(np.array(slots, np.int32))))
                    for s in slots:
                        r = active.pop(s)
                        r.status, r.finished = "cancelled", now
                        self.free[r.template].append(s)
                        done.append(r)
                for rid in [x for x in own if x in cancel]:
                    mua, r = own.pop(rid)
                    mua.close()
                    r.status, r.finished = "cancelled", now
                    done.append(r)
            # admit arrived requests into free slots of their template (FIFO per template); a
            # request with its own mesh by its memory estimate
            admit, keep = [], _Keep()
            still = collections.deque()
            while pending:
                r = pending.popleft()
                if r.problem is not None:
                    h = self._admit_own(r, now)
                    if h is None:
                        done.append(r)
                    else:
                        own[r.rid] = (h, r)
                elif self.free[r.template]:
                    r.slot = self.free[r.template].popleft()
                    r.admitted = now
                    admit.append(r)
                else:
                    still.append(r)
            pending = still
            if admit:
                sys_ids = np.array([r.slot for r in admit], np.int32)
                cfs = (L.ua_fields * len(admit))()
                for i, r in enumerate(admit):
                    cfs[i] = self._fields(r, keep)
                L.check(lib.ua_serve_begin(self.mua.handle, C.byref(self._p), len(admit), L.iptr(sys_ids), cfs))
                for r in admit:
                    active[r.slot] = r
            if not active and not own:
                if queue and realtime:
                    sleep(max(0.0, queue[0].arrival - (time.perf_counter() - t0)))
                continue
            max_active = max(max_active, len(active) + len(own))
            if active:
                L.check(lib.ua_serve_step(self.mua.handle, C.byref(self._p), L.iptr(finished), C.byref(nact)))
            for rid, (h, r) in list(own.items()):
                L.check(lib.ua_serve_step(h.handle, C.byref(self._p), L.iptr(fin1), C.byref(nact)))
                if fin1[0]:
                    self._result(h, 0, r, r.problem, time.perf_counter() - t0)
                    h.close()
                    del own[rid]
                    done.append(r)
            steps += 1
            tnow = time.perf_counter() - t0
            if active:
                for s in np.flatnonzero(finished):
                    r = active.pop(int(s))
                    self._result(self.mua, s, r, self.templates[r.template], tnow)
                    self.free[r.template].append(int(s))
                    done.append(r)
            if on_step is not None:
                on_step(steps, self)
        makespan = time.perf_counter() - t0
        served = [r for r in done if r.status == "done"]
        lat = sorted(1000 * r.latency for r in served)
        q = [1000 * (r.admitted - r.arrival) for r in served]
        pct = lambda a, f: a[min(len(a) - 1, int(f * len(a)))] if a else float("nan")
        return ServeStats(len(served), makespan, len(served) / makespan if makespan > 0 else float("nan"),
                          pct(lat, 0.5), pct(lat, 0.99), float(np.mean(q)) if q else float("nan"), nslots, steps,
                          max_active, lat)

    def close(self):
        self.mua.close()


def perturbed_C(P, rng, sigma=0.3):
    """Lognormal perturbation of a template's C: C * exp(sigma z), z ~ N(0,1) per node."""
    return P.C * np.exp(sigma * rng.standard_normal(P.Nnodes))


def poisson_arrivals(n, rate, rng):
    """Arrival times (s) of n requests of a Poisson process with the given rate (1/s)."""
    return np.cumsum(rng.exponential(1.0 / rate, n))
