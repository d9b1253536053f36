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
"""
from __future__ import annotations

import collections
import ctypes as C
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
    # filled by the server
    admitted: float = None
    finished: float = None
    slot: int = None
    ub: np.ndarray = None
    vb: np.ndarray = None
    info: object = None

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

    def __init__(self, templates, ctrl: CtrlVar, device=0, replicas=None, hbm_fraction=0.5, max_replicas=8):
        self.templates = list(templates)
        self.ctrl = ctrl
        self.device = device
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
        P = self.templates[req.template]
        F = Fields.from_problem(P)
        F.C = req.C
        F.ub = req.ub0
        F.vb = req.vb0
        cf, _, _ = _c_fields(F, keep, P.Nnodes)
        return cf

    def run(self, requests, realtime=True, sleep=time.sleep):
        """Serve `requests` (sorted by arrival time).  With realtime=False the
        arrivals are taken as already due when the loop reaches them (offline batch)."""
        lib = L.load()
        queue = collections.deque(sorted(requests, key=lambda r: r.arrival))
        pending = collections.deque()
        active = {}
        nslots = self.nslots
        finished = np.zeros(nslots, np.int32)
        nact = C.c_int32()
        t0 = time.perf_counter()
        steps = 0
        max_active = 0
        done = []
        while queue or pending or active:
            now = time.perf_counter() - t0
            while queue and (queue[0].arrival <= now or not realtime):
                pending.append(queue.popleft())
            # admit arrived requests into free slots of their template (FIFO per template)
            admit, keep = [], _Keep()
            still = collections.deque()
            while pending:
                r = pending.popleft()
                if self.free[r.template]:
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
            if not active:
                if queue and realtime:
                    sleep(max(0.0, queue[0].arrival - (time.perf_counter() - t0)))
                continue
            max_active = max(max_active, len(active))
            L.check(lib.ua_serve_step(self.mua.handle, C.byref(self._p), L.iptr(finished), C.byref(nact)))
            steps += 1
            tnow = time.perf_counter() - t0
            for s in np.flatnonzero(finished):
                r = active.pop(int(s))
                P = self.templates[r.template]
                r.ub = np.zeros(P.Nnodes)
                r.vb = np.zeros(P.Nnodes)
                rep = L.ua_newton_report()
                cap = 2 * (self.ctrl.NRitmax + 2)
                recs = (L.ua_newton_iter * cap)()
                rep.iters = C.cast(recs, C.POINTER(L.ua_newton_iter))
                rep.iters_capacity = cap
                L.check(lib.ua_serve_result(self.mua.handle, int(s), L.dptr(r.ub), L.dptr(r.vb), C.byref(rep)))
                r.info = _report(rep, recs)
                r.finished = tnow
                self.free[r.template].append(int(s))
                done.append(r)
        makespan = time.perf_counter() - t0
        lat = sorted(1000 * r.latency for r in done)
        q = [1000 * (r.admitted - r.arrival) for r in done]
        pct = lambda a, f: a[min(len(a) - 1, int(f * len(a)))] if a else float("nan")
        return ServeStats(len(done), makespan, len(done) / makespan if makespan > 0 else float("nan"),
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
