"""Benchmark: uv Newton solves/s of the SSA (SSTREAM) diagnostic solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one complete uv Newton solve from u=v=0 to rForce<1e-20):
the ice-stream/ice-shelf rectangle of 100 km x 50 km, 141x71 vertices,
19,600 P1 elements (seeded synthetic fields: bed, thickness with bumps,
smoothed Glen A and Weertman C, n=m=3; u=v=0 at x=0, free-slip sides,
calving front).  Inputs are ~4 MB, far below the 126 MB L2, so a 512 MB
buffer is written between timed steps to flush L2.

Reported: ``value`` = solves/s of the mixed-precision form (FP32 tangents and
PCG, FP64 residual/line search/update) with inputs resident in HBM;
``plain_fp64`` = the same for the all-FP64 form; ``e2e`` = the mixed form
through the public C-ABI with host buffers (host->device copies and the
device->host read of the solution inside the timed region).  Errors of each
form against the FP64 result are reported; the CPU baseline is the numpy
restatement of the reference algorithm (oracle/ua_ref.py).

Multi-GPU: independent replicas (the diagnostic solve of one mesh does not
shard; whole meshes are independent work units), one process per GPU, time
= max over ranks.  ``--impl reference`` times the CPU restatement on the
host cores (a process pool, one solve per worker per step).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, SEED = 141, 71, 0
WORKLOAD = (f"uv diagnostic Newton solve (SSTREAM2dNR2), ice stream/shelf 100x50 km, {NX}x{NY} vertices, "
            f"{2 * (NX - 1) * (NY - 1)} P1 elements, 10011 nodes, seed {SEED}, rForce<1e-20")
METRIC = "uv Newton solves/s (mixed FP32/FP64, <=1e-8 rel err vs FP64)"


MESH = (NX, NY)


def _problem():
    from uasource_b200 import synth
    return synth.ice_stream_shelf(MESH[0], MESH[1], nod=3, seed=SEED)


# ----------------------------------------------------------------------------- CPU reference arm

def _ref_solve_once(seed):
    """One full oracle solve (child process)."""
    import numpy as np  # noqa: F401
    sys.path.insert(0, ROOT)
    from oracle import ua_ref as R
    P = _problem()
    mua = R.create_mua(P.coordinates, P.connectivity)
    p = R.Params()
    p.set_force_tolerance(1e-20)
    F = R.Fields(h=P.h, S=P.S, B=P.B, rho=P.rho, AGlen=P.AGlen, n=P.n, C=P.C, m=P.m, ub=P.ub, vb=P.vb)
    bcs = R.BCs(ubFixedNode=P.ubFixedNode, ubFixedValue=P.ubFixedValue, vbFixedNode=P.vbFixedNode,
                vbFixedValue=P.vbFixedValue)
    t = time.perf_counter()
    res = R.uv(p, mua, bcs, F)
    return time.perf_counter() - t, bool(res.converged)


def _cpu_baseline_single(max_seconds=25.0):
    """Oracle port on one core: solves until ~max_seconds of CPU work."""
    ts = []
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < max_seconds * 0.5 or not ts:
        dt, ok = _ref_solve_once(SEED)
        ts.append(dt)
        if time.perf_counter() - t0 > max_seconds:
            break
    return len(ts) / sum(ts), len(ts)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"
    cores = os.cpu_count() or 1
    workers = max(1, min(cores, 32))
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        for _ in range(args.warmup):
            pool.map(_ref_solve_once, [SEED] * workers)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            res = pool.map(_ref_solve_once, [SEED] * workers)
        el = time.perf_counter() - t0
    solves = args.steps * workers
    value = solves / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": workers, "kind": "port",
                         "sample": f"{workers} concurrent oracle solves per step (numpy/scipy restatement, "
                                   f"one process per core)"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "converged": all(ok for _, ok in res),
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- GPU arm

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in open(self.path):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1])); smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _flush_l2(buf):
    buf.add_(1.0)


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    import uasource_b200 as ua
    from uasource_b200 import lib as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return t.item()

    P = _problem()
    mua = ua.CreateMUA(P.coordinates, P.connectivity, device=local)
    bcs = ua.BCs.from_problem(P)
    names = ("h", "S", "B", "rho", "AGlen", "n", "C", "m")
    dev_in = {k: torch.tensor(getattr(P, k), dtype=torch.float64, device=dev) for k in names}
    ub = torch.zeros(P.Nnodes, dtype=torch.float64, device=dev)
    vb = torch.zeros_like(ub)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float64, device=dev)  # 512 MB > L2
    ctrl64 = ua.CtrlVar(precision=L.UA_PREC_FP64, krylov_rtol=1e-12).set_force_tolerance(1e-20)
    ctrlmx = ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6).set_force_tolerance(1e-20)
    if args.newton_its:
        ctrl64.NRitmax = ctrlmx.NRitmax = args.newton_its
    if args.krylov_maxit:
        ctrl64.krylov_maxit = ctrlmx.krylov_maxit = args.krylov_maxit

    def solve_resident(ctrl):
        ub.zero_(); vb.zero_()
        torch.cuda.synchronize()
        ptrs = {k: v.data_ptr() for k, v in dev_in.items()}
        ptrs["ub"] = ub.data_ptr(); ptrs["vb"] = vb.data_ptr()
        _, info = ua.uv_resident(ctrl, mua, bcs, ptrs, rhow=P.rhow, g=P.g)
        return info

    def timed(ctrl, steps, warmup, sampler=None):
        for _ in range(warmup):
            solve_resident(ctrl)
        barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        per, lat, launches, infos = [], [], 0, []
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        for _ in range(steps):
            _flush_l2(flush)
            torch.cuda.synchronize()
            e0.record()
            info = solve_resident(ctrl)
            e1.record()
            torch.cuda.synchronize()
            per.append(e0.elapsed_time(e1))
            lat.append(info.device_ms)
            launches += info.gpu_launches
            infos.append(info)
        clocks = sampler.stop() if sampler else None
        barrier()
        return per, lat, launches, infos, clocks

    if args.legs == "mixed":  # profiling runs: the timed mixed-precision solves only
        timed(ctrlmx, args.steps, args.warmup)
        mua.close()
        if world > 1:
            dist.destroy_process_group()
        return 0
    # reference solution of the plain FP64 form (for the error report)
    info64 = solve_resident(ctrl64)
    u64 = torch.cat([ub, vb]).cpu().numpy()
    sampler = ClockSampler(local)
    per_mx, lat_mx, launches_mx, infos_mx, clocks = timed(ctrlmx, args.steps, args.warmup, sampler)
    u_mx = torch.cat([ub, vb]).cpu().numpy()
    per_64, lat_64, launches_64, infos_64, _ = timed(ctrl64, args.steps, max(1, args.warmup // 2))
    err_mx = float(np.linalg.norm(u_mx - u64) / np.linalg.norm(u64))

    # kernel timings (separate profiled solves; CUDA events on the library's stream)
    prof = solve_resident(ua.CtrlVar(precision=L.UA_PREC_MIXED, krylov_rtol=1e-6, profile=1)
                          .set_force_tolerance(1e-20))
    prof64 = solve_resident(ua.CtrlVar(precision=L.UA_PREC_FP64, krylov_rtol=1e-12, profile=1)
                            .set_force_tolerance(1e-20))

    # e2e: the public API with host buffers (pinned), copies inside the timed region
    pin = {k: torch.tensor(getattr(P, k), dtype=torch.float64).pin_memory() for k in names}
    pin_u = torch.zeros(P.Nnodes, dtype=torch.float64).pin_memory()
    Fh = ua.Fields(**{k: pin[k].numpy() for k in names}, ub=pin_u.numpy(), vb=pin_u.numpy(), rhow=P.rhow, g=P.g)
    for _ in range(max(1, args.warmup // 2)):
        ua.uv(ctrlmx, mua, bcs, Fh)
    barrier(); torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    e2e_ms = []
    for _ in range(args.steps):
        _flush_l2(flush); torch.cuda.synchronize()
        e0.record()
        Fo, _, _, _, info_e = ua.uv(ctrlmx, mua, bcs, Fh)
        e1.record(); torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    barrier()
    Nn = P.Nnodes
    h2d = 8 * Nn * (len(names) + 2) + 12 * (len(bcs.ubFixedNode) + len(bcs.vbFixedNode))
    d2h = 8 * 2 * Nn + 8 * (len(bcs.ubFixedNode) + len(bcs.vbFixedNode))

    t_mx = max_over_ranks(sum(per_mx))
    t_64 = max_over_ranks(sum(per_64))
    t_e2e = max_over_ranks(sum(e2e_ms))
    value = world * args.steps / (t_mx / 1000)
    value64 = world * args.steps / (t_64 / 1000)
    e2e_value = world * args.steps / (t_e2e / 1000)

    # roofline of the dominant kernel class (by measured device time)
    nnz = int(mua.pattern()[1].size)
    Ne = P.Nele
    rows = 2 * Nn
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    k = prof.kernels
    cand = {
        "uv_patch_kernel<3,K,float> (tangent+residual assembly)":
            (k["asmK_ms"], k["asmK_n"], 12 * Ne + 16 * Nn + 80 * Nn + 4 * nnz + 8 * rows),
        "uv_patch_kernel<3,R> (residual-only assembly)":
            (k["asmR_ms"], k["asmR_n"], 12 * Ne + 16 * Nn + 80 * Nn + 8 * rows),
        "k_pcg_spmv<float,float> (PCG SpMV + p.q)":
            (k["spmv_ms"], k["spmv_n"], 8 * nnz + 4 * (rows + 1) + 4 * rows + 4 * rows + rows),
    }
    dom = max(cand, key=lambda c: cand[c][0])
    ms, n, alg = cand[dom]
    avg_ms = ms / max(n, 1)
    achieved = alg / (avg_ms / 1000) / 1e9 if n else 0.0
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "traffic": None,
            "alg_bytes_per_launch": alg, "avg_launch_ms": avg_ms, "launches": n,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (burst copy)" if "hbm_gbs" in peaks else "fallback 6650",
            "kernel_share": {c: v[0] / max(sum(x[0] for x in cand.values()), 1e-12) for c, v in cand.items()}}

    cpu = None
    if rank == 0 and not args.skip_cpu:
        v, nsamp = _cpu_baseline_single(args.cpu_seconds)
        cpu = {"value": v, "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": f"{nsamp} full oracle solve(s) of the same workload, single process"}

    if rank == 0:
        lat_sorted = sorted(lat_mx)
        p99 = lat_sorted[min(len(lat_sorted) - 1, int(0.99 * len(lat_sorted)))]
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_mx / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 mixed", "data": "synthetic",
            "config": {"workload": WORKLOAD, "l2": "flushed (512 MB write) between timed steps",
                       "parallelism": f"replicas x{world}", "precision": "mixed", "krylov": "Jacobi-PCG",
                       "newton_iterations": infos_mx[-1].iterations,
                       "pcg_iterations": infos_mx[-1].krylov_its_total},
            "p50_ms": statistics.median(lat_mx), "p99_ms": p99,
            "rel_err_vs_fp64": err_mx,
            "plain_fp64": {"value": value64, "unit": "solves/s", "ms_per_step": t_64 / args.steps,
                           "newton_iterations": infos_64[-1].iterations,
                           "pcg_iterations": infos_64[-1].krylov_its_total,
                           "p99_ms": sorted(lat_64)[min(len(lat_64) - 1, int(0.99 * len(lat_64)))]},
            "mixed_over_plain": value / value64,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": roof,
            "kernels_fp64": prof64.kernels,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches_mx,
        }
        print(json.dumps(line), flush=True)
    mua.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    # profiling-only options (ncu captures on bounded cases); the bench line uses the defaults
    ap.add_argument("--legs", default="all", choices=["all", "mixed"])
    ap.add_argument("--mesh", default=None, help="NXxNY vertices instead of the workload mesh")
    ap.add_argument("--newton-its", type=int, default=0)
    ap.add_argument("--krylov-maxit", type=int, default=0)
    args = ap.parse_args()
    if args.mesh:
        global MESH
        MESH = tuple(int(v) for v in args.mesh.lower().split("x"))
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
