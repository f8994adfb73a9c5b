"""Benchmark: UA-AMG-PCG time to a 1e-8 FP64 relative residual on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload c2|c1|c5]

Workload (default c2): 3D P1 diffusion -div(k grad u) = f on the Kuhn
tetrahedral mesh of 128^3 cubes (127^3 = 2,048,383 dofs, 30,340,171 stored
entries of the 15-point pattern), k = exp(g) per cube with g a unit-variance
Gaussian field of correlation length 8 cubes (seed 2), b ~ U[-1,1] (seed 3),
x0 = 0.  Synthetic, seeded inputs of the configuration's shapes.

One step = one UA-AMG-PCG solve of that system from x0 = 0 to 1e-8 FP64
relative residual, setup (aggregation + Galerkin products + coarse
factorisation) included: the time a user pays for one call.  `value` is that
time with the matrix and vectors resident in HBM (FP32 V-cycle inside FP64
flexible CG, the mixed form); `e2e` is the same solve through the drop-in C
entry point with host arrays (copies included).  The plain FP64 drop-in is
timed beside it (`plain_fp64_*`), and the level SpMV is timed on its own for
the roofline.  The stored matrix (364 MB) exceeds the 126 MB L2, so no
explicit flush is needed between steps.

--impl reference times the reference HAZmath implementation (compiled from
its sources, single-threaded C) on the same workload and settings.
Multi-GPU: the path does not shard; N ranks run N independent replicas.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from hazmath_b200 import problems as P  # noqa: E402

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def workload(name: str):
    if name == "c1":
        ia, ja, val = P.poisson2d_5pt(255)
        b = P.rhs_uniform(len(ia) - 1, 1)
        desc = {"workload": "2D P1 Poisson 257^2 vertices (255^2 dofs, 5-pt)",
                "dofs": int(len(b)), "nnz": int(ia[-1])}
        return ia, ja, val, b, desc
    N, sigma, seeds = (128, 1.0, (2, 3)) if name == "c2" else (256, 1.5, (7, 8))
    k = P.lognormal_field(N, sigma, 8.0, seeds[0])
    ia, ja, val = P.kuhn3d_p1(N, k)
    b = P.rhs_uniform(len(ia) - 1, seeds[1])
    desc = {"workload": f"3D P1 log-normal diffusion, Kuhn mesh {N}^3 cubes "
                        f"(sigma={sigma}, corr 8 cubes)",
            "dofs": int(len(b)), "nnz": int(ia[-1])}
    return ia, ja, val, b, desc


class Clocks:
    """nvidia-smi sampler during the timed region."""

    def __init__(self, index: int):
        self.p = None
        self.path = os.path.join("/tmp", f"hzb_clocks_{os.getpid()}.csv")
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        rows = []
        for ln in open(self.path):
            f = [x.strip() for x in ln.split(",")]
            if len(f) >= 7:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][1]) if rows[0][1].replace(".", "").isdigit()
                else None, "reasons": reasons, "samples": len(rows)}


def hbm_peak():
    try:
        return float(json.load(open(PEAKS))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM, "fallback"


def amg_l1(hz):
    return hz.survey_amg(smoother=hz.SMOOTHER_L1DIAG, presmooth_iter=2, postsmooth_iter=2)


def itparam(hz):
    return hz.itsolver_param(linear_itsolver_type=hz.SOLVER_CG,
                             linear_precond_type=hz.PREC_AMG, linear_tol=1e-8,
                             linear_maxit=500, linear_stop_type=hz.STOP_REL_RES)


def run_reference(args, ia, ja, val, b, desc):
    import oracle
    kind = "reference" if oracle.ref_available() else "port"
    R = oracle.ref() if kind == "reference" else oracle.port()
    prm = oracle.AMGParams(smoother=10, presmooth_iter=2, postsmooth_iter=2)
    times, iters = [], 0
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        assert R.setup(ia, ja, val, prm) == 0
        iters, x, _ = R.pcg(b, None, 1e-8, 500, 1)
        t = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(t)
    R.free()
    v = statistics.mean(times)
    line = {"metric": "AMG-PCG time to 1e-8 FP64 relative residual (setup + solve)",
            "value": v, "unit": "s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "iterations": int(iters),
            "config": dict(desc, smoother="l1-Jacobi x2, V(2,2), HEM, coarse direct",
                           parallelism="replicas", l2="inputs larger than L2"),
            "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": kind,
                             "sample": "full workload, one solve per step, 1 thread"},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c5"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        if rank != 0:
            return
        ia, ja, val, b, desc = workload(args.workload)
        run_reference(args, ia, ja, val, b, desc)
        return

    import torch
    import hazmath_b200 as hz
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    ia, ja, val, b, desc = workload(args.workload)
    n, nnz = len(b), int(ia[-1])
    dev = f"cuda:{local}"
    dia, dja = torch.from_numpy(ia).to(dev), torch.from_numpy(ja).to(dev)
    dval, db = torch.from_numpy(val).to(dev), torch.from_numpy(b).to(dev)
    dx = torch.zeros_like(db)
    p = lambda t: t.data_ptr()  # noqa: E731
    bp_mixed = hz.b200_param(precision=hz.HZB_PREC_MIXED, matching=hz.HZB_MATCH_PARALLEL,
                             device=local)
    bp_plain = hz.b200_param(device=local)

    def solve_once(S):
        dx.zero_()
        rc = S.setup_device(n, nnz, p(dia), p(dja), p(dval))
        if rc:
            raise RuntimeError(f"setup failed {rc}: {hz.last_error()}")
        it = S.solve_device(p(db), p(dx))
        if it < 0:
            raise RuntimeError(f"solve failed {it}: {hz.last_error()}")
        return it

    S = hz.Solver(amg_l1(hz), itparam(hz), bp_mixed)
    for _ in range(args.warmup):
        solve_once(S)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    setup_s, solve_s, launches, iters = [], [], 0, 0
    ev0.record()
    for _ in range(args.steps):
        iters = solve_once(S)
        st = S.stats()
        setup_s.append(st.setup_seconds)
        solve_s.append(st.solve_seconds)
        launches += st.launches
    ev1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = ev0.elapsed_time(ev1)
    step_s = total_ms * 1e-3 / args.steps
    if dist:
        t = torch.tensor([step_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_s = float(t.item())
    x = dx.cpu().numpy()
    import scipy.sparse as sp
    A = sp.csr_matrix((val, ja, ia), shape=(n, n))
    relres = float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))

    # plain FP64 drop-in (exact HEM, FP64 V-cycle, same smoother) beside it
    S64 = hz.Solver(amg_l1(hz), itparam(hz), bp_plain)
    solve_once(S64)
    it64 = solve_once(S64)
    st64 = S64.stats()
    x64 = dx.cpu().numpy()
    err_vs_fp64 = float(np.linalg.norm(x - x64) / np.linalg.norm(x64))

    # roofline: level-0 SpMV (FP64 drop-in operator) and FP32 l1 sweep
    peak, peak_kind = hbm_peak()
    ms, by = C.c_double(), C.c_double()
    assert hz.lib().hzb_time_kernel(S64.h, 0, 0, 50, C.byref(ms), C.byref(by)) == 0
    spmv64_gbs = by.value / (ms.value * 1e-3) / 1e9
    spmv64_ms = ms.value
    spmv64_bytes = by.value
    assert hz.lib().hzb_time_kernel(S.h, 3, 0, 50, C.byref(ms), C.byref(by)) == 0
    l1_32_gbs = by.value / (ms.value * 1e-3) / 1e9

    # e2e: the drop-in C entry point with host arrays (mixed form)
    e2e = []
    xb = np.zeros(n)
    amg = amg_l1(hz)
    for k in range(1 + min(args.steps, 3)):
        xb[:] = 0.0
        amg.strong_coupled = 0.0
        t0 = time.perf_counter()
        rc = hz.linear_solver_dcsr_krylov_amg(ia, ja, val, b, xb, itparam(hz), amg, bp_mixed)
        t = time.perf_counter() - t0
        assert rc > 0, (rc, hz.last_error())
        if k:
            e2e.append(t)
    e2e_s = statistics.mean(e2e)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle
        kind = "reference" if oracle.ref_available() else "port"
        R = oracle.ref() if kind == "reference" else oracle.port()
        prm = oracle.AMGParams(smoother=10, presmooth_iter=2, postsmooth_iter=2)
        t0 = time.perf_counter()
        R.setup(ia, ja, val, prm)
        it_ref, _, _ = R.pcg(b, None, 1e-8, 500, 1)
        cpu_t = time.perf_counter() - t0
        R.free()
        cpu = {"value": cpu_t, "unit": "s", "cores": 1, "kind": kind,
               "sample": "one full setup+solve of the workload, single thread",
               "iterations": int(it_ref)}

    if rank == 0:
        line = {
            "metric": "AMG-PCG time to 1e-8 FP64 relative residual (setup + solve)",
            "value": step_s, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-cycle/f64-outer",
            "data": "synthetic",
            "config": dict(desc, solver="UA-AMG (HEM, parallel matching) V(2,2) l1-Jacobi, "
                           "FP32 cycle in FP64 flexible CG", parallelism="replicas",
                           l2="inputs larger than L2 (no flush)"),
            "iterations": int(iters), "final_relres": relres,
            "setup_s": statistics.mean(setup_s), "solve_s": statistics.mean(solve_s),
            "dof_per_s": n / statistics.mean(solve_s),
            "plain_fp64": {"iterations": int(it64), "setup_s": st64.setup_seconds,
                           "solve_s": st64.solve_seconds,
                           "total_s": st64.setup_seconds + st64.solve_seconds},
            "speedup_solve_vs_plain": st64.solve_seconds / statistics.mean(solve_s),
            "err_vs_fp64": err_vs_fp64,
            "roofline": {"bound": "hbm", "kernel": "level-0 SpMV FP64 (row bundles)",
                         "achieved": spmv64_gbs, "peak": peak, "unit": "GB/s",
                         "frac": spmv64_gbs / peak, "peak_kind": peak_kind,
                         "bytes_per_launch": spmv64_bytes, "ms_per_launch": spmv64_ms,
                         "traffic": None},
            "l1_sweep_fp32_gbs": l1_32_gbs,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_s, "unit": "s",
                    "h2d_bytes_per_step": int(ia.nbytes + ja.nbytes + val.nbytes + b.nbytes
                                              + xb.nbytes),
                    "d2h_bytes_per_step": int(xb.nbytes)},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line))
    S.close()
    S64.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
