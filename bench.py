"""Benchmark: UA-AMG-PCG time to a 1e-8 FP64 relative residual on B200,
mixed precision + learned smoother weights against the plain FP64 drop-in.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload c5|c2|c1|c3] [--no-cpu-baseline]

Workload c5 (default): 3D P1 diffusion -div(k grad u) = f on the Kuhn
tetrahedral mesh of 256^3 cubes (255^3 = 16,581,375 dofs, 247,163,083 stored
entries of the 15-point pattern), k = exp(1.5 g) per cube with g a
unit-variance Gaussian field of correlation length 8 cubes (seed 7),
b ~ U[-1,1] (seed 8), x0 = 0.  c2 is the 128^3 instance (sigma 1, seeds
2/3), c1 the 2D 255^2 Poisson problem.  Synthetic, seeded inputs of the
configurations' shapes.

One step = one solve of that system from x0 = 0 to 1e-8 FP64 relative
residual as a user pays for it: UA-AMG setup (parallel matching, Galerkin
products, coarse factorisation) and flexible CG with the FP32 V-cycle
(l1-Jacobi V(2,2)).  `value` is that time with the inputs resident in HBM;
`e2e` is the same through the handle API with host arrays (matrix and
vectors copied in, the solution copied out, all inside the timed region).
Beside it: the plain FP64 drop-in (exact HEM, FP64 cycle, same smoother;
`plain_fp64`, with its level sizes and iterations against the reference's
on the same system), the same step with the learned smoother weights
(network inference, the measured-contraction fallback check, the solve;
`mixed_learned`, with the iterations of uniform weights 0.7 and 1.3, which
bound what per-row weights can change on this problem) and the learned
weights on unseen 1024^2-vertex anisotropic problems of their training
class (`learned_c4`), and the other configurations as short legs on the
same box (`configs`: c1 the 2D FP64 Gauss-Seidel drop-in with the
reference timed beside it, c2 the 128^3 mixed-vs-plain comparison with its
parity and oracle errors, c3 the 512-system batch).  Every level of both
hierarchies is timed
(`levels_mixed`, `levels_fp64`), the solve as a whole against the HBM
roofline from its algorithmic bytes (`solve_roofline`), and both solutions
against the reference's FP64 solve tightened to 1e-12 (`error_vs_oracle`,
from tests/golden/c5_kuhn.npz).  The stored matrix (2.97 GB) is far larger
than the 126 MB L2, so no flush is needed between steps.

Workload bsr: the block (BSR) path, linear_solver_dbsr_krylov_amg's pieces on
the device: problems.block_system of the 64^3-cube Kuhn matrix (sigma 1,
seeds 2/3) with 3 x 3 blocks (250,047 block rows, 750,141 dofs), one step =
amg_setup_ua_bsr (HEM, coarse_dof 100) + CG preconditioned by
precond_dbsr_amg (block Gauss-Seidel V(1,1), coarsest level by GMRES(25)) to
1e-8; the reference's BSR solver on the same system is the CPU baseline.

--variant NAME (workloads c1, c2) times one of the drop-in's other
configurations instead, FP64 as linear_solver_dcsr_krylov_amg runs it: the
W, AMLI, nonlinear AMLI and additive cycles, GMRES / flexible GMRES /
MINRES, smoothed aggregation, VMB aggregation (table VARIANTS); one step =
setup + solve to 1e-8, the reference running the same configuration beside
it.

Workload c3: 512 independent SPD systems (2D/3D anisotropic P1 diffusion,
1k-200k dofs log-uniform, seed 11) solved together (hzb_batch_*); one step
= batch setup + batch solve; reports the batch time and the p50/p99 of the
per-system solve times.

--impl reference times the reference HAZmath implementation (compiled from
its own C sources, single-threaded -- the reference has no threading): on
c5 one measured setup + PCG solve of the full 256^3 system (minutes on one
core, so exactly one is timed whatever --steps asks; the line reports
steps = 1 and steps_requested), on c1/c2 the full workload every step, on
c3 a sample of the systems scaled by the dof count.  The b200 line's
cpu_baseline is a bounded sample (the 128^3 instance, scaled by the dof
ratio).
Multi-GPU: the path does not shard; N ranks run N independent replicas.
"""
from __future__ import annotations

import argparse
import ctypes as C
import datetime
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
METRIC = "AMG-PCG time to 1e-8 FP64 residual: mixed+learned vs plain on B200; SpMV GB/s"


_FIELD = {}   # the per-cube coefficient field of each instance generated, by N


def kuhn_case(N: int, sigma: float, seeds):
    k = P.lognormal_field(N, sigma, 8.0, seeds[0])
    _FIELD[N] = k
    ia, ja, val = P.kuhn3d_p1(N, k)
    b = P.rhs_uniform(len(ia) - 1, seeds[1])
    desc = {"workload": f"3D P1 log-normal diffusion, Kuhn mesh {N}^3 cubes "
                        f"(sigma={sigma}, corr 8 cubes)",
            "dofs": int(len(b)), "nnz": int(ia[-1])}
    return ia, ja, val, b, desc


CASES = {"c5": (256, 1.5, (7, 8)), "c2": (128, 1.0, (2, 3))}


def workload(name: str):
    if name == "c1":
        ia, ja, val = P.poisson2d_5pt(255)
        b = P.rhs_uniform(len(ia) - 1, 1)
        desc = {"workload": "2D P1 Poisson 257^2 vertices (255^2 dofs, 5-pt)",
                "dofs": int(len(b)), "nnz": int(ia[-1])}
        return ia, ja, val, b, desc
    return kuhn_case(*CASES[name])


def cpu_sample(name: str, variant: str = ""):
    """The bounded CPU sample of a workload and its scale to the full one:
    the 128^3 instance of the same family for c5 (about 30 s single-threaded),
    for smoothed aggregation (whose coarse levels fill in) the 127^2 Poisson
    problem for c1 and the 32^3 Kuhn instance for c2, the workload itself
    otherwise."""
    if variant == "sa" and name in ("c1", "c2"):
        if name == "c1":
            ia, ja, val = P.poisson2d_5pt(127)
            b = P.rhs_uniform(len(ia) - 1, 1)
            what = "2D Poisson 127^2 dofs (16,129)"
        else:
            ia, ja, val, b, _ = kuhn_case(32, 1.0, (2, 3))
            what = "the 32^3-cube instance (29,791 dofs)"
        full = 65025 if name == "c1" else 2048383
        scale = full / (len(ia) - 1)
        return ia, ja, val, b, scale, (f"reference setup+solve of {what}, scaled by the "
                                       f"dof ratio {scale:.2f}")
    if name == "c5":
        N, sigma, seeds = CASES["c5"]
        ia, ja, val, b, _ = kuhn_case(128, sigma, seeds)
        return ia, ja, val, b, 16581375 / (len(ia) - 1), \
            "reference setup+solve of the 128^3-cube instance of the same family " \
            "(2,048,383 dofs, sigma 1.5, seeds 7/8), scaled by the dof ratio 8.095"
    ia, ja, val, b, _ = workload(name)
    return ia, ja, val, b, 1.0, "reference setup+solve of the full workload"


class Clocks:
    """nvidia-smi sampler (every 200 ms).  Started before the warm-up steps, so
    that its start-up (NVML initialisation, which can hold up the driver for a
    few hundred ms) falls outside the timed region; mark() records the start
    of the timed region and stop() keeps the samples taken after it (all of
    them when none is, or when the timestamps do not parse)."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.p = None
        self.t_mark = None
        self.path = os.path.join("/tmp", f"hzb_clocks_{os.getpid()}.csv")
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def mark(self):
        self.t_mark = datetime.datetime.now()

    @staticmethod
    def summary(lines, t_mark=None) -> dict:
        rows = []
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) >= 8:
                rows.append(f)
        if t_mark is not None:
            def after(r):
                try:
                    return datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f") >= t_mark
                except ValueError:
                    return True
            timed = [r for r in rows if after(r)]
            rows = timed or rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit()
                else None, "reasons": reasons, "samples": len(rows)}

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        with open(self.path) as fh:
            lines = fh.readlines()
        os.unlink(self.path)
        return self.summary(lines, self.t_mark)


def hbm_peak():
    try:
        return float(json.load(open(PEAKS))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM, "fallback"


def amg_l1(hz):
    return hz.bench_amg(smoother=hz.SMOOTHER_L1DIAG, presmooth_iter=2, postsmooth_iter=2)


def itparam(hz, maxit=500):
    return hz.itsolver_param(linear_itsolver_type=hz.SOLVER_CG,
                             linear_precond_type=hz.PREC_AMG, linear_tol=1e-8,
                             linear_maxit=maxit, linear_stop_type=hz.STOP_REL_RES)


def time_reference(ia, ja, val, b):
    """One setup + PCG solve by the reference compiled from its sources (the
    C restatement if the reference library is absent), single-threaded."""
    import oracle
    kind = "reference" if oracle.ref_available() else "port"
    R = oracle.ref() if kind == "reference" else oracle.port()
    prm = oracle.AMGParams(smoother=10, presmooth_iter=2, postsmooth_iter=2)
    t0 = time.perf_counter()
    assert R.setup(ia, ja, val, prm) == 0
    t1 = time.perf_counter()
    it, _, _ = R.pcg(b, None, 1e-8, 500, 1)
    t = time.perf_counter() - t0
    R.free()
    LAST_REFERENCE.update(setup_s=t1 - t0, solve_s=t - (t1 - t0))
    return t, int(it), kind


LAST_REFERENCE = {}   # setup / solve seconds of the last time_reference call


# --variant: (what, AMG_param fields over bench_amg's setting, Krylov method)
VARIANTS = {
    "v": ("V-cycle, PCG", {}, "pcg"),
    "w": ("W-cycle, PCG", dict(cycle_type=2), "pcg"),
    "amli": ("AMLI cycle of degree 2, PCG", dict(cycle_type=3), "pcg"),
    "nlamli": ("nonlinear AMLI cycle (flexible GMRES on the coarse levels), "
               "flexible GMRES(100)", dict(cycle_type=4), "fgmres"),
    "add": ("additive cycle, flexible GMRES(100)", dict(cycle_type=5), "fgmres"),
    "gmres": ("V-cycle, GMRES(25)", {}, "gmres"),
    "fgmres": ("V-cycle, flexible GMRES(100)", {}, "fgmres"),
    "minres": ("V-cycle, MINRES", {}, "minres"),
    "sa": ("smoothed aggregation, V-cycle, PCG", dict(AMG_type=2), "pcg"),
    "vmb": ("VMB aggregation, V-cycle, PCG", dict(aggregation_type=1), "pcg"),
}
KRYLOV_TYPE = {"pcg": 1, "minres": 2, "gmres": 3, "fgmres": 4}
RESTART = {"gmres": 25, "fgmres": 100}


def variant_metric(name):
    return (f"UA-AMG drop-in, {VARIANTS[name][0]}: time to 1e-8 FP64 residual "
            f"(setup + solve)")


def time_reference_variant(ia, ja, val, b, name):
    """One setup + solve of a variant by the reference compiled from its
    sources, single-threaded."""
    import oracle
    _, over, method = VARIANTS[name]
    R = oracle.ref()
    prm = oracle.AMGParams(amli_degree=2, nl_amli_krylov_type=4, **over)
    t0 = time.perf_counter()
    assert R.setup(ia, ja, val, prm) == 0
    if method == "pcg":
        it = R.pcg(b, None, 1e-8, 500, 1)[0]
    elif method == "minres":
        it = R.minres(b, tol=1e-8, maxit=500)[0]
    else:
        it = R.gmres(b, tol=1e-8, maxit=500, restart=RESTART[method],
                     flexible=method == "fgmres")[0]
    t = time.perf_counter() - t0
    R.free()
    return t, int(it), "reference"


def run_variant(args, rank, world, local, dist):
    import torch
    import hazmath_b200 as hz
    name = args.variant
    what, over, method = VARIANTS[name]
    ia, ja, val, b, desc = workload(args.workload)
    n, nnz = len(b), int(ia[-1])
    dev = f"cuda:{local}"
    dia, dja = torch.from_numpy(ia).to(dev), torch.from_numpy(ja).to(dev)
    dval, db = torch.from_numpy(val).to(dev), torch.from_numpy(b).to(dev)
    dx = torch.zeros_like(db)
    p = lambda t: t.data_ptr()  # noqa: E731
    amg = hz.bench_amg(amli_degree=2, nl_amli_krylov_type=4, **over)
    it_par = hz.itsolver_param(linear_itsolver_type=KRYLOV_TYPE[method],
                               linear_precond_type=hz.PREC_AMG, linear_tol=1e-8,
                               linear_maxit=500, linear_stop_type=hz.STOP_REL_RES,
                               linear_restart=RESTART.get(method, 100))

    def check(rc, what_):
        if rc < 0:
            raise RuntimeError(f"{what_} failed {rc}: {hz.last_error()}")
        return rc

    S = hz.Solver(amg, it_par, hz.b200_param(device=local))

    def step():
        dx.zero_()
        check(S.setup_device(n, nnz, p(dia), p(dja), p(dval)), "setup")
        return check(S.solve_device(p(db), p(dx)), "solve")

    clocks = Clocks(local)
    for _ in range(args.warmup):
        step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    setup_s, solve_s, launches, iters = [], [], 0, 0
    torch.cuda.profiler.start()
    clocks.mark()
    ev0.record()
    for _ in range(args.steps):
        iters = step()
        st = S.stats()
        setup_s.append(st.setup_seconds)
        solve_s.append(st.solve_seconds)
        launches += st.launches
    ev1.record()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    clk = clocks.stop()
    step_s = max_over_ranks(dist, ev0.elapsed_time(ev1) * 1e-3 / args.steps, dev)
    x = dx.cpu().numpy()
    import scipy.sparse as sp
    A = sp.csr_matrix((val, ja, ia), shape=(n, n))
    relres = float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))
    peak, peak_kind = hbm_peak()
    sp_ms, sp_by = S.time_kernel(hz.HZB_K_SPMV64, 0, 50)
    sp_gbs = sp_by / (sp_ms * 1e-3) / 1e9
    Se = hz.Solver(amg, it_par, hz.b200_param(device=local))
    hia, hja, hval, hb = pinned(torch, ia, ja, val, b)
    xh = pinned(torch, np.zeros(n))[0]
    e2e = []
    for k in range(1 + min(args.steps, 3)):
        xh[:] = 0.0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(Se.setup_host(hia, hja, hval), "setup_host")
        check(Se.solve_host(hb, xh), "solve_host")
        if k:
            e2e.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(dist, statistics.mean(e2e), dev)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            sia, sja, sval, sb, scale, sample = cpu_sample(args.workload, name)
            t, it_ref, kind = time_reference_variant(sia, sja, sval, sb, name)
            cpu = {"value": t * scale, "unit": "s", "cores": 1, "kind": kind,
                   "sample": f"{sample} ({it_ref} iterations)"}
    if rank == 0:
        line = {
            "metric": variant_metric(name), "value": step_s, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": dict(desc, variant=name, solver=what, parallelism="replicas",
                           l2="inputs larger than L2 (no flush)" if nnz > 10_000_000
                           else "inputs smaller than L2, resident between steps"),
            "iterations": int(iters), "final_relres": relres,
            "setup_s": statistics.mean(setup_s), "solve_s": statistics.mean(solve_s),
            "roofline": {"bound": "hbm", "kernel": "level-0 FP64 SpMV of the drop-in "
                         "(k_spmv_bundle<double>)", "achieved": sp_gbs, "peak": peak,
                         "unit": "GB/s", "frac": sp_gbs / peak, "peak_kind": peak_kind,
                         "bytes_per_launch": sp_by, "ms_per_launch": sp_ms,
                         "traffic": None},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_s, "unit": "s",
                    "h2d_bytes_per_step": int(ia.nbytes + ja.nbytes + val.nbytes + b.nbytes
                                              + xh.nbytes),
                    "d2h_bytes_per_step": int(xh.nbytes)},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line))
    S.close()
    Se.close()


BSR_NB = 3


def bsr_case(N: int):
    """The block system of the bsr workload on N^3 cubes: (ia, ja, val, b)."""
    kia, kja, kval = P.kuhn3d_p1(N, P.lognormal_field(N, 1.0, 8.0, 2))
    ia, ja, val = P.block_system(kia, kja, kval, BSR_NB, 31)
    return ia, ja, val, P.rhs_uniform((len(ia) - 1) * BSR_NB, 3)


def bsr_amg(hz):
    return hz.bench_amg(coarse_dof=100, coarse_solver=0)


def time_reference_bsr(ia, ja, val, b):
    """One linear_solver_dbsr_krylov_amg (setup + CG) by the reference
    compiled from its sources, single-threaded."""
    import oracle
    R = oracle.ref()
    prm = oracle.AMGParams(coarse_dof=100, coarse_solver=0)
    t0 = time.perf_counter()
    it, _ = R.bsr_krylov_amg(BSR_NB, ia, ja, val, b, 1, tol=1e-8, maxit=500, params=prm)
    return time.perf_counter() - t0, int(it), "reference"


def run_reference(args):
    name = args.workload
    if args.variant:
        import oracle
        if not oracle.ref_available():
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference library (oracle/_ref) was not built"}))
            return
        wia, wja, wval, wb, _ = kuhn_case(12, 1.0, (2, 3))
        sia, sja, sval, sb, scale, sample = cpu_sample(name, args.variant)
        times, iters = [], 0
        for step in range(args.warmup + args.steps):
            if step < args.warmup:   # the same code on a small instance, untimed
                time_reference_variant(wia, wja, wval, wb, args.variant)
                continue
            t, iters, _ = time_reference_variant(sia, sja, sval, sb, args.variant)
            times.append(t * scale)
        v = statistics.mean(times)
        line = {"metric": variant_metric(args.variant), "value": v, "unit": "s",
                "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "iterations": int(iters),
                "config": dict(workload_desc(name), variant=args.variant,
                               solver=VARIANTS[args.variant][0]),
                "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if name == "bsr":
        import oracle
        if not oracle.ref_available():
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference library (oracle/_ref) was not built"}))
            return
        wia, wja, wval, wb = bsr_case(16)
        sia, sja, sval, sb = bsr_case(64)
        times, iters = [], 0
        for step in range(args.warmup + args.steps):
            if step < args.warmup:   # the same code on the 16^3 instance, untimed
                time_reference_bsr(wia, wja, wval, wb)
                continue
            t, iters, _ = time_reference_bsr(sia, sja, sval, sb)
            times.append(t)
        v = statistics.mean(times)
        what = "reference BSR setup+CG of the full workload"
        line = {"metric": "BSR UA-AMG-PCG time to 1e-8 (setup + solve)", "value": v,
                "unit": "s", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "iterations": int(iters), "config": workload_desc("bsr"),
                "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": "reference",
                                 "sample": what},
                "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    if name == "c3":
        systems, _ = P.batch_anisotropic(512, 11)
        rng = np.random.default_rng(5)
        pick = sorted(rng.choice(len(systems), 24, replace=False))
        total = sum(len(s[3]) for s in systems)
        sample = sum(len(systems[k][3]) for k in pick)
        scale = total / sample
        what = (f"reference setup+solve of 24 of the 512 systems one after another "
                f"({sample} of {total} dofs), scaled by the dof ratio {scale:.2f}")
        warm = [systems[pick[0]]]
        work = [systems[k] for k in pick]
    elif name == "c5":
        # the full 256^3 system: one reference solve takes minutes on one
        # core, so exactly one is timed whatever --steps asks for (the line
        # says so: steps = 1, steps_requested = K)
        ia, ja, val, b, desc = workload(name)
        scale, what = 1.0, ("reference setup+solve of the full 256^3 system (16,581,375 dofs), "
                            "measured, one timed solve")
        wia, wja, wval, wb, _ = kuhn_case(48, 1.0, (2, 3))
        warm = [(wia, wja, wval, wb)]
        work = [(ia, ja, val, b)]
    else:
        ia, ja, val, b, scale, what = cpu_sample(name)
        wia, wja, wval, wb, _ = kuhn_case(48, 1.0, (2, 3))
        warm = [(wia, wja, wval, wb)]
        work = [(ia, ja, val, b)]
    timed_steps = 1 if name == "c5" else args.steps
    times, iters, kind = [], 0, "reference"
    for step in range(args.warmup + timed_steps):
        # warm-up steps run the same code on a small instance (untimed)
        batch = warm if step < args.warmup else work
        t = 0.0
        for (ia, ja, val, b) in batch:
            dt, iters, kind = time_reference(ia, ja, val, b)
            t += dt
        if step >= args.warmup:
            times.append(t * scale)
    v = statistics.mean(times)
    desc = workload_desc(name)
    line = {"metric": METRIC if name != "c3" else "batched UA-AMG-PCG: 512 systems, batch time",
            "value": v, "unit": "s", "impl": "reference", "n_gpus": args.gpus,
            "steps": timed_steps, "steps_requested": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "iterations": int(iters),
            "config": dict(desc, smoother="l1-Jacobi V(2,2), HEM, coarse direct, FP64 CG",
                           parallelism="replicas", l2="inputs larger than L2"),
            "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": kind,
                             "sample": what},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    if name != "c3":
        line["setup_s"], line["solve_s"] = LAST_REFERENCE["setup_s"], LAST_REFERENCE["solve_s"]
    print(json.dumps(line))


def workload_desc(name):
    if name == "bsr":
        return {"workload": "block system K (x) B + seeded SPD diagonal blocks, K the 3D P1 "
                            "log-normal diffusion on the Kuhn mesh of 64^3 cubes (sigma 1), "
                            "3 x 3 blocks", "block_rows": 63 ** 3, "dofs": 63 ** 3 * BSR_NB,
                "solver": "amg_setup_ua_bsr (HEM, coarse_dof 100), CG with "
                          "precond_dbsr_amg (block GS V(1,1), GMRES(25) coarsest)"}
    if name == "c3":
        return {"workload": "512 independent 2D/3D anisotropic P1 diffusion systems, "
                            "1k-200k dofs log-uniform (seed 11)"}
    if name == "c1":
        return {"workload": "2D P1 Poisson 257^2 vertices (255^2 dofs, 5-pt)"}
    N, sigma, _ = CASES[name]
    return {"workload": f"3D P1 log-normal diffusion, Kuhn mesh {N}^3 cubes "
                        f"(sigma={sigma}, corr 8 cubes)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c5", choices=["c1", "c2", "c5", "c3", "bsr"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the c1/c2/c3 legs of the default c5 run")
    ap.add_argument("--steps-only", action="store_true",
                    help="run the warm-up and timed steps only, print a short line (for "
                         "launch lists taken under a profiler; not a bench line)")
    ap.add_argument("--variant", default="", choices=[""] + sorted(VARIANTS))
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.variant and args.workload not in ("c1", "c2"):
        ap.error("--variant runs on the c1 and c2 workloads")

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.variant:
            run_variant(args, rank, world, local, dist)
        elif args.workload == "c3":
            run_batch(args, rank, world, local, dist)
        elif args.workload == "bsr":
            run_bsr(args, rank, world, local, dist)
        else:
            run_single(args, rank, world, local, dist)
    finally:
        if dist:
            dist.barrier()
            dist.destroy_process_group()


def pinned(torch, *arrays):
    """Copies of numpy arrays in page-locked host memory (numpy views of
    pinned torch tensors): the host side of the e2e measurement."""
    return [torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in arrays]


def max_over_ranks(dist, v, dev):
    if not dist:
        return v
    import torch
    t = torch.tensor([v], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_single(args, rank, world, local, dist):
    import torch
    import hazmath_b200 as hz
    from hazmath_b200 import learn
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
    gnn = learn.GNN(device=local, weights=learn.WEIGHTS)
    NS_SELECT = 2

    def check(rc, what):
        if rc < 0:
            raise RuntimeError(f"{what} failed {rc}: {hz.last_error()}")
        return rc

    def step(S, learned):
        """setup + (learned weights with fallback) + solve; device seconds
        of each part from the handle's events and a sync around the check"""
        dx.zero_()
        check(S.setup_device(n, nnz, p(dia), p(dja), p(dval)), "setup")
        sel = None
        if learned:
            t0 = time.perf_counter()
            rp, rl, used = gnn.select(S, NS_SELECT, 99)
            sel = {"rho_plain": rp, "rho_learned": rl, "learned_used": used,
                   "select_s": time.perf_counter() - t0}
        it = check(S.solve_device(p(db), p(dx)), "solve")
        return it, sel

    # the headline step: the mixed solve with plain l1-Jacobi weights (the
    # learned weights, which do not reduce this problem's iteration count,
    # are measured beside it below)
    S = hz.Solver(amg_l1(hz), itparam(hz), bp_mixed)
    clocks = Clocks(local)
    for _ in range(args.warmup):
        step(S, False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    setup_s, solve_s, launches, iters = [], [], 0, 0
    torch.cuda.profiler.start()
    clocks.mark()
    ev0.record()
    for _ in range(args.steps):
        iters, _ = step(S, False)
        st = S.stats()
        setup_s.append(st.setup_seconds)
        solve_s.append(st.solve_seconds)
        launches += st.launches
    ev1.record()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    clk = clocks.stop()
    step_s = max_over_ranks(dist, ev0.elapsed_time(ev1) * 1e-3 / args.steps, dev)
    x = dx.cpu().numpy()
    import scipy.sparse as sp
    A = sp.csr_matrix((val, ja, ia), shape=(n, n))
    relres = float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))
    if args.steps_only:   # the timed steps alone (for launch lists under a profiler)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": step_s, "unit": "s",
                              "steps_only": True, "iterations": int(iters),
                              "setup_s": statistics.mean(setup_s),
                              "setup_s_steps": [round(v, 4) for v in setup_s],
                              "solve_s": statistics.mean(solve_s),
                              "final_relres": relres, "config": desc}))
        S.close()
        gnn.close()
        return

    # the same step with the learned weights: network inference and the
    # measured-contraction fallback check, then the solve (one warm-up step,
    # one timed between CUDA events); then the solve with uniform weights,
    # which shows how far any per-row weights can move this problem
    Sl = hz.Solver(amg_l1(hz), itparam(hz), bp_mixed)
    step(Sl, True)
    torch.cuda.synchronize()
    ev0.record()
    it_l, sel = step(Sl, True)
    ev1.record()
    torch.cuda.synchronize()
    st_l = Sl.stats()
    learned = dict(sel, ns=NS_SELECT, step_s=ev0.elapsed_time(ev1) * 1e-3,
                   iterations=int(it_l), setup_s=st_l.setup_seconds,
                   solve_s=st_l.solve_seconds)
    om = torch.empty(n, dtype=torch.float32, device=dev)
    uniform = {}
    for w in (0.7, 1.3):
        om.fill_(w)
        check(Sl.set_omega_device(p(om)), "set_omega")
        dx.zero_()
        uniform[str(w)] = int(check(Sl.solve_device(p(db), p(dx)), "solve"))
    check(Sl.set_omega_device(None), "set_omega")
    learned["iterations_uniform_omega"] = uniform
    del om
    c4 = c4_leg(gnn, local)
    legs = config_legs(local) if args.workload == "c5" and not args.no_legs else None

    # plain FP64 drop-in (exact HEM, FP64 V-cycle, same smoother) beside it
    S64 = hz.Solver(amg_l1(hz), itparam(hz), bp_plain)
    step(S64, False)
    it64 = step(S64, False)[0]
    st64 = S64.stats()
    x64 = dx.cpu().numpy()
    err_vs_fp64 = float(np.linalg.norm(x - x64) / np.linalg.norm(x64))
    total64 = st64.setup_seconds + st64.solve_seconds

    # roofline of the step's dominant kernel (the level-0 FP32 l1-Jacobi
    # sweep, with the weights the step ran) and of the drop-in's level-0 FP64
    # SpMV (the level SpMV the 70 % target names): each timed as 50 launches
    # on the solver's stream between CUDA events; then every level of both
    # hierarchies, and the solve-level figure
    peak, peak_kind = hbm_peak()

    def kernel(h, which, level=0, reps=50):
        ms, by = C.c_double(), C.c_double()
        check(hz.lib().hzb_time_kernel(h, which, level, reps, C.byref(ms), C.byref(by)),
              "time_kernel")
        return ms.value, by.value, by.value / (ms.value * 1e-3) / 1e9

    l1_ms, l1_by, l1_gbs = kernel(S.h, hz.HZB_K_L1_32)
    sp_ms, sp_by, spmv64_gbs = kernel(S64.h, hz.HZB_K_SPMV64)
    spmv32_gbs = kernel(S.h, hz.HZB_K_SPMV32)[2]
    lv_mixed = level_table(S, kernel, hz.HZB_K_L1_32, peak, mixed=True)
    lv_fp64 = level_table(S64, kernel, hz.HZB_K_SPMV64, peak, mixed=False)
    solve_by = solve_bytes_mixed(lv_mixed, int(iters), False)
    oracle_err = oracle_errors(args.workload, x, x64)

    # device assembly of the same matrix from the per-cube coefficients
    asm = assembly_leg(hz, torch, args.workload, dja, dval, n, nnz, dev, peak) \
        if args.workload in CASES else None

    # e2e: the handle API with host arrays in pinned memory (copies in and out
    # inside the region)
    Se = hz.Solver(amg_l1(hz), itparam(hz), bp_mixed)
    hia, hja, hval, hb = pinned(torch, ia, ja, val, b)
    xh = pinned(torch, np.zeros(n))[0]
    e2e = []
    for k in range(1 + min(args.steps, 3)):
        xh[:] = 0.0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(Se.setup_host(hia, hja, hval), "setup_host")
        check(Se.solve_host(hb, xh), "solve_host")
        t = time.perf_counter() - t0
        if k:
            e2e.append(t)
    e2e_s = max_over_ranks(dist, statistics.mean(e2e), dev)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        sia, sja, sval, sb, scale, what = cpu_sample(args.workload)
        t, it_ref, kind = time_reference(sia, sja, sval, sb)
        cpu = {"value": t * scale, "unit": "s", "cores": 1, "kind": kind, "sample": what,
               "sample_seconds": t, "sample_iterations": it_ref}

    if rank == 0:
        solve_ml = statistics.mean(solve_s)
        line = {
            "metric": METRIC, "value": step_s, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32-cycle/f64-outer", "data": "synthetic",
            "config": dict(desc, solver="UA-AMG (parallel matching) V(2,2) l1-Jacobi, FP32 "
                           "cycle in FP64 flexible CG; the learned weights with their "
                           "fallback check are timed beside it (mixed_learned)",
                           parallelism="replicas", l2="inputs larger than L2 (no flush)"),
            "iterations": int(iters), "final_relres": relres,
            "setup_s": statistics.mean(setup_s),
            "setup_s_steps": [round(v, 4) for v in setup_s],
            "solve_s": solve_ml, "dof_per_s": n / solve_ml,
            "mixed_learned": learned,
            "learned_c4": c4,
            "configs": legs,
            "plain_fp64": {"iterations": int(it64), "setup_s": st64.setup_seconds,
                           "solve_s": st64.solve_seconds, "total_s": total64,
                           "parity": parity_vs_fixture(args.workload, st64, it64)},
            "speedup_vs_plain": total64 / step_s,
            "speedup_solve_vs_plain": st64.solve_seconds / solve_ml,
            "err_vs_fp64": err_vs_fp64,
            "roofline": {"bound": "hbm", "kernel": "level-0 FP32 l1-Jacobi sweep of the "
                         "mixed cycle (k_l1_sell / k_l1_vec / k_l1_bundle<float>, autotuned), "
                         "with the weights the step ran", "achieved": l1_gbs, "peak": peak,
                         "unit": "GB/s", "frac": l1_gbs / peak, "peak_kind": peak_kind,
                         "bytes_per_launch": l1_by, "ms_per_launch": l1_ms,
                         "traffic": TRAFFIC_PER_BYTE["l1_32"] * l1_by,
                         "traffic_source": "ncu DRAM bytes per algorithmic byte of the "
                         "sliced-ELL sweep (level 1 of the 192^3 instance), times this "
                         "launch's bytes"},
            "solve_roofline": {"bound": "hbm", "bytes": solve_by,
                               "seconds": solve_ml, "achieved": solve_by / solve_ml / 1e9,
                               "peak": peak, "unit": "GB/s",
                               "frac": solve_by / solve_ml / 1e9 / peak,
                               "model": "per V-cycle and level: first sweep from x = 0 "
                               "(12n), 3 l1 sweeps (8 nnz32 + 4(n+1) + 12n [+4n weights]), "
                               "residual (8 nnz32 + 4(n+1) + 12n), restriction (4(nc+1) + "
                               "8n + 4nc), prolongation (12n + 4nc); coarsest 8 nc^2 + 8 nc; "
                               "per iteration the FP64 SpMV with its dot (12 nnz + 4(n+1) "
                               "+ 16n) and 112n of flexible-CG vector work and precision "
                               "conversions; iterations + 1 cycles, 2 extra residuals"},
            "levels_mixed": lv_mixed,
            "levels_fp64": lv_fp64,
            "error_vs_oracle": oracle_err,
            "drop_in_spmv64": {"kernel": "level-0 FP64 SpMV of the drop-in "
                               "(k_spmv_bundle<double>)", "achieved": spmv64_gbs,
                               "peak": peak, "unit": "GB/s", "frac": spmv64_gbs / peak,
                               "bytes_per_launch": sp_by, "ms_per_launch": sp_ms,
                               "traffic": TRAFFIC_PER_BYTE["spmv64"] * sp_by},
            "spmv_fp32_gbs": spmv32_gbs,
            "assembly": asm,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_s, "unit": "s",
                    "h2d_bytes_per_step": int(ia.nbytes + ja.nbytes + val.nbytes + b.nbytes
                                              + xh.nbytes),
                    "d2h_bytes_per_step": int(xh.nbytes)},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line))
    for h in (S, Sl, S64, Se):
        h.close()
    gnn.close()


def assembly_leg(hz, torch, name, dja, dval, n, nnz, dev, peak):
    """hzb_assemble_p1_kuhn_device on the workload's per-cube field (resident
    in HBM): device seconds per call (row counts, scan, entries) between CUDA
    events, its bytes (row pointers, columns and values written, field read)
    against the HBM peak, and whether it reproduced the generator's arrays."""
    N = CASES[name][0]
    kd = torch.from_numpy(_FIELD[N]).to(dev)
    ia = torch.empty(n + 1, dtype=torch.int32, device=dev)
    ja = torch.empty(nnz, dtype=torch.int32, device=dev)
    va = torch.empty(nnz, dtype=torch.float64, device=dev)
    ptrs = (kd.data_ptr(), ia.data_ptr(), ja.data_ptr(), va.data_ptr())

    def call():
        rc, got = hz.assemble_p1_kuhn_device(N, *ptrs)
        if rc < 0 or got != nnz:
            raise RuntimeError(f"assembly failed {rc}: {hz.last_error()}")

    call()
    same = bool(torch.equal(ja, dja)) and bool(torch.equal(va.view(torch.int64),
                                                           dval.view(torch.int64)))
    reps = 5
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        call()
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) * 1e-3 / reps
    by = 4.0 * (n + 1) + 12.0 * nnz + 8.0 * N ** 3
    out = {"kernel": "hzb_assemble_p1_kuhn_device (one k_kuhn_fill launch)",
           "seconds": t, "bytes": by, "achieved": by / t / 1e9, "peak": peak, "unit": "GB/s",
           "frac": by / t / 1e9 / peak, "matches_host_generator": same}
    del kd, ia, ja, va
    return out


def _timed_steps(torch, step, steps):
    """steps calls of step() between CUDA events after one warm-up call:
    seconds per call and the last call's result."""
    step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        out = step()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / steps, out


def config_legs(device, steps=3):
    """The other configurations of the benchmark, each as its own short leg
    of the default run (same clock and box as the headline):
    c1 -- the FP64 drop-in as configured there (2D 255^2 Poisson, HEM, GS
          V(1,1), PCG), with the reference timed on the same system;
    c2 -- the 128^3 Kuhn system (sigma 1): mixed solve against the FP64
          drop-in, the drop-in's level sizes and iterations against the
          reference's, both errors against the reference's 1e-12 solve;
    c3 -- 512 independent systems (~20M dofs) solved as one batch."""
    import torch
    import hazmath_b200 as hz
    dev = f"cuda:{device}"
    p = lambda t: t.data_ptr()  # noqa: E731
    out = {}

    def up(*arrs):
        return [torch.from_numpy(a).to(dev) for a in arrs]

    # c1
    ia, ja, val, b, _ = workload("c1")
    dia, dja, dval, db = up(ia, ja, val, b)
    dx = torch.zeros_like(db)
    S = hz.Solver(hz.bench_amg(), itparam(hz), hz.b200_param(device=device))

    def c1_step():
        dx.zero_()
        assert S.setup_device(len(b), len(ja), p(dia), p(dja), p(dval)) == 0, hz.last_error()
        return S.solve_device(p(db), p(dx))

    t, it = _timed_steps(torch, c1_step, steps)
    st = S.stats()
    S.close()
    leg = {"workload": "2D P1 Poisson 257^2 vertices (65,025 dofs), FP64 drop-in, HEM, GS "
                       "V(1,1), coarse direct, PCG to 1e-8", "step_s": t, "iterations": int(it),
           "setup_s": st.setup_seconds, "solve_s": st.solve_seconds, "steps": steps}
    import oracle
    if oracle.ref_available():
        tr, itr, _ = time_reference_variant(ia, ja, val, b, "v")
        leg["reference"] = {"step_s": tr, "iterations": itr, "cores": 1,
                            "kind": "reference", "measured": "this run, this host"}
    out["c1"] = leg
    del dia, dja, dval, db, dx

    # c2
    ia, ja, val, b, _ = workload("c2")
    n = len(b)
    dia, dja, dval, db = up(ia, ja, val, b)
    dx = torch.zeros_like(db)
    leg = {"workload": "3D P1 log-normal diffusion, Kuhn mesh 128^3 cubes (sigma 1; "
                       "2,048,383 dofs), l1-Jacobi V(2,2), to 1e-8", "steps": steps}
    for tag, bp in (("mixed", hz.b200_param(precision=hz.HZB_PREC_MIXED,
                                            matching=hz.HZB_MATCH_PARALLEL, device=device)),
                    ("plain_fp64", hz.b200_param(device=device))):
        S = hz.Solver(amg_l1(hz), itparam(hz), bp)

        def c2_step():
            dx.zero_()
            assert S.setup_device(n, len(ja), p(dia), p(dja), p(dval)) == 0, hz.last_error()
            return S.solve_device(p(db), p(dx))

        t, it = _timed_steps(torch, c2_step, steps if tag == "mixed" else 1)
        st = S.stats()
        x = dx.cpu().numpy()
        leg[tag] = {"step_s": t, "iterations": int(it), "setup_s": st.setup_seconds,
                    "solve_s": st.solve_seconds}
        if tag == "plain_fp64":
            leg[tag]["parity"] = parity_vs_fixture("c2", st, it)
        g = fixture("c2")
        if g is not None:
            xt = g["l1/tight/x_sample"]
            leg[tag]["error_vs_oracle"] = float(np.linalg.norm(x[::int(g["stride"])] - xt)
                                                / np.linalg.norm(xt))
        S.close()
    leg["speedup_vs_plain"] = leg["plain_fp64"]["step_s"] / leg["mixed"]["step_s"]
    leg["speedup_solve_vs_plain"] = leg["plain_fp64"]["solve_s"] / leg["mixed"]["solve_s"]
    g = fixture("c2")
    if g is not None:
        leg["reference_recorded"] = {"setup_s": float(g["l1/seconds"][0]),
                                     "solve_s": float(g["l1/seconds"][1]), "cores": 1,
                                     "measured": "tests/golden/make_golden.py, build container"}
    out["c2"] = leg
    del dia, dja, dval, db, dx

    # c3
    systems, (off, ia, ja, val, b) = P.batch_anisotropic(512, 11)
    dia, dja, dval, db = up(ia, ja, val, b)
    dx = torch.zeros_like(db)
    bp = hz.b200_param(precision=hz.HZB_PREC_MIXED, matching=hz.HZB_MATCH_PARALLEL,
                       device=device)
    S = hz.Solver(amg_l1(hz), itparam(hz, 1000), bp)

    def c3_step():
        dx.zero_()
        assert S.batch_setup_device(off, int(ia[-1]), p(dia), p(dja), p(dval)) == 0
        rc, its, rel, sec = S.batch_solve_device(p(db), p(dx))
        assert rc > 0, hz.last_error()
        return its, rel, sec

    t, (its, rel, sec) = _timed_steps(torch, c3_step, steps)
    out["c3"] = {"workload": "512 independent 2D/3D anisotropic P1 systems, 1k-200k dofs "
                             f"log-uniform (seed 11), {len(b)} dofs", "batch_s": t,
                 "steps": steps, "per_system_solve_s": {
                     "p50": float(np.percentile(sec, 50)), "p99": float(np.percentile(sec, 99))},
                 "iterations": {"p50": float(np.percentile(its, 50)), "max": int(its.max())},
                 "worst_relres": float(rel.max())}
    S.close()
    return out


def c4_leg(gnn, device, count=4):
    """The learned weights on unseen problems of their training class: 2D
    anisotropic P1 diffusion on 1024^2-vertex meshes (epsilon log-uniform in
    [1e-4, 1], random rotation; learn.eval_problem, seed 20260), plain
    l1-Jacobi weights against the learned ones with their fallback check, in
    the mixed solve to 1e-8: iterations, solve and selection seconds."""
    from hazmath_b200 import learn
    rng = np.random.default_rng(20260)
    rows = learn.evaluate(gnn, [learn.eval_problem(rng) for _ in range(count)],
                          device=device, ns=2)
    keep = ("eps", "angle", "dofs", "plain_iters", "learned_iters", "plain_solve_s",
            "learned_solve_s", "select_s", "learned_used", "rho_plain", "rho_learned")
    rows = [{k: r[k] for k in keep} for r in rows]
    return {"problems": rows,
            "plain_iters": sum(r["plain_iters"] for r in rows),
            "learned_iters": sum(r["learned_iters"] for r in rows),
            "plain_solve_s": sum(r["plain_solve_s"] for r in rows),
            "learned_solve_plus_select_s": sum(r["learned_solve_s"] + r["select_s"]
                                               for r in rows)}


def level_table(S, kernel, which, peak, mixed):
    """Per level of a hierarchy: rows, stored entries (the FP32 copy's,
    without exact zeros, for the mixed cycle), and the GB/s of its l1 sweep
    (mixed) or FP64 SpMV (drop-in) against the HBM peak; levels whose data
    fit twice into the 126 MB L2 are marked (they run from L2)."""
    st = S.stats()
    out = []
    for l in range(st.num_levels):
        n = st.rows[l]
        if mixed and l == st.num_levels - 1:
            out.append({"level": l, "rows": n, "coarsest": True})
            break
        reps = 50 if n > 100000 else 200
        ms, by, gbs = kernel(S.h, which, l, reps)
        sp_by = kernel(S.h, hz_const("HZB_K_SPMV32"), l, 1)[1] if mixed else None
        row = {"level": l, "rows": n, "nnz": st.nnz[l], "bytes": by, "ms": ms, "gbs": gbs,
               "frac": gbs / peak, "l2_resident": by < 63e6}
        if mixed:
            row["nnz32"] = int(round((sp_by - 4.0 * (n + 1) - 8.0 * n) / 8.0))
        out.append(row)
    return out


def hz_const(name):
    import hazmath_b200 as hz
    return getattr(hz, name)


def solve_bytes_mixed(levels, iters, omega):
    """Algorithmic bytes of one mixed solve (FP64 flexible CG around the
    FP32 V(2,2) l1-Jacobi cycle) from the level sizes; the terms are listed
    in the bench line's solve_roofline.model."""
    n0, nnz0 = levels[0]["rows"], levels[0]["nnz"]
    outer = 12.0 * nnz0 + 4.0 * (n0 + 1) + 16.0 * n0 + 112.0 * n0
    cyc = 0.0
    for l in range(len(levels) - 1):
        n, nz, nc = levels[l]["rows"], levels[l]["nnz32"], levels[l + 1]["rows"]
        w = 4.0 * n if (omega and l == 0) else 0.0
        sweep = 8.0 * nz + 4.0 * (n + 1) + 12.0 * n + w
        first = 12.0 * n + w
        res = 8.0 * nz + 4.0 * (n + 1) + 12.0 * n
        restr = 4.0 * (nc + 1) + 8.0 * n + 4.0 * nc
        prol = 12.0 * n + 4.0 * nc
        cyc += first + 3.0 * sweep + res + restr + prol
    nc = levels[-1]["rows"]
    cyc += 8.0 * nc * nc + 8.0 * nc
    res0 = 12.0 * nnz0 + 4.0 * (n0 + 1) + 24.0 * n0
    return iters * outer + (iters + 1) * cyc + 2.0 * res0


def fixture(name):
    path = os.path.join(ROOT, "tests", "golden", f"{name}_kuhn.npz")
    return np.load(path) if os.path.exists(path) else None


def oracle_errors(name, x_mixed, x_fp64):
    """Errors of the mixed and of the FP64 (1e-8) solutions against the
    reference's FP64 solve tightened to 1e-12 (a strided sample of it,
    recorded by tests/golden/make_golden.py)."""
    g = fixture(name)
    if g is None:
        return None
    st = int(g["stride"])
    xt = g["l1/tight/x_sample"]
    nt = np.linalg.norm(xt)
    return {"mixed": float(np.linalg.norm(x_mixed[::st] - xt) / nt),
            "plain_fp64": float(np.linalg.norm(x_fp64[::st] - xt) / nt),
            "oracle": f"reference FP64 PCG to 1e-12 ({int(g['l1/tight/iters'])} iterations), "
                      f"every {st}th entry ({len(xt)} entries)"}


def parity_vs_fixture(name, st, iters):
    """The drop-in's level sizes and PCG iterations against the reference's
    on the same system (the full digests are compared by the GPU tests)."""
    g = fixture(name)
    if g is None:
        return None
    info = g["l1/info"]
    sizes = [(st.rows[l], st.nnz[l]) for l in range(st.num_levels)]
    return {"levels_equal": sizes == [(int(r[0]), int(r[1])) for r in info],
            "iterations": int(iters), "reference_iterations": int(g["l1/iters"]),
            "theta_equal": st.strong_coupled == float(g["l1/theta_after"])}


# DRAM bytes (read + written) per algorithmic byte of one launch, measured by
# ncu over the bytes hzb_time_kernel counts: the FP32 l1-Jacobi sweep in the
# sliced-ELL schedule the autotuner picks on the fine levels (level 1 of the
# 192^3 instance of the family: dram__bytes.sum.per_second 4.804 TB/s over
# 68.288 us = 328.1 MB for 311,596,604 algorithmic bytes), and the drop-in's
# FP64 SpMV on level 0 of the 128^3 case.  The 256^3 launches run the same
# kernels over more entries, and their traffic is this ratio times their
# algorithmic bytes.
TRAFFIC_PER_BYTE = {"l1_32": 4.804461e12 * 68.288e-6 / 311596604.0,
                    "spmv64": 404.52e6 / 405049716.0}


def run_bsr(args, rank, world, local, dist):
    import torch
    import hazmath_b200 as hz
    ia, ja, val, b = bsr_case(64)
    nrow, nnzb, n = len(ia) - 1, int(ia[-1]), len(b)
    dev = f"cuda:{local}"
    dia, dja = torch.from_numpy(ia).to(dev), torch.from_numpy(ja).to(dev)
    dval, db = torch.from_numpy(val).to(dev), torch.from_numpy(b).to(dev)
    dx = torch.zeros_like(db)
    p = lambda t: t.data_ptr()  # noqa: E731
    it_par = itparam(hz)
    S = hz.Solver(bsr_amg(hz), it_par, hz.b200_param(device=local))

    def check(rc, what):
        if rc < 0:
            raise RuntimeError(f"{what} failed {rc}: {hz.last_error()}")
        return rc

    def step():
        dx.zero_()
        check(S.setup_bsr_device(nrow, nnzb, BSR_NB, p(dia), p(dja), p(dval)), "bsr setup")
        return check(S.bsr_solve_device(p(db), p(dx)), "bsr solve")

    clocks = Clocks(local)
    for _ in range(args.warmup):
        step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    setup_s, solve_s, launches, iters = [], [], 0, 0
    clocks.mark()
    ev0.record()
    for _ in range(args.steps):
        iters = step()
        st = S.stats()
        setup_s.append(st.setup_seconds)
        solve_s.append(st.solve_seconds)
        launches += st.launches
    ev1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    step_s = max_over_ranks(dist, ev0.elapsed_time(ev1) * 1e-3 / args.steps, dev)
    x = dx.cpu().numpy()
    import scipy.sparse as sp
    sia, sja, sval = P.bsr_to_csr(ia, ja, val, BSR_NB)
    A = sp.csr_matrix((sval, sja, sia), shape=(n, n))
    relres = float(np.linalg.norm(b - A @ x) / np.linalg.norm(b))
    peak, peak_kind = hbm_peak()
    gs_ms, gs_by = S.time_kernel(hz.HZB_K_BSR_GS, 0, 20)
    res_ms, res_by = S.time_kernel(hz.HZB_K_BSR_RES, 0, 50)
    gs_gbs = gs_by / (gs_ms * 1e-3) / 1e9
    res_gbs = res_by / (res_ms * 1e-3) / 1e9
    # e2e through the host entry points (matrix and vectors copied in, the
    # solution out, inside the timed region)
    Se = hz.Solver(bsr_amg(hz), it_par, hz.b200_param(device=local))
    xh = np.zeros(n)
    e2e = []
    for k in range(1 + min(args.steps, 3)):
        xh[:] = 0.0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(Se.setup_bsr_host(BSR_NB, ia, ja, val), "bsr setup_host")
        check(Se.bsr_solve_host(b, xh), "bsr solve_host")
        if k:
            e2e.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(dist, statistics.mean(e2e), dev)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            t, it_ref, kind = time_reference_bsr(ia, ja, val, b)
            cpu = {"value": t, "unit": "s", "cores": 1, "kind": kind,
                   "sample": f"reference BSR setup+CG of the full workload "
                             f"({it_ref} iterations)"}
    if rank == 0:
        line = {
            "metric": "BSR UA-AMG-PCG time to 1e-8 (setup + solve)", "value": step_s,
            "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_desc("bsr"), nnz_blocks=nnzb, parallelism="replicas",
                           l2="inputs larger than L2 (no flush)"),
            "iterations": int(iters), "final_relres": relres,
            "setup_s": statistics.mean(setup_s), "solve_s": statistics.mean(solve_s),
            "dof_per_s": n / statistics.mean(solve_s),
            "roofline": {"bound": "hbm", "kernel": "level-0 ascending block Gauss-Seidel "
                         "sweep (k_bsr_gs_set<3> / k_bsr_gs_run<3> over the level sets)",
                         "achieved": gs_gbs, "peak": peak, "unit": "GB/s",
                         "frac": gs_gbs / peak, "peak_kind": peak_kind,
                         "bytes_per_launch": gs_by, "ms_per_launch": gs_ms, "traffic": None},
            "block_residual": {"kernel": "k_bsr_residual<3>, level 0", "achieved": res_gbs,
                               "frac": res_gbs / peak, "bytes_per_launch": res_by,
                               "ms_per_launch": res_ms},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_s, "unit": "s",
                    "h2d_bytes_per_step": int(ia.nbytes + ja.nbytes + val.nbytes + b.nbytes
                                              + xh.nbytes),
                    "d2h_bytes_per_step": int(xh.nbytes)},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line))
    S.close()
    Se.close()


def run_batch(args, rank, world, local, dist):
    import torch
    import hazmath_b200 as hz
    systems, (off, ia, ja, val, b) = P.batch_anisotropic(512, 11)
    n, nnz = len(b), int(ia[-1])
    dev = f"cuda:{local}"
    dia, dja = torch.from_numpy(ia).to(dev), torch.from_numpy(ja).to(dev)
    dval, db = torch.from_numpy(val).to(dev), torch.from_numpy(b).to(dev)
    dx = torch.zeros_like(db)
    p = lambda t: t.data_ptr()  # noqa: E731
    bp = hz.b200_param(precision=hz.HZB_PREC_MIXED, matching=hz.HZB_MATCH_PARALLEL,
                       device=local)
    S = hz.Solver(amg_l1(hz), itparam(hz, 1000), bp)

    def step():
        dx.zero_()
        rc = S.batch_setup_device(off, nnz, p(dia), p(dja), p(dval))
        if rc:
            raise RuntimeError(f"batch setup {rc}: {hz.last_error()}")
        su = S.stats().setup_seconds
        rc, its, rel, sec = S.batch_solve_device(p(db), p(dx))
        if rc < 0:
            raise RuntimeError(f"batch solve {rc}: {hz.last_error()}")
        return su, S.stats().solve_seconds, its, rel, sec

    clocks = Clocks(local)
    for _ in range(args.warmup):
        step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res = []
    launches = 0
    torch.cuda.profiler.start()
    clocks.mark()
    ev0.record()
    for _ in range(args.steps):
        res.append(step())
        launches += S.stats().launches
    ev1.record()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    clk = clocks.stop()
    step_s = max_over_ranks(dist, ev0.elapsed_time(ev1) * 1e-3 / args.steps, dev)
    su, so, its, rel, sec = res[-1]
    x = dx.cpu().numpy()
    import scipy.sparse as sp
    worst = 0.0
    for k, (sia, sja, sval, sb) in enumerate(systems):
        A = sp.csr_matrix((sval, sja, sia))
        xk = x[off[k]:off[k + 1]]
        worst = max(worst, float(np.linalg.norm(sb - A @ xk) / np.linalg.norm(sb)))
    peak, peak_kind = hbm_peak()
    ms, by = C.c_double(), C.c_double()
    rc = hz.lib().hzb_time_kernel(S.h, hz.HZB_K_L1_32, 0, 50, C.byref(ms), C.byref(by))
    l1_gbs = by.value / (ms.value * 1e-3) / 1e9 if rc == 0 else None
    rc = hz.lib().hzb_time_kernel(S.h, hz.HZB_K_SPMV64, 0, 50, C.byref(ms), C.byref(by))
    spmv_gbs = by.value / (ms.value * 1e-3) / 1e9 if rc == 0 else None
    # e2e through the API with host arrays: upload, batch setup + solve, download
    e2e = []
    xh = np.zeros(n)
    for k in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tia, tja = torch.from_numpy(ia).to(dev), torch.from_numpy(ja).to(dev)
        tval, tb = torch.from_numpy(val).to(dev), torch.from_numpy(b).to(dev)
        tx = torch.zeros_like(tb)
        S.batch_setup_device(off, nnz, p(tia), p(tja), p(tval))
        S.batch_solve_device(p(tb), p(tx))
        xh[:] = tx.cpu().numpy()
        e2e.append(time.perf_counter() - t0)
        del tia, tja, tval, tb, tx
    e2e_s = max_over_ranks(dist, e2e[-1], dev)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        rng = np.random.default_rng(5)
        pick = sorted(rng.choice(len(systems), 24, replace=False))
        t, kind = 0.0, "reference"
        for k in pick:
            dt, _, kind = time_reference(*systems[k])
            t += dt
        sample = sum(len(systems[k][3]) for k in pick)
        scale = n / sample
        cpu = {"value": t * scale, "unit": "s", "cores": 1, "kind": kind,
               "sample": f"reference setup+solve of 24 of the 512 systems one after another "
                         f"({sample} of {n} dofs, {t:.1f} s), scaled by the dof ratio "
                         f"{scale:.2f}"}
    if rank == 0:
        line = {
            "metric": "batched UA-AMG-PCG: 512 systems, batch time", "value": step_s,
            "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32-cycle/f64-outer", "data": "synthetic",
            "config": dict(workload_desc("c3"), systems=len(systems), dofs=n, nnz=nnz,
                           solver="one union hierarchy (parallel matching), per-system "
                           "flexible CG, FP32 V(2,2) l1-Jacobi", parallelism="replicas",
                           l2="inputs larger than L2 (no flush)"),
            "setup_s": su, "solve_s": so,
            "per_system_solve_s": {"p50": float(np.percentile(sec, 50)),
                                   "p99": float(np.percentile(sec, 99)),
                                   "max": float(sec.max())},
            "iterations": {"p50": float(np.percentile(its, 50)),
                           "p99": float(np.percentile(its, 99)), "max": int(its.max())},
            "worst_true_relres": worst,
            "roofline": {"bound": "hbm", "kernel": "level-0 FP32 l1-Jacobi sweep of the union",
                         "achieved": l1_gbs, "peak": peak, "unit": "GB/s",
                         "frac": (l1_gbs / peak) if l1_gbs else None, "peak_kind": peak_kind,
                         "traffic": None},
            "spmv_fp64_gbs": spmv_gbs,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_s, "unit": "s",
                    "h2d_bytes_per_step": int(ia.nbytes + ja.nbytes + val.nbytes + b.nbytes),
                    "d2h_bytes_per_step": int(xh.nbytes)},
            "gpu_launches": int(launches), "clocks": clk,
        }
        print(json.dumps(line))
    S.close()


if __name__ == "__main__":
    main()
