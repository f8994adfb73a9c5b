"""Level-kernel timing on a workload's hierarchy.

    python -m hazmath_b200.kernel_bench [--case c1|c2|c5] [--cubes N] [--levels 0,1,2]
        [--kernels spmv64,spmv32,res64,l1_32,l1_64,gs64] [--reps 50]
        [--precision mixed|fp64] [--matching parallel|exact] [--smoother l1|gs]
    python -m hazmath_b200.kernel_bench --assemble [--case c2|c5] [--reps 20]

Builds the UA-AMG hierarchy (l1-Jacobi V(2,2) settings, or Gauss-Seidel
V(1,1) with --smoother gs, whose sweep gs64 times on the level schedules) of
the 3D P1 log-normal diffusion problem on the Kuhn mesh of 128^3 (c2,
sigma 1) or 256^3 (c5, sigma 1.5) cubes, or of the 2D 255^2 Poisson problem
(c1) -- or, with --cubes N, of the c5 family (sigma 1.5) on N^3 cubes, a
smaller instance whose levels still exceed the L2 -- then times each
requested kernel on each
requested level with hzb_time_kernel: `reps` back-to-back launches on the
handle's stream between CUDA events, after one warm-up launch.  Prints
achieved GB/s from the kernel's algorithmic bytes and the fraction of the
measured HBM copy bandwidth.  The timed launches are bracketed by
cudaProfilerStart/Stop, so `ncu --profile-from-start off` sees only them.

--assemble times the device assembly of the case's matrix from its per-cube
field instead (hzb_assemble_p1_kuhn_device, `reps` calls between CUDA events):
algorithmic bytes = row pointers, columns and values written + the field read.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os

import numpy as np

from . import (HZB_K_GS64, HZB_K_L1_32, HZB_K_L1_64, HZB_K_RES64, HZB_K_SPMV32, HZB_K_SPMV64,
               HZB_MATCH_EXACT, HZB_MATCH_PARALLEL, HZB_PREC_FP64, HZB_PREC_MIXED,
               SMOOTHER_GS, SMOOTHER_L1DIAG, Solver, b200_param, last_error, lib,
               bench_amg)
from . import problems as P

KERNELS = {"spmv64": HZB_K_SPMV64, "spmv32": HZB_K_SPMV32, "res64": HZB_K_RES64,
           "l1_32": HZB_K_L1_32, "l1_64": HZB_K_L1_64, "gs64": HZB_K_GS64}
CASES = {"c1": None, "c2": (128, 1.0, 2), "c5": (256, 1.5, 7)}
PEAKS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                     "MEASURED_PEAKS.json")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="c2", choices=sorted(CASES))
    ap.add_argument("--levels", default="0,1,2")
    ap.add_argument("--kernels", default="spmv64,spmv32,res64,l1_32,l1_64")
    ap.add_argument("--reps", type=int, default=50)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--matching", default="parallel", choices=["parallel", "exact"])
    ap.add_argument("--assemble", action="store_true")
    ap.add_argument("--smoother", default="l1", choices=["l1", "gs"])
    ap.add_argument("--cubes", type=int, default=0)
    a = ap.parse_args()
    if a.assemble and a.case == "c1":
        ap.error("--assemble times the Kuhn-mesh cases c2 and c5")
    import torch
    if a.assemble:
        return assemble(a, torch)
    if a.case == "c1":
        ia, ja, val = P.poisson2d_5pt(255)
    else:
        N, sigma, seed = CASES[a.case]
        if a.cubes:
            N, sigma, seed = a.cubes, 1.5, 7
        ia, ja, val = P.kuhn3d_p1(N, P.lognormal_field(N, sigma, 8.0, seed))
    n = len(ia) - 1
    dia, dja, dval = (torch.from_numpy(v).cuda() for v in (ia, ja, val))
    amg = bench_amg(smoother=SMOOTHER_L1DIAG, presmooth_iter=2, postsmooth_iter=2) \
        if a.smoother == "l1" else bench_amg(smoother=SMOOTHER_GS)
    prec = HZB_PREC_MIXED if a.precision == "mixed" else HZB_PREC_FP64
    match = HZB_MATCH_PARALLEL if a.matching == "parallel" else HZB_MATCH_EXACT
    S = Solver(amg, None, b200_param(precision=prec, matching=match))
    rc = S.setup_device(n, len(ja), dia.data_ptr(), dja.data_ptr(), dval.data_ptr())
    if rc:
        raise SystemExit(f"setup failed {rc}: {last_error()}")
    peak = hbm_peak()
    st = S.stats()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for lv in (int(x) for x in a.levels.split(",")):
        if lv >= st.num_levels:
            continue
        for name in a.kernels.split(","):
            ms, by = C.c_double(), C.c_double()
            rc = lib().hzb_time_kernel(S.h, KERNELS[name], lv, a.reps, C.byref(ms),
                                       C.byref(by))
            if rc:
                print(f"level {lv} {name}: error {rc} {last_error()}")
                continue
            gbs = by.value / (ms.value * 1e-3) / 1e9
            print(json.dumps({"case": a.case, "level": lv, "rows": int(st.rows[lv]),
                              "nnz": int(st.nnz[lv]), "kernel": name,
                              "us_per_launch": ms.value * 1e3,
                              "bytes_per_launch": by.value, "gbs": gbs,
                              "frac_of_measured_peak": gbs / peak}), flush=True)
    torch.cuda.profiler.stop()
    S.close()


def hbm_peak() -> float:
    try:
        return float(json.load(open(PEAKS))["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def assemble(a, torch):
    from . import assemble_p1_kuhn_device
    N, sigma, seed = CASES[a.case]
    k = torch.from_numpy(P.lognormal_field(N, sigma, 8.0, seed)).cuda()
    m = N - 1
    ia = torch.empty(m ** 3 + 1, dtype=torch.int32, device="cuda")
    rc, nnz = assemble_p1_kuhn_device(N, k.data_ptr(), ia.data_ptr())
    ja = torch.empty(nnz, dtype=torch.int32, device="cuda")
    va = torch.empty(nnz, dtype=torch.float64, device="cuda")
    args = (N, k.data_ptr(), ia.data_ptr(), ja.data_ptr(), va.data_ptr())
    rc = assemble_p1_kuhn_device(*args)[0]   # warm-up
    if rc:
        raise SystemExit(f"assembly failed {rc}: {last_error()}")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.profiler.start()
    e0.record()
    for _ in range(a.reps):
        assemble_p1_kuhn_device(*args)
    e1.record()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    t = e0.elapsed_time(e1) * 1e-3 / a.reps
    by = 4.0 * (m ** 3 + 1) + 12.0 * nnz + 8.0 * N ** 3
    gbs = by / t / 1e9
    print(json.dumps({"case": a.case, "kernel": "assemble_p1_kuhn", "rows": m ** 3, "nnz": nnz,
                      "us_per_call": t * 1e6, "bytes_per_call": by, "gbs": gbs,
                      "frac_of_measured_peak": gbs / hbm_peak()}), flush=True)


if __name__ == "__main__":
    main()
