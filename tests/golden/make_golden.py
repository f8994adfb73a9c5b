"""Generate the golden fixtures of tests/golden/ from the reference itself.

    python tests/golden/make_golden.py [REFERENCE_DIR] [--only gmres|cycles|cube|minres|sa|bsr|vmb|hec|layout|c2|c5|batch]

Runs the reference HAZmath library compiled from its own sources
(oracle/build_ref.sh -> oracle/_ref/libhazref.so) on seeded synthetic inputs
and on the reference's only shipped known-answer case for this path
(examples/solvers/A.dat + b.dat: 128x128 5-point Laplacian), and stores its
outputs: hierarchy sizes, aggregate maps, coarse operators (full arrays for
small cases, SHA-256 digests for large ones), PCG iteration counts, residual
histories and solutions, smoother outputs, the RAP product, and the struct
layout of the reference headers.  The fixtures let the CPU tests pin the
C restatement (oracle/hzoracle.c) without the reference present, and the GPU
tests compare the CUDA path against the same numbers.
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from hazmath_b200 import problems as P  # noqa: E402

ARGS = [a for i, a in enumerate(sys.argv[1:], 1)
        if a != "--only" and sys.argv[i - 1] != "--only"]
REF = ARGS[0] if ARGS else os.environ.get("HAZ_REF", "")
if not os.path.isdir(os.path.join(REF, "src")):
    sys.exit("make_golden.py: give the reference's source tree as REFERENCE_DIR or $HAZ_REF")


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def hierarchy(R, ia, ja, val, params, full: bool):
    st = R.setup(ia, ja, val, params)
    assert st == 0, st
    nl = R.num_levels()
    info = np.array([R.level_info(l)[:3] for l in range(nl)], np.int64)
    out = {"info": info, "theta_after": np.float64(R.strong_coupled())}
    for l in range(nl):
        A = R.level_A(l)
        if full:
            out[f"A{l}_ia"], out[f"A{l}_ja"], out[f"A{l}_val"] = A
        else:
            out[f"A{l}_sha"] = np.array([sha(A[0]), sha(A[1]), sha(A[2])])
        if l < nl - 1:
            out[f"agg{l}"] = R.level_agg(l)
    return out


def solve(R, b, tol=1e-8, maxit=500):
    it, x, hist = R.pcg(b, None, tol, maxit, 1)
    return {"iters": np.int64(it), "x": x, "hist": hist}


def layout() -> dict:
    """sizeof/offsetof of the drop-in structures, from the reference headers."""
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "hazmath.h"
#define S(T) printf("\"sizeof(" #T ")\": %zu,\n", sizeof(T));
#define O(T,f) printf("\"" #T "." #f "\": %zu,\n", offsetof(T,f));
int main(){S(dCSRmat)S(dvector)S(ivector)S(linear_itsolver_param)S(AMG_param)
S(precond)S(Schwarz_data)S(AMG_data)S(precond_data)
O(dCSRmat,IA)O(dCSRmat,val)O(linear_itsolver_param,linear_tol)
O(linear_itsolver_param,AL_scaling_param)O(AMG_param,tol)O(AMG_param,coarse_dof)
O(AMG_param,relaxation)O(AMG_param,amli_coef)O(AMG_param,strong_coupled)
O(AMG_param,max_aggregation)O(AMG_param,tentative_smooth)O(AMG_param,HAZDIR)
O(AMG_param,damping_param)O(AMG_param,fpwr)O(AMG_param,smoother_function)
O(precond,fct)O(precond,setup_time)O(AMG_data,A)O(AMG_data,R)O(AMG_data,P)
O(AMG_data,b)O(AMG_data,x)O(AMG_data,Numeric)O(AMG_data,near_kernel_dim)
O(AMG_data,Schwarz)O(AMG_data,w)O(AMG_data,cycle_type)O(AMG_data,wdata)
O(precond_data,tol)O(precond_data,amli_coef)O(precond_data,mgl_data)
O(precond_data,fpwr)O(precond_data,A)O(precond_data,w)
S(dBSRmat)O(dBSRmat,nb)O(dBSRmat,val)O(dBSRmat,IA)O(dBSRmat,JA)
printf("\"end\": 0\n");return 0;}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "lay.c")
        exe = os.path.join(d, "lay")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-w", "-I", os.path.join(ROOT, "oracle", "_ref", "include"),
                        "-I", os.path.join(REF, "include"), c, "-o", exe], check=True)
        txt = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    d = json.loads("{" + txt + "}")
    d.pop("end")
    return d


def gmres_cases(R):
    """The reference's variable-restart GMRES (type 3) and flexible GMRES
    (type 4) with its AMG preconditioner: iterations, solution and the
    residual norm at every preconditioner call."""
    out = {}
    ia, ja, val = P.read_coo(os.path.join(REF, "examples", "solvers", "A.dat"))
    b = np.loadtxt(os.path.join(REF, "examples", "solvers", "b.dat"), skiprows=1)
    k = P.lognormal_field(14, 1.0, 4.0, 5)
    kia, kja, kval = P.kuhn3d_p1(14, k)
    kb = P.rhs_uniform(len(kia) - 1, 6)
    cases = [("fix", ia, ja, val, b, oracle.AMGParams()),
             ("kuhn", kia, kja, kval, kb,
              oracle.AMGParams(smoother=10, presmooth_iter=2, postsmooth_iter=2, coarse_dof=100))]
    for name, cia, cja, cval, cb, prm in cases:
        assert R.setup(cia, cja, cval, prm) == 0
        out[f"{name}/A_ia"], out[f"{name}/A_ja"], out[f"{name}/A_val"] = cia, cja, cval
        out[f"{name}/b"] = cb
        out[f"{name}/params"] = np.array(prm.arrays()[0][:], np.int64)
        out[f"{name}/dparams"] = np.array(prm.arrays()[1][:])
        for flex in (0, 1):
            for restart in (3, 7, 25, 100):
                for stop in ((1, 2, 3) if restart == 25 else (1,)):
                    it, x, hist = R.gmres(cb, tol=1e-8, maxit=300, restart=restart,
                                          flexible=bool(flex), stop_type=stop)
                    key = f"{name}/{'f' if flex else 'v'}{restart}_s{stop}"
                    out[key + "/iters"] = np.int64(it)
                    if restart in (3, 25) and stop == 1:
                        out[key + "/x"] = x
                    out[key + "/hist"] = hist
                    print("gmres", key, it)
        R.free()
    np.savez_compressed(os.path.join(HERE, "gmres.npz"), **out)


# cycle variants of cycles.npz: AMG_param overrides on top of each case's
CYCLE_VARIANTS = {
    "a2": dict(cycle_type=3),
    "a1": dict(cycle_type=3, amli_degree=1),
    "a3": dict(cycle_type=3, amli_degree=3),
    "a2s": dict(cycle_type=3, coarse_scaling=1),
    "a2i": dict(cycle_type=3, coarse_solver=0),
    "a2d": dict(cycle_type=3, coarse_dof=50),
    "n": dict(cycle_type=4),
    "ng": dict(cycle_type=4, nl_amli_krylov_type=5),
    "nd": dict(cycle_type=4, coarse_dof=50),
    "ngd": dict(cycle_type=4, coarse_dof=50, nl_amli_krylov_type=5),
    "ni": dict(cycle_type=4, coarse_solver=0),
    "d": dict(cycle_type=5),
    "ds": dict(cycle_type=5, coarse_scaling=1),
    "di": dict(cycle_type=5, coarse_solver=0),
    "v": dict(cycle_type=1),
}
CYCLE_X_FIX = {"a2/fgmres", "a2/pcg", "n/fgmres", "d/fgmres", "v/gcg"}


def cycle_cases(R):
    """The AMLI (cycle_type 3), nonlinear AMLI (4) and additive (5) cycles
    as linear_solver_dcsr_krylov_amg hands them to the Krylov methods: PCG,
    flexible GMRES(100) and GCG with the cycle's preconditioner, on the two
    matrices of gmres.npz; iterations, the residual norm at every
    preconditioner call, one preconditioner application z = B b, and
    solutions; plus amg_amli_coef for degrees 0 to 4."""
    out = {}
    g = np.load(os.path.join(HERE, "gmres.npz"))
    bases = {"fix": {}, "kuhn": dict(smoother=10, presmooth_iter=2, postsmooth_iter=2,
                                     coarse_dof=100)}
    for name, base in bases.items():
        cia, cja, cval = g[f"{name}/A_ia"], g[f"{name}/A_ja"], g[f"{name}/A_val"]
        cb = g[f"{name}/b"]
        for var, over in CYCLE_VARIANTS.items():
            kw = dict(base)
            kw.update(over)
            prm = oracle.AMGParams(**kw)
            assert R.setup(cia, cja, cval, prm) == 0
            key = f"{name}/{var}"
            out[key + "/params"] = np.array(prm.arrays()[0][:], np.int64)
            out[key + "/dparams"] = np.array(prm.arrays()[1][:])
            out[key + "/levels"] = np.int64(R.num_levels())
            if name == "kuhn" or var in ("a2", "n", "d"):
                out[key + "/z"] = R.precond(cb)
            runs = {"gcg": R.gcg(cb, tol=1e-8, maxit=100)}
            if var != "v":
                runs["pcg"] = R.pcg(cb, None, 1e-8, 300, 1)
                runs["fgmres"] = R.gmres(cb, tol=1e-8, maxit=300, restart=100, flexible=True)
            for kr, (it, x, hist) in runs.items():
                out[f"{key}/{kr}/iters"] = np.int64(it)
                out[f"{key}/{kr}/hist"] = hist
                if f"{var}/{kr}" in CYCLE_X_FIX or (
                        name == "kuhn" and (kr == "fgmres" or var in ("a2", "n", "d", "v"))):
                    out[f"{key}/{kr}/x"] = x
                print("cycles", key, kr, it)
            R.free()
    for d in range(5):
        out[f"amli_coef/{d}"] = R.amli_coef(2.0, 0.5, d)
    out["amli_coef/wide3"] = R.amli_coef(10.0, 0.1, 3)
    np.savez_compressed(os.path.join(HERE, "cycles.npz"), **out)


def cube_cases(R):
    """The reference's own P1 stiffness matrix on its own cube mesh
    (mesh_cube_init with uniform refinement + the elliptic_p1 example's
    call_assembly, unit coefficient), restricted to the interior vertices and
    renumbered lexicographically (x fastest) through the vertex coordinates:
    the matrix the Kuhn-mesh generator and the device assembly reproduce."""
    out = {}
    for ndiv in (4, 8, 12):
        ia, ja, val, xv, d = R.cube_p1(ndiv)
        g = np.rint(xv * ndiv).astype(np.int64)
        assert np.abs(g - xv * ndiv).max() < 1e-9
        m = ndiv - 1
        lex = (g[:, 0] - 1) + m * ((g[:, 1] - 1) + m * (g[:, 2] - 1))
        rows, cols, vals = [], [], []
        for i in np.where(d == 0)[0]:
            for k in range(ia[i], ia[i + 1]):
                assert d[ja[k]] == 0
                rows.append(lex[i])
                cols.append(lex[ja[k]])
                vals.append(val[k])
        rows, cols, vals = np.array(rows), np.array(cols), np.array(vals)
        order = np.lexsort((cols, rows))
        rows, cols, vals = rows[order], cols[order], vals[order]
        cia = np.zeros(m ** 3 + 1, np.int32)
        np.add.at(cia, rows + 1, 1)
        out[f"n{ndiv}/ia"] = np.cumsum(cia).astype(np.int32)
        out[f"n{ndiv}/ja"] = cols.astype(np.int32)
        out[f"n{ndiv}/val"] = vals
        print("cube", ndiv, len(vals))
    np.savez_compressed(os.path.join(HERE, "cube_p1.npz"), **out)


def minres_cases(R):
    """The reference's preconditioned MINRES (dcsr_pminres) on the matrices
    of gmres.npz with the V-cycle preconditioner, for the three stopping
    types, and without a preconditioner: iterations, the residual norm at
    every preconditioner call, solutions."""
    out = {}
    g = np.load(os.path.join(HERE, "gmres.npz"))
    bases = {"fix": {}, "kuhn": dict(smoother=10, presmooth_iter=2, postsmooth_iter=2,
                                     coarse_dof=100)}
    for name, base in bases.items():
        cia, cja, cval = g[f"{name}/A_ia"], g[f"{name}/A_ja"], g[f"{name}/A_val"]
        cb = g[f"{name}/b"]
        prm = oracle.AMGParams(**base)
        assert R.setup(cia, cja, cval, prm) == 0
        for stop in (1, 2, 3):
            it, x, hist = R.minres(cb, tol=1e-8, maxit=500, stop_type=stop)
            out[f"{name}/s{stop}/iters"] = np.int64(it)
            out[f"{name}/s{stop}/x"] = x
            out[f"{name}/s{stop}/hist"] = hist
            print("minres", name, stop, it)
        if name == "kuhn":
            it, x, _ = R.minres(cb, tol=1e-6, maxit=2000, stop_type=1, use_pc=False)
            out[f"{name}/nopc/iters"] = np.int64(it)
            out[f"{name}/nopc/x"] = x
            print("minres", name, "no pc", it)
        R.free()
    np.savez_compressed(os.path.join(HERE, "minres.npz"), **out)


SA_VARIANTS = {
    "fix/sa": ("fix", {}),
    "fix/sa_nf": ("fix", dict(smooth_filter=0)),
    "kuhn/sa": ("kuhn", {}),
    "kuhn/sa_nf": ("kuhn", dict(smooth_filter=0)),
    "kuhn/sa_t": ("kuhn", dict(strong_coupled=0.08)),
    "kuhn/sa_w": ("kuhn", dict(cycle_type=2, coarse_solver=0)),
}


def sa_cases(R):
    """Smoothed aggregation (amg_setup_sa) on the matrices of gmres.npz: the
    level sizes, SHA-256 digests of every coarse operator and of every
    smoothed prolongation (their arrays are large: the coarse levels of
    smoothed aggregation fill in), the adapted threshold, and PCG /
    flexible GMRES(100) iterations and solutions with the V-cycle (W-cycle
    with the iterative coarse solver for one variant)."""
    out = {}
    g = np.load(os.path.join(HERE, "gmres.npz"))
    bases = {"fix": {}, "kuhn": dict(smoother=10, presmooth_iter=2, postsmooth_iter=2,
                                     coarse_dof=100)}
    for key, (name, over) in SA_VARIANTS.items():
        cia, cja, cval = g[f"{name}/A_ia"], g[f"{name}/A_ja"], g[f"{name}/A_val"]
        cb = g[f"{name}/b"]
        kw = dict(bases[name])
        kw.update(over)
        kw["AMG_type"] = 2
        prm = oracle.AMGParams(**kw)
        assert R.setup(cia, cja, cval, prm) == 0
        nl = R.num_levels()
        out[key + "/params"] = np.array(prm.arrays()[0][:], np.int64)
        out[key + "/dparams"] = np.array(prm.arrays()[1][:])
        out[key + "/info"] = np.array([R.level_info(l)[:4] for l in range(nl)], np.int64)
        out[key + "/theta_after"] = np.float64(R.strong_coupled())
        for l in range(nl):
            out[f"{key}/A{l}_sha"] = np.array([sha(a) for a in R.level_A(l)])
            if l < nl - 1:
                out[f"{key}/P{l}_sha"] = np.array([sha(a) for a in R.level_P(l)])
        it, x, hist = R.pcg(cb, None, 1e-8, 300, 1)
        out[key + "/pcg/iters"] = np.int64(it)
        out[key + "/pcg/x"] = x
        out[key + "/pcg/hist"] = hist
        it, x, _ = R.gmres(cb, tol=1e-8, maxit=300, restart=100, flexible=True)
        out[key + "/fgmres/iters"] = np.int64(it)
        print("sa", key, nl, out[key + "/pcg/iters"], it)
        R.free()
    np.savez_compressed(os.path.join(HERE, "sa.npz"), **out)


VMB_VARIANTS = {
    "fix/vmb": ("fix", dict(coarse_dof=100)),
    "fix/vmb4": ("fix", dict(coarse_dof=100, max_aggregation=4)),
    "kuhn/vmb": ("kuhn", {}),
    "kuhn/vmb_t": ("kuhn", dict(strong_coupled=0.08)),
    "kuhn/vmb_w": ("kuhn", dict(cycle_type=2, max_aggregation=9)),
}


def vmb_cases(R):
    """VMB aggregation (aggregation_type 1, aggregation_vmb) on the matrices
    of gmres.npz: level sizes, every aggregate map, SHA-256 digests of every
    coarse operator, the adapted threshold, PCG iterations and solutions."""
    out = {}
    g = np.load(os.path.join(HERE, "gmres.npz"))
    bases = {"fix": {}, "kuhn": dict(smoother=10, presmooth_iter=2, postsmooth_iter=2,
                                     coarse_dof=100)}
    for key, (name, over) in VMB_VARIANTS.items():
        cia, cja, cval = g[f"{name}/A_ia"], g[f"{name}/A_ja"], g[f"{name}/A_val"]
        cb = g[f"{name}/b"]
        kw = dict(bases[name])
        kw.update(over)
        kw["aggregation_type"] = 1
        prm = oracle.AMGParams(**kw)
        assert R.setup(cia, cja, cval, prm) == 0
        nl = R.num_levels()
        out[key + "/params"] = np.array(prm.arrays()[0][:], np.int64)
        out[key + "/dparams"] = np.array(prm.arrays()[1][:])
        out[key + "/info"] = np.array([R.level_info(l)[:3] for l in range(nl)], np.int64)
        out[key + "/theta_after"] = np.float64(R.strong_coupled())
        for l in range(nl):
            out[f"{key}/A{l}_sha"] = np.array([sha(a) for a in R.level_A(l)])
            if l < nl - 1:
                out[f"{key}/agg{l}"] = R.level_agg(l)
        it, x, hist = R.pcg(cb, None, 1e-8, 300, 1)
        out[key + "/pcg/iters"] = np.int64(it)
        out[key + "/pcg/x"] = x
        print("vmb", key, out[key + "/info"][:, 0], it)
        R.free()
    np.savez_compressed(os.path.join(HERE, "vmb.npz"), **out)


def hec_cases(R):
    """HEC aggregation (aggregation_type 4, the reference's default) with the
    process's rand() seeded 1 (a fresh process), on the matrices of gmres.npz:
    every level's aggregate map and the adapted threshold."""
    out = {}
    g = np.load(os.path.join(HERE, "gmres.npz"))
    for name in ("fix", "kuhn"):
        prm = oracle.AMGParams(aggregation_type=4, strong_coupled=0.04, coarse_dof=100)
        R.srand(1)
        assert R.setup(g[f"{name}/A_ia"], g[f"{name}/A_ja"], g[f"{name}/A_val"], prm) == 0
        nl = R.num_levels()
        out[f"{name}/info"] = np.array([R.level_info(l)[:3] for l in range(nl)], np.int64)
        out[f"{name}/theta_after"] = np.float64(R.strong_coupled())
        for l in range(nl):
            out[f"{name}/A{l}_sha"] = np.array([sha(a) for a in R.level_A(l)])
            if l < nl - 1:
                out[f"{name}/agg{l}"] = R.level_agg(l)
        print("hec", name, out[f"{name}/info"][:, 0])
        R.free()
    np.savez_compressed(os.path.join(HERE, "hec.npz"), **out)


BSR_VARIANTS = {
    "kuhn/gs": ("kuhn", {}),
    "kuhn/jac": ("kuhn", dict(smoother=1, presmooth_iter=2, postsmooth_iter=2)),
    "kuhn/sgs": ("kuhn", dict(smoother=3)),
    "kuhn/w": ("kuhn", dict(cycle_type=2)),
    "kuhn/cs": ("kuhn", dict(coarse_scaling=1)),
    "kuhn/m2": ("kuhn", dict(maxit=2)),
    "kuhn/t": ("kuhn", dict(strong_coupled=0.08)),
    "kuhn/vmb": ("kuhn", dict(aggregation_type=1)),
    "fix/gs": ("fix", {}),
}
BSR_NB = {"kuhn": 3, "fix": 2}
BSR_SEED = {"kuhn": 31, "fix": 32}


def bsr_cases(R):
    """UA-AMG for block matrices (amg_setup_ua_bsr, precond_dbsr_amg,
    linear_solver_dbsr_krylov_amg) on problems.block_system of the matrices
    of gmres.npz (nb = 3 on the Kuhn case, 2 on the 5-point case): the
    level sizes, block aggregates, SHA-256 digests of every level's block
    matrix, one preconditioner application on b, and CG / GMRES(25) /
    flexible GMRES(25) iterations (and solutions on the Kuhn case)."""
    out = {}
    g = np.load(os.path.join(HERE, "gmres.npz"))
    bases = {"kuhn": dict(coarse_dof=100, coarse_solver=0),
             "fix": dict(coarse_solver=0)}
    for key, (name, over) in BSR_VARIANTS.items():
        nb = BSR_NB[name]
        ia, ja, val = P.block_system(g[f"{name}/A_ia"], g[f"{name}/A_ja"], g[f"{name}/A_val"],
                                     nb, BSR_SEED[name])
        if f"{name}/A_sha" not in out:
            out[f"{name}/A_sha"] = np.array([sha(ia), sha(ja), sha(val)])
            out[f"{name}/b"] = P.rhs_uniform((len(ia) - 1) * nb, BSR_SEED[name] + 1)
        b = out[f"{name}/b"]
        kw = dict(bases[name])
        kw.update(over)
        prm = oracle.AMGParams(**kw)
        assert R.bsr_setup(nb, ia, ja, val, prm) == 0
        nl = R.bsr_num_levels()
        out[key + "/params"] = np.array(prm.arrays()[0][:], np.int64)
        out[key + "/dparams"] = np.array(prm.arrays()[1][:])
        info = []
        for l in range(nl):
            A = R.bsr_level_A(l, nb)
            info.append((len(A[0]) - 1, len(A[1])))
            out[f"{key}/A{l}_sha"] = np.array([sha(a) for a in A])
            if l < nl - 1:
                out[f"{key}/agg{l}"] = R.bsr_level_agg(l)
        out[key + "/info"] = np.array(info, np.int64)
        out[key + "/z"] = R.bsr_precond(b)
        R.bsr_free()
        for typ, tag in ((1, "pcg"), (3, "gmres"), (4, "fgmres")):
            it, x = R.bsr_krylov_amg(nb, ia, ja, val, b, typ, tol=1e-8, maxit=300,
                                     restart=25, params=prm)
            out[f"{key}/{tag}/iters"] = np.int64(it)
            if name == "kuhn":
                out[f"{key}/{tag}/x"] = x
        print("bsr", key, info, [int(out[f"{key}/{t}/iters"]) for t in ("pcg", "gmres", "fgmres")])
    np.savez_compressed(os.path.join(HERE, "bsr.npz"), **out)


# The benchmark configurations' 3D instances: (cubes per edge, sigma, field
# seed, rhs seed, stride of the solution sample, smoothers recorded)
BIG = {
    "c2": (128, 1.0, 2, 3, 97, ("l1", "gs")),
    "c5": (256, 1.5, 7, 8, 797, ("l1",)),
}
BIG_SMOOTHERS = {"l1": dict(smoother=10, presmooth_iter=2, postsmooth_iter=2), "gs": {}}


def big_cases(R, name):
    """The FP64 drop-in at a benchmark configuration's full size: the 3D P1
    log-normal diffusion on the Kuhn mesh of N^3 cubes (128^3: sigma 1,
    seeds 2/3; 256^3: sigma 1.5, seeds 7/8), UA-AMG with HEM, theta 0,
    coarse_dof 2000, direct coarsest solve, with l1-Jacobi V(2,2) (and, at
    128^3, Gauss-Seidel V(1,1)); PCG to 1e-8 from x0 = 0.  Stored: level
    sizes, SHA-256 digests of every coarse operator and aggregate map, the
    adapted threshold, PCG iterations, the residual at every preconditioner
    call, a strided sample of the solution, the reference's own setup and
    solve seconds on this machine, and a strided sample of the l1-Jacobi
    solve tightened to 1e-12 (the FP64 oracle solve that the mixed-precision
    error is stated against)."""
    N, sigma, fseed, bseed, stride, smoothers = BIG[name]
    k = P.lognormal_field(N, sigma, 8.0, fseed)
    ia, ja, val = P.kuhn3d_p1(N, k)
    b = P.rhs_uniform(len(ia) - 1, bseed)
    out = {"A_sha": np.array([sha(ia), sha(ja), sha(val)]), "b_sha": np.array([sha(b)]),
           "stride": np.int64(stride)}
    for sm in smoothers:
        prm = oracle.AMGParams(**BIG_SMOOTHERS[sm])
        assert R.setup(ia, ja, val, prm) == 0
        nl = R.num_levels()
        out[f"{sm}/params"] = np.array(prm.arrays()[0][:], np.int64)
        out[f"{sm}/dparams"] = np.array(prm.arrays()[1][:])
        out[f"{sm}/info"] = np.array([R.level_info(l)[:3] for l in range(nl)], np.int64)
        out[f"{sm}/theta_after"] = np.float64(R.strong_coupled())
        for l in range(nl):
            out[f"{sm}/A{l}_sha"] = np.array([sha(a) for a in R.level_A(l)])
            if l < nl - 1:
                out[f"{sm}/agg{l}_sha"] = np.array([sha(R.level_agg(l))])
        it, x, hist = R.pcg(b, None, 1e-8, 500, 1)
        setup_s, solve_s = R.timings()
        out[f"{sm}/iters"] = np.int64(it)
        out[f"{sm}/hist"] = hist
        out[f"{sm}/x_sample"] = x[::stride].copy()
        out[f"{sm}/x_norm"] = np.float64(np.linalg.norm(x))
        out[f"{sm}/seconds"] = np.array([setup_s, solve_s])
        print(name, sm, "levels", out[f"{sm}/info"][:, 0], "iters", it,
              f"setup {setup_s:.1f} s solve {solve_s:.1f} s", flush=True)
        if sm == "l1":
            it12, x12, _ = R.pcg(b, None, 1e-12, 1000, 1)
            out["l1/tight/iters"] = np.int64(it12)
            out["l1/tight/x_sample"] = x12[::stride].copy()
            out["l1/tight/x_norm"] = np.float64(np.linalg.norm(x12))
            print(name, "tight iters", it12, flush=True)
        R.free()
    np.savez_compressed(os.path.join(HERE, f"{name}_kuhn.npz"), **out)


BATCH = (24, 3, 500, 30000)   # systems, seed, dof range of problems.batch_anisotropic
BATCH_STRIDE = 4


def batch_cases(R):
    """Each system of the GPU tests' batch (problems.batch_anisotropic(24,
    seed 3, 500-30000 dofs)) solved on its own by the reference: UA-AMG with
    HEM, theta 0, coarse_dof 2000, l1-Jacobi V(2,2), PCG to 1e-8 (iterations)
    and to 1e-12 (every 4th entry of the solution: the FP64 oracle the
    batch's answers are compared with)."""
    systems, _ = P.batch_anisotropic(BATCH[0], BATCH[1], BATCH[2], BATCH[3])
    out = {"stride": np.int64(BATCH_STRIDE)}
    prm = oracle.AMGParams(smoother=10, presmooth_iter=2, postsmooth_iter=2)
    for k, (ia, ja, val, b) in enumerate(systems):
        assert R.setup(ia, ja, val, prm) == 0
        out[f"{k}/A_sha"] = np.array([sha(ia), sha(ja), sha(val)])
        out[f"{k}/levels"] = np.int64(R.num_levels())
        it, _, _ = R.pcg(b, None, 1e-8, 500, 1)
        out[f"{k}/iters"] = np.int64(it)
        it12, x12, _ = R.pcg(b, None, 1e-12, 1000, 1)
        out[f"{k}/tight_iters"] = np.int64(it12)
        out[f"{k}/x_sample"] = x12[::BATCH_STRIDE].copy()
        out[f"{k}/x_norm"] = np.float64(np.linalg.norm(x12))
        print("batch", k, len(b), R.num_levels(), it, it12)
        R.free()
    np.savez_compressed(os.path.join(HERE, "batch.npz"), **out)


def main():
    if not oracle.ref_available():
        oracle.build(ref=True)
    R = oracle.ref()
    only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None
    if only in BIG:
        big_cases(R, only)
        return
    if only == "batch":
        batch_cases(R)
        return
    if only == "gmres":
        gmres_cases(R)
        return
    if only == "cycles":
        cycle_cases(R)
        return
    if only == "cube":
        cube_cases(R)
        return
    if only == "minres":
        minres_cases(R)
        return
    if only == "sa":
        sa_cases(R)
        return
    if only == "hec":
        hec_cases(R)
        return
    if only == "vmb":
        vmb_cases(R)
        return
    if only == "bsr":
        bsr_cases(R)
        return
    if only == "layout":
        with open(os.path.join(HERE, "layout.json"), "w") as f:
            json.dump(layout(), f, indent=1, sort_keys=True)
        return
    rng = np.random.default_rng(20261203)
    base = oracle.AMGParams()

    # 1. struct layouts
    with open(os.path.join(HERE, "layout.json"), "w") as f:
        json.dump(layout(), f, indent=1, sort_keys=True)

    # 2. the reference's known-answer case: examples/solvers A.dat / b.dat
    ia, ja, val = P.read_coo(os.path.join(REF, "examples", "solvers", "A.dat"))
    gia, gja, gval = P.poisson2d_5pt(128)
    assert np.array_equal(ia, gia) and np.array_equal(ja, gja) and np.array_equal(val, gval)
    b = np.loadtxt(os.path.join(REF, "examples", "solvers", "b.dat"), skiprows=1)
    g = hierarchy(R, ia, ja, val, base, full=False)
    g.update(solve(R, b))
    g["b"] = b
    g["A_sha"] = np.array([sha(ia), sha(ja), sha(val)])
    np.savez_compressed(os.path.join(HERE, "fixture128.npz"), **g)
    print("fixture128: levels", g["info"][:, 0], "iters", g["iters"])

    # 3. C1: 255^2 interior 5-point, b ~ U[-1,1] seed 1
    ia, ja, val = P.poisson2d_5pt(255)
    b = P.rhs_uniform(len(ia) - 1, 1)
    g = hierarchy(R, ia, ja, val, base, full=False)
    g.update(solve(R, b))
    g["x_sha"] = np.array([sha(g["x"])])
    g["x_head"] = g.pop("x")[:64]
    np.savez_compressed(os.path.join(HERE, "c1_poisson255.npz"), **g)
    print("C1: levels", g["info"][:, 0], "iters", g["iters"])

    # 4. small cases: full hierarchies, one preconditioner application, PCG
    small = {}
    cases = {
        "p2d_40": (P.poisson2d_5pt(40), base),
        "aniso2d_31": (P.aniso2d_p1(31, 0.02, 0.7), oracle.AMGParams(coarse_dof=60)),
        "kuhn_12": (P.kuhn3d_p1(12, P.lognormal_field(12, 1.0, 3.0, 2)),
                    oracle.AMGParams(coarse_dof=100)),
        "p2d_40_l1": (P.poisson2d_5pt(40), oracle.AMGParams(smoother=10, presmooth_iter=2,
                                                           postsmooth_iter=2, coarse_dof=80)),
        "p2d_40_sgs_w": (P.poisson2d_5pt(40), oracle.AMGParams(smoother=3, cycle_type=2,
                                                              coarse_dof=80)),
        "p2d_40_sor_cs": (P.poisson2d_5pt(40), oracle.AMGParams(smoother=5, relaxation=1.3,
                                                               coarse_scaling=1,
                                                               coarse_dof=80)),
        "p2d_40_jac_cg": (P.poisson2d_5pt(40), oracle.AMGParams(smoother=1, presmooth_iter=2,
                                                               postsmooth_iter=2,
                                                               coarse_solver=0,
                                                               coarse_dof=80)),
        "theta_p2d_40": (P.poisson2d_5pt(40), oracle.AMGParams(strong_coupled=0.25,
                                                              coarse_dof=50)),
    }
    for name, ((ia, ja, val), prm) in cases.items():
        n = len(ia) - 1
        g = hierarchy(R, ia, ja, val, prm, full=True)
        r = rng.uniform(-1, 1, n)
        z = R.precond(r)
        b = rng.uniform(-1, 1, n)
        s = solve(R, b)
        for k, v in g.items():
            small[f"{name}/{k}"] = v
        small[f"{name}/A_ia"], small[f"{name}/A_ja"], small[f"{name}/A_val"] = ia, ja, val
        small[f"{name}/params"] = np.array(
            [prm.max_levels, prm.coarse_dof, prm.cycle_type, prm.smoother, prm.presmooth_iter,
             prm.postsmooth_iter, prm.coarse_solver, prm.aggregation_type,
             prm.max_aggregation, prm.coarse_scaling, prm.print_level, prm.maxit], np.int64)
        small[f"{name}/dparams"] = np.array([prm.strong_coupled, prm.relaxation, prm.tol])
        small[f"{name}/r"], small[f"{name}/z"] = r, z
        small[f"{name}/b"] = b
        small[f"{name}/iters"], small[f"{name}/x"], small[f"{name}/hist"] = (
            s["iters"], s["x"], s["hist"])
        print(name, "levels", g["info"][:, 0], "iters", s["iters"])
    np.savez_compressed(os.path.join(HERE, "small_cases.npz"), **small)

    # 5. smoothers (pre = mgcycle's forward call, post = backward call)
    ia, ja, val = P.aniso2d_p1(19, 0.05, 1.1)
    n = len(ia) - 1
    b = rng.uniform(-1, 1, n)
    x0 = rng.uniform(-1, 1, n)
    sm = {"ia": ia, "ja": ja, "val": val, "b": b, "x0": x0}
    for s_id in (1, 2, 3, 5, 6, 7, 8, 10):
        for pre in (1, 0):
            sm[f"s{s_id}_pre{pre}"] = R.smooth(s_id, pre, 2, ia, ja, val, b, x0, relax=1.2)
    sm["mxv"] = R.mxv(ia, ja, val, x0)
    sm["aAxpy_m1"] = R.aAxpy(-1.0, ia, ja, val, x0, b)
    sm["aAxpy_07"] = R.aAxpy(0.7, ia, ja, val, x0, b)
    np.savez_compressed(os.path.join(HERE, "smoothers.npz"), **sm)

    # 6. RAP on a 3D anisotropic Kuhn matrix with a seeded aggregate map
    ia, ja, val = P.aniso3d_p1(7, 0.1, 0.8, (1.0, 2.0, 0.5))
    n = len(ia) - 1
    nc = n // 3
    agg = rng.integers(-1, nc, n).astype(np.int32)
    agg[:nc] = np.arange(nc)          # every aggregate non-empty
    cia, cja, cval = R.rap(ia, ja, val, nc, agg)
    np.savez_compressed(os.path.join(HERE, "rap.npz"), ia=ia, ja=ja, val=val, agg=agg,
                        nc=np.int64(nc), cia=cia, cja=cja, cval=cval)
    R.free()
    # 7. GMRES and flexible GMRES (Krylov types 3 and 4)
    gmres_cases(R)
    cycle_cases(R)
    cube_cases(R)
    minres_cases(R)
    sa_cases(R)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
