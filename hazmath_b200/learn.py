"""Learned l1-Jacobi weights: the network handle, its training loop and the
fallback selection, over the library's C ABI (hzb_gnn_*, hzb_learn_*).

Training follows the method: for each training problem a UA-AMG hierarchy
(l1-Jacobi V(2,2)) is built on the GPU, and the loss is the two-cycle A-norm
contraction of the errors the network's cycle itself leaves after two cycles
from random smooth vectors, ||E^4 z||^2 / ||E^2 z||^2.  Its exact gradient
(adjoint cycles through all four cycles) drives the network's backward
kernels and an Adam step.

    python -m hazmath_b200.learn --steps 300 --out hazmath_b200/gnn_weights.npy

trains on seeded synthetic problems -- 2D anisotropic P1 diffusion (epsilon
log-uniform in [1e-4, 1], random rotation) and 3D log-normal Kuhn diffusion --
and writes the FP32 master weights.
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import time

import numpy as np

from . import problems as P
from . import (HZB_MATCH_PARALLEL, HZB_PREC_FP64, SMOOTHER_L1DIAG, Solver, b200_param, lib,
               last_error, bench_amg)

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "gnn_weights.npy")


def _setup_lib():
    L = lib()
    L.hzb_gnn_create.argtypes = [C.POINTER(C.c_void_p), C.c_ulonglong, C.c_int]
    L.hzb_gnn_destroy.argtypes = [C.c_void_p]
    for f in ("hzb_gnn_get_params", "hzb_gnn_set_params", "hzb_gnn_get_grads"):
        getattr(L, f).argtypes = [C.c_void_p, C.c_void_p]
    L.hzb_gnn_zero_grad.argtypes = [C.c_void_p]
    L.hzb_gnn_adam_step.argtypes = [C.c_void_p, C.c_double]
    L.hzb_gnn_infer.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.hzb_gnn_backward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.hzb_learn_errors.argtypes = [C.c_void_p, C.c_int, C.c_ulonglong, C.c_void_p,
                                   C.c_void_p, C.c_int]
    L.hzb_learn_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                      C.POINTER(C.c_double), C.c_void_p]
    L.hzb_learn_select_omega.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_ulonglong,
                                         C.POINTER(C.c_double), C.POINTER(C.c_double)]
    return L


def _check(rc, what):
    if rc:
        raise RuntimeError(f"{what}: {rc} {last_error()}")


class GNN:
    """The weight-predicting network (device resident)."""

    def __init__(self, seed: int = 0, device: int = 0, weights: str | None = None):
        self.L = _setup_lib()
        self.h = C.c_void_p()
        _check(self.L.hzb_gnn_create(C.byref(self.h), seed, device), "hzb_gnn_create")
        self.nparam = self.L.hzb_gnn_num_params()
        if weights:
            self.load(weights)

    def params(self) -> np.ndarray:
        p = np.empty(self.nparam, np.float32)
        _check(self.L.hzb_gnn_get_params(self.h, p.ctypes.data), "get_params")
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparam
        _check(self.L.hzb_gnn_set_params(self.h, p.ctypes.data), "set_params")

    def grads(self) -> np.ndarray:
        g = np.empty(self.nparam, np.float32)
        _check(self.L.hzb_gnn_get_grads(self.h, g.ctypes.data), "get_grads")
        return g

    def save(self, path: str) -> None:
        np.save(path, self.params())

    def load(self, path: str) -> None:
        self.set_params(np.load(path))

    def infer(self, solver: Solver, omega_ptr: int) -> None:
        _check(self.L.hzb_gnn_infer(self.h, solver.h, C.c_void_p(omega_ptr)), "infer")

    def backward(self, solver: Solver, domega_ptr: int) -> None:
        _check(self.L.hzb_gnn_backward(self.h, solver.h, C.c_void_p(domega_ptr)), "backward")

    def zero_grad(self) -> None:
        _check(self.L.hzb_gnn_zero_grad(self.h), "zero_grad")

    def adam(self, lr: float) -> None:
        _check(self.L.hzb_gnn_adam_step(self.h, lr), "adam")

    def select(self, solver: Solver, ns: int = 4, seed: int = 99):
        """Learned weights with fallback on the solver (see
        hzb_learn_select_omega); returns (rho_plain, rho_learned, used)."""
        rp, rl = C.c_double(), C.c_double()
        _check(self.L.hzb_learn_select_omega(solver.h, self.h, ns, seed, C.byref(rp),
                                             C.byref(rl)), "select_omega")
        return rp.value, rl.value, bool(solver.stats().omega_used)

    def close(self) -> None:
        if self.h:
            self.L.hzb_gnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def loss_grad(solver: Solver, omega_ptr: int, E_ptr: int, ns: int, domega_ptr: int,
              ncycles: int = 2) -> float:
    """mean ||E^k e||_A^2 / ||e||_A^2 over the ns vectors (k = ncycles) and
    its gradient with respect to omega into domega_ptr."""
    L = _setup_lib()
    loss = C.c_double()
    _check(L.hzb_learn_loss_grad(solver.h, C.c_void_p(omega_ptr), ns, C.c_void_p(E_ptr),
                                 ncycles, C.byref(loss), C.c_void_p(domega_ptr)), "loss_grad")
    return loss.value


def errors(solver: Solver, ns: int, seed: int, E_ptr: int, omega_ptr: int | None = None,
           ncycles: int = 2) -> None:
    """ns error vectors: random, three plain l1 sweeps, then ncycles cycles
    with fine-level weights omega_ptr (plain weights if None)."""
    om = C.c_void_p(omega_ptr) if omega_ptr else None
    _check(_setup_lib().hzb_learn_errors(solver.h, ns, seed, C.c_void_p(E_ptr), om, ncycles),
           "errors")


def training_problem(rng: np.random.Generator, small: bool = False):
    """A seeded training matrix: 2D anisotropic P1 diffusion (epsilon
    log-uniform in [1e-4, 1], angle uniform in [0, pi)) or 3D log-normal
    Kuhn diffusion (sigma in [0.5, 1.5], correlation 4-8 cells)."""
    if rng.uniform() < 0.5:
        m = int(rng.integers(40, 96) if small else rng.integers(127, 512))
        eps = float(10 ** rng.uniform(-4, 0))
        return P.aniso2d_p1(m, eps, float(rng.uniform(0, np.pi)))
    N = int(rng.integers(12, 24) if small else rng.integers(24, 64))
    k = P.lognormal_field(N, float(rng.uniform(0.5, 1.5)), float(rng.uniform(4, 8)),
                          int(rng.integers(1 << 30)))
    return P.kuhn3d_p1(N, k)


def l1_solver(device: int = 0) -> Solver:
    amg = bench_amg(smoother=SMOOTHER_L1DIAG, presmooth_iter=2, postsmooth_iter=2,
                     coarse_dof=400)
    return Solver(amg, None, b200_param(precision=HZB_PREC_FP64, matching=HZB_MATCH_PARALLEL,
                                        device=device))


def train(gnn: GNN, steps: int, lr: float = 3e-3, ns: int = 4, seed: int = 5,
          small: bool = False, device: int = 0, log=print):
    """Adam on the two-cycle contraction over a stream of seeded problems."""
    import torch
    rng = np.random.default_rng(seed)
    dev = f"cuda:{device}"
    hist = []
    t0 = time.time()
    for step in range(steps):
        ia, ja, val = training_problem(rng, small)
        n = len(ia) - 1
        S = l1_solver(device)
        tia, tja = torch.from_numpy(ia).to(dev), torch.from_numpy(ja).to(dev)
        tval = torch.from_numpy(val).to(dev)
        _check(S.setup_device(n, len(ja), tia.data_ptr(), tja.data_ptr(), tval.data_ptr()),
               "setup")
        if S.stats().num_levels < 2:
            S.close()
            continue
        E = torch.empty((ns, n), dtype=torch.float64, device=dev)
        om = torch.empty(n, dtype=torch.float32, device=dev)
        d4 = torch.empty(n, dtype=torch.float32, device=dev)
        d2 = torch.empty(n, dtype=torch.float32, device=dev)
        gnn.infer(S, om.data_ptr())
        # The objective is the two-cycle contraction of the errors the current
        # cycle leaves, rho^4 = ||E^4 z||^2 / ||E^2 z||^2 with z independent of
        # omega (random vectors after three plain sweeps).  Its gradient takes
        # the dependence of those errors on omega into account: d log rho^4 =
        # d log ||E^4 z||^2 - d log ||E^2 z||^2.  (Holding the errors fixed
        # instead pushes omega up everywhere: it misses the modes a larger
        # omega leaves behind.)
        errors(S, ns, int(rng.integers(1 << 40)), E.data_ptr(), None, 0)
        l4 = loss_grad(S, om.data_ptr(), E.data_ptr(), ns, d4.data_ptr(), 4)
        l2 = loss_grad(S, om.data_ptr(), E.data_ptr(), ns, d2.data_ptr(), 2)
        dom = d4 / l4 - d2 / l2
        gnn.zero_grad()
        gnn.backward(S, dom.data_ptr())
        gnn.adam(lr)
        loss = l4 / l2
        hist.append(loss)
        if log and (step % 20 == 0 or step == steps - 1):
            log(f"step {step:4d} n {n:7d} loss {loss:.4e} "
                f"mean(last 20) {np.mean(hist[-20:]):.4e} omega [{float(om.min()):.3f}, "
                f"{float(om.max()):.3f}] {time.time() - t0:.1f}s")
        S.close()
    return hist


def eval_problem(rng: np.random.Generator, m: int = 1022):
    """An unseen evaluation matrix: 2D anisotropic P1 diffusion on the
    (m+2)^2-vertex square mesh (m^2 dofs; 1024^2 vertices by default),
    epsilon log-uniform in [1e-4, 1],
    random rotation, with a uniform random right-hand side."""
    eps = float(10 ** rng.uniform(-4, 0))
    theta = float(rng.uniform(0, np.pi))
    ia, ja, val = P.aniso2d_p1(m, eps, theta)
    b = rng.uniform(-1.0, 1.0, len(ia) - 1)
    return ia, ja, val, b, {"eps": eps, "angle": theta, "dofs": len(ia) - 1}


def evaluate(gnn: GNN, problems, precision: int | None = None, device: int = 0,
             ns: int = 4, seed: int = 99):
    """Plain l1-Jacobi AMG-PCG against the learned weights (with fallback) on
    each (ia, ja, val, b, info): iterations and solve seconds to 1e-8, the
    measured per-cycle contractions, and which weights the selection kept."""
    import torch
    from . import HZB_PREC_MIXED, PREC_AMG, SOLVER_CG, STOP_REL_RES, itsolver_param
    prec = HZB_PREC_MIXED if precision is None else precision
    dev = f"cuda:{device}"
    out = []
    for ia, ja, val, b, info in problems:
        n = len(ia) - 1
        tia, tja = torch.from_numpy(ia).to(dev), torch.from_numpy(ja).to(dev)
        tval, tb = torch.from_numpy(val).to(dev), torch.from_numpy(b).to(dev)
        x = torch.zeros_like(tb)
        amg = bench_amg(smoother=SMOOTHER_L1DIAG, presmooth_iter=2, postsmooth_iter=2)
        it = itsolver_param(linear_itsolver_type=SOLVER_CG, linear_precond_type=PREC_AMG,
                            linear_tol=1e-8, linear_maxit=1000,
                            linear_stop_type=STOP_REL_RES)
        S = Solver(amg, it, b200_param(precision=prec, matching=HZB_MATCH_PARALLEL,
                                        device=device))
        _check(S.setup_device(n, len(ja), tia.data_ptr(), tja.data_ptr(), tval.data_ptr()),
               "setup")
        row = dict(info)
        for label in ("plain", "learned"):
            if label == "learned":
                t0 = time.perf_counter()
                rp, rl, used = gnn.select(S, ns, seed)
                torch.cuda.synchronize()
                row.update(rho_plain=rp, rho_learned=rl, learned_used=used,
                           select_s=time.perf_counter() - t0)
            x.zero_()
            its = S.solve_device(tb.data_ptr(), x.data_ptr())
            if its < 0:
                raise RuntimeError(f"solve failed {its}: {last_error()}")
            st = S.stats()
            row[f"{label}_iters"] = int(its)
            row[f"{label}_solve_s"] = st.solve_seconds
            row[f"{label}_relres"] = st.final_relres
        S.close()
        out.append(row)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--ns", type=int, default=4)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--small", action="store_true")
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--init", default=None)
    ap.add_argument("--eval", type=int, default=0,
                    help="then evaluate on this many unseen 1024^2-vertex problems")
    a = ap.parse_args()
    g = GNN(seed=a.seed, weights=a.init)
    if a.steps > 0:
        train(g, a.steps, a.lr, a.ns, a.seed, a.small)
        g.save(a.out)
        print("saved", a.out)
    if a.eval:
        rng = np.random.default_rng(20260)
        for row in evaluate(g, (eval_problem(rng) for _ in range(a.eval))):
            print(row, flush=True)


if __name__ == "__main__":
    main()
