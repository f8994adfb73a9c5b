"""CPU oracle for the UA-AMG-PCG path -- TEST INFRASTRUCTURE ONLY.

Two interchangeable back ends with one Python interface:

* ``port`` -- ``libhzoracle.so``, the plain-C restatement of HAZmath's
  algorithm (oracle/hzoracle.c), available wherever gcc built it;
* ``ref``  -- ``_ref/libhazref.so``, the reference HAZmath library compiled
  from its own sources (oracle/build_ref.sh) plus a thin harness
  (oracle/ref_harness.c).  It exists where the reference sources were present
  at build time and travels with the repository snapshot as a built file.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package; the product (hazmath_b200) never does.
"""
from __future__ import annotations

import ctypes
import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "libhzoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhazref.so")

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)


def build(ref: bool = True) -> None:
    """Compile the oracle (and the reference harness when its sources exist)."""
    target = "all" if ref else "libhzoracle.so"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


@dataclass
class AMGParams:
    """The AMG_param fields this path reads (include/param.h of the reference),
    with the benchmark configurations' values as defaults: UA, HEM, theta = 0,
    V(1,1) Gauss-Seidel, coarse direct solve below 2000 rows."""

    max_levels: int = 20
    coarse_dof: int = 2000
    cycle_type: int = 1
    smoother: int = 2
    presmooth_iter: int = 1
    postsmooth_iter: int = 1
    coarse_solver: int = 32
    aggregation_type: int = 5
    max_aggregation: int = 20
    coarse_scaling: int = 0
    print_level: int = 0
    maxit: int = 1
    amli_degree: int = 2
    nl_amli_krylov_type: int = 4
    AMG_type: int = 1
    smooth_filter: int = 1
    strong_coupled: float = 0.0
    relaxation: float = 1.0
    tol: float = 1e-6
    tentative_smooth: float = 0.67

    def arrays(self):
        ip = (ctypes.c_int * 16)(
            self.max_levels, self.coarse_dof, self.cycle_type, self.smoother,
            self.presmooth_iter, self.postsmooth_iter, self.coarse_solver,
            self.aggregation_type, self.max_aggregation, self.coarse_scaling,
            self.print_level, self.maxit, self.amli_degree, self.nl_amli_krylov_type,
            self.AMG_type, self.smooth_filter)
        dp = (ctypes.c_double * 4)(self.strong_coupled, self.relaxation, self.tol,
                                   self.tentative_smooth)
        return ip, dp


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class _Backend:
    prefix = ""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path}")
        self.lib = ctypes.CDLL(path)
        self._keep = None
        pre = self.prefix
        self._f = lambda name: getattr(self.lib, pre + name)
        self._f("pcg").restype = ctypes.c_int
        self._f("strong_coupled").restype = ctypes.c_double

    # -- hierarchy ---------------------------------------------------------
    def setup(self, ia, ja, val, params: AMGParams | None = None) -> int:
        params = params or AMGParams()
        ia = np.ascontiguousarray(ia, np.int32)
        ja = np.ascontiguousarray(ja, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        self._keep = (ia, ja, val)   # the reference keeps pointers to A
        ip, dp = params.arrays()
        n = len(ia) - 1
        return self._f("setup")(n, int(ia[-1]), _p(ia), _p(ja), _p(val), ip, dp)

    def num_levels(self) -> int:
        return self._f("num_levels")()

    def strong_coupled(self) -> float:
        return self._f("strong_coupled")()

    def level_info(self, l: int):
        out = (ctypes.c_int * 5)()
        self._f("level_info")(l, out)
        return list(out)

    def level_A(self, l: int):
        n, nnz = self.level_info(l)[:2]
        ia = np.empty(n + 1, np.int32)
        ja = np.empty(nnz, np.int32)
        val = np.empty(nnz, np.float64)
        self._f("level_A")(l, _p(ia), _p(ja), _p(val))
        return ia, ja, val

    def level_agg(self, l: int):
        n = self.level_info(l)[0]
        agg = np.empty(n, np.int32)
        self._f("level_agg")(l, _p(agg))
        return agg

    def precond(self, r):
        r = np.ascontiguousarray(r, np.float64).copy()
        z = np.zeros_like(r)
        self._f("precond")(_p(r), _p(z))
        return z

    def pcg(self, b, x0=None, tol=1e-8, maxit=500, stop_type=1, hist_cap=1024):
        b = np.ascontiguousarray(b, np.float64).copy()
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
        hist = np.zeros(hist_cap)
        nh = ctypes.c_int()
        it = self._pcg_call(b, x, tol, maxit, stop_type, hist, hist_cap, nh)
        return it, x, hist[: min(nh.value, hist_cap)].copy()


class Port(_Backend):
    """The C restatement."""

    prefix = "or_"

    def __init__(self):
        super().__init__(PORT_SO)
        self.lib.or_hem_agg.restype = ctypes.c_int
        self.lib.or_rap.restype = ctypes.c_int

    def _pcg_call(self, b, x, tol, maxit, stop_type, hist, cap, nh):
        return self.lib.or_pcg(_p(b), _p(x), ctypes.c_double(tol), maxit,
                               stop_type, _p(hist), cap, ctypes.byref(nh))

    def level_info(self, l: int):
        out = (ctypes.c_int * 3)()
        self.lib.or_level_info(l, out)
        return list(out)

    def set_omega(self, omega):
        self._omega = None if omega is None else np.ascontiguousarray(omega, np.float32)
        self.lib.or_set_omega(None if omega is None else _p(self._omega))

    def free(self):
        self.lib.or_free()

    # -- learned weights ---------------------------------------------------
    def gnn_num_params(self):
        return self.lib.or_gnn_num_params()

    def gnn_forward(self, ia, ja, val, params, rounding=True):
        self.lib.or_gnn_set_rounding(1 if rounding else 0)
        self._gnn_keep = (np.ascontiguousarray(ia, np.int32), np.ascontiguousarray(ja, np.int32),
                          np.ascontiguousarray(val, np.float64))
        ia, ja, val = self._gnn_keep
        prm = np.ascontiguousarray(params, np.float32)
        om = np.empty(len(ia) - 1, np.float32)
        self.lib.or_gnn_forward(len(ia) - 1, _p(ia), _p(ja), _p(val), _p(prm), _p(om))
        return om

    def gnn_backward(self, params, domega):
        prm = np.ascontiguousarray(params, np.float32)
        d = np.ascontiguousarray(domega, np.float32)
        g = np.empty(self.gnn_num_params(), np.float32)
        self.lib.or_gnn_backward(_p(prm), _p(d), _p(g))
        return g

    def learn_errors(self, ns, seed, omega=None, ncycles=2):
        n = self.level_info(0)[0]
        E = np.empty((ns, n))
        om = None if omega is None else np.ascontiguousarray(omega, np.float32)
        self.lib.or_learn_errors(ns, C.c_ulonglong(seed), _p(E),
                                 None if om is None else _p(om), ncycles)
        return E

    def learn_loss_grad(self, omega, E, ncycles=2):
        om = np.ascontiguousarray(omega, np.float32)
        E = np.ascontiguousarray(E, np.float64)
        d = np.empty(E.shape[1])
        self.lib.or_learn_loss_grad.restype = C.c_double
        loss = self.lib.or_learn_loss_grad(_p(om), E.shape[0], _p(E), ncycles, _p(d))
        return loss, d

    # -- kernels -----------------------------------------------------------
    def mxv(self, ia, ja, val, x):
        y = np.empty(len(ia) - 1)
        self.lib.or_mxv(len(ia) - 1, _p(ia), _p(ja), _p(val), _p(x), _p(y))
        return y

    def aAxpy(self, alpha, ia, ja, val, x, y):
        y = np.array(y, np.float64)
        self.lib.or_aAxpy(ctypes.c_double(alpha), len(ia) - 1, _p(ia), _p(ja),
                          _p(val), _p(x), _p(y))
        return y

    def smooth(self, smoother, pre, sweeps, ia, ja, val, b, x, relax=1.0, omega=None):
        x = np.array(x, np.float64)
        om = None if omega is None else np.ascontiguousarray(omega, np.float32)
        rc = self.lib.or_smooth(smoother, int(pre), sweeps, ctypes.c_double(relax),
                                len(ia) - 1, _p(ia), _p(ja), _p(val), _p(b), _p(x),
                                None if om is None else _p(om))
        if rc:
            raise ValueError(f"smoother {smoother}: {rc}")
        return x

    def hem(self, ia, ja, val, theta=0.0):
        n = len(ia) - 1
        agg = np.empty(n, np.int32)
        nc = self.lib.or_hem_agg(n, _p(ia), _p(ja), _p(val), ctypes.c_double(theta), _p(agg))
        return nc, agg

    def minres_port(self, b, tol=1e-8, maxit=500, stop_type=1, use_pc=True, hist_cap=1024):
        """dcsr_pminres from x = 0 with the V/W cycle of the last setup (or
        none): (iterations, x, ||v|| of every vector preconditioned)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b)
        hist = np.zeros(hist_cap)
        nh = ctypes.c_int()
        it = self.lib.or_minres(_p(b), _p(x), ctypes.c_double(tol), maxit, stop_type,
                                int(use_pc), _p(hist), hist_cap, ctypes.byref(nh))
        return it, x, hist[: min(nh.value, hist_cap)].copy()

    def gmres_port(self, b, tol=1e-8, maxit=500, restart=25, flexible=True, stop_type=1,
                   hist_cap=1024):
        """dcsr_pvgmres / dcsr_pvfgmres from x = 0 with the V/W cycle of the
        last setup: (iterations, x, ||v|| of every vector preconditioned)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b)
        hist = np.zeros(hist_cap)
        nh = ctypes.c_int()
        it = self.lib.or_gmres(int(flexible), _p(b), _p(x), ctypes.c_double(tol), maxit,
                               restart, stop_type, _p(hist), hist_cap, ctypes.byref(nh))
        return it, x, hist[: min(nh.value, hist_cap)].copy()

    def gcg(self, b, kind=1, coef=None, amg_tol=1e-6, tol=1e-8, maxit=100, hist_cap=1024):
        """dcsr_pgcg from x = 0 with the cycle of the last setup (kind 1
        V/W, 3 AMLI with coef, 5 additive): (iterations, x, ||r|| at each
        preconditioner call)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b)
        c = np.ascontiguousarray(coef if coef is not None else [1.0], np.float64)
        hist = np.zeros(hist_cap)
        nh = ctypes.c_int()
        it = self.lib.or_gcg(_p(b), _p(x), ctypes.c_double(tol), maxit, kind, _p(c),
                             len(c) - 1, ctypes.c_double(amg_tol), _p(hist), hist_cap,
                             ctypes.byref(nh))
        return it, x, hist[: min(nh.value, hist_cap)].copy()

    def precond_nl_amli(self, r, degree=2, krylov=4, tol=1e-6):
        """z = B r with maxit nonlinear AMLI cycles of the last setup
        (coarse-level Krylov: 5 GCG, else flexible GMRES(30))."""
        r = np.ascontiguousarray(r, np.float64)
        z = np.zeros_like(r)
        self.lib.or_precond_nl_amli(degree, krylov, ctypes.c_double(tol), _p(r), _p(z))
        return z

    def precond_cycle(self, kind, r, coef=None, tol=1e-6):
        """z = B r with maxit AMLI (kind 3, polynomial coefficients coef) or
        additive (kind 5) cycles of the last setup's hierarchy."""
        r = np.ascontiguousarray(r, np.float64)
        z = np.zeros_like(r)
        c = np.ascontiguousarray(coef if coef is not None else [1.0], np.float64)
        rc = self.lib.or_precond_cycle(kind, _p(c), len(c) - 1, ctypes.c_double(tol), _p(r),
                                       _p(z))
        if rc:
            raise ValueError(f"cycle kind {kind}: {rc}")
        return z

    def sa_hierarchy(self, ia, ja, val, theta=0.0, coarse_dof=2000, max_levels=20,
                     aggregation_type=5, max_aggregation=20, smooth_filter=1,
                     tentative_smooth=0.67, coarse_solver=32):
        """The hierarchy of amg_setup_sa: a list of A per level, a list of the
        smoothed P per level below the coarsest, and the adapted threshold."""
        ia = np.ascontiguousarray(ia, np.int32)
        ja = np.ascontiguousarray(ja, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        th = ctypes.c_double()
        nl = self.lib.or_sa_setup(len(ia) - 1, int(ia[-1]), _p(ia), _p(ja), _p(val),
                                  ctypes.c_double(theta), coarse_dof, max_levels,
                                  aggregation_type, max_aggregation, int(smooth_filter == 1),
                                  ctypes.c_double(tentative_smooth), coarse_solver,
                                  ctypes.byref(th))
        As, Ps = [], []
        for l in range(nl):
            out = (ctypes.c_int * 3)()
            self.lib.or_sa_level_info(l, out)
            a = (np.empty(out[0] + 1, np.int32), np.empty(out[1], np.int32), np.empty(out[1]))
            self.lib.or_sa_level_A(l, *(_p(x) for x in a))
            As.append(a)
            if l < nl - 1:
                pp = (np.empty(out[0] + 1, np.int32), np.empty(out[2], np.int32),
                      np.empty(out[2]))
                self.lib.or_sa_level_P(l, *(_p(x) for x in pp))
                Ps.append(pp)
        return As, Ps, th.value

    def bsr_hierarchy(self, nb, ia, ja, val, theta=0.0, coarse_dof=2000, max_levels=20,
                      aggregation_type=5, max_aggregation=20):
        """The block hierarchy of amg_setup_ua_bsr: a list of (ia, ja, val) per
        level and the block aggregate maps of the levels below the coarsest."""
        ia = np.ascontiguousarray(ia, np.int32)
        ja = np.ascontiguousarray(ja, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        nl = self.lib.or_bsr_setup(len(ia) - 1, int(ia[-1]), nb, _p(ia), _p(ja), _p(val),
                                   ctypes.c_double(theta), coarse_dof, max_levels,
                                   aggregation_type, max_aggregation)
        levels, aggs = [], []
        for l in range(nl):
            out = (ctypes.c_int * 2)()
            self.lib.or_bsr_level_info(l, out)
            lia = np.empty(out[0] + 1, np.int32)
            lja = np.empty(out[1], np.int32)
            lval = np.empty(out[1] * nb * nb)
            self.lib.or_bsr_level_A(l, _p(lia), _p(lja), _p(lval))
            levels.append((lia, lja, lval))
            if l < nl - 1:
                agg = np.empty(out[0], np.int32)
                self.lib.or_bsr_level_agg(l, _p(agg))
                aggs.append(agg)
        return levels, aggs

    def bsr_precond(self, r, cycle_type=1, smoother=2, presmooth_iter=1, coarse_scaling=0,
                    maxit=1):
        """z = B r of precond_dbsr_amg on the last bsr_hierarchy."""
        r = np.ascontiguousarray(r, np.float64)
        z = np.zeros_like(r)
        rc = self.lib.or_bsr_precond(cycle_type, smoother, presmooth_iter, coarse_scaling,
                                     maxit, _p(r), _p(z))
        if rc:
            raise ValueError(f"or_bsr_precond: {rc}")
        return z

    def srand(self, seed: int) -> None:
        """Seed the oracle's restatement of the C library's rand() stream."""
        self.lib.or_srand(ctypes.c_uint(seed))

    def rand(self) -> int:
        return self.lib.or_rand()

    def hec(self, ia, ja, val, theta=0.0):
        """aggregation_hec on the strength graph of (ia, ja, val), its row order
        drawn from the rand() stream (continuing from the last call)."""
        n = len(ia) - 1
        agg = np.empty(n, np.int32)
        nc = self.lib.or_hec_agg(n, _p(ia), _p(ja), _p(val), ctypes.c_double(theta), _p(agg))
        return nc, agg

    def vmb(self, ia, ja, val, theta=0.0, max_aggregation=20):
        """aggregation_vmb on the strength graph of (ia, ja, val)."""
        n = len(ia) - 1
        agg = np.empty(n, np.int32)
        nc = self.lib.or_vmb_agg(n, _p(ia), _p(ja), _p(val), ctypes.c_double(theta),
                                 max_aggregation, _p(agg))
        return nc, agg

    def rap(self, ia, ja, val, nc, agg):
        n = len(ia) - 1
        agg = np.ascontiguousarray(agg, np.int32)
        cia = np.empty(nc + 1, np.int32)
        nnz = self.lib.or_rap(n, _p(ia), _p(ja), _p(val), nc, _p(agg), _p(cia), None, None)
        cja = np.empty(nnz, np.int32)
        cv = np.empty(nnz)
        self.lib.or_rap(n, _p(ia), _p(ja), _p(val), nc, _p(agg), _p(cia), _p(cja), _p(cv))
        return cia, cja, cv


class Ref(_Backend):
    """The reference library compiled from its sources."""

    prefix = "ref_"

    def __init__(self):
        super().__init__(REF_SO)
        self.lib.ref_rap_agg.restype = ctypes.c_int
        self.lib.ref_setup_seconds.restype = ctypes.c_double
        self.lib.ref_solve_seconds.restype = ctypes.c_double

    def _pcg_call(self, b, x, tol, maxit, stop_type, hist, cap, nh):
        return self.lib.ref_pcg(_p(b), _p(x), ctypes.c_double(tol), maxit,
                                stop_type, 0, _p(hist), cap, ctypes.byref(nh))

    def timings(self):
        return self.lib.ref_setup_seconds(), self.lib.ref_solve_seconds()

    def gmres(self, b, x0=None, tol=1e-8, maxit=500, restart=25, flexible=True,
              stop_type=1, hist_cap=1024):
        """dcsr_pvfgmres (flexible) or dcsr_pvgmres with the AMG
        preconditioner of the last setup: (iterations, x, ||r|| at each
        preconditioner call)."""
        b = np.ascontiguousarray(b, np.float64).copy()
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
        hist = np.zeros(hist_cap)
        nh = ctypes.c_int()
        it = self.lib.ref_gmres(4 if flexible else 3, _p(b), _p(x), ctypes.c_double(tol),
                                maxit, restart, stop_type, 0, _p(hist), hist_cap,
                                ctypes.byref(nh))
        return it, x, hist[: min(nh.value, hist_cap)].copy()

    def minres(self, b, x0=None, tol=1e-8, maxit=500, stop_type=1, use_pc=True, hist_cap=1024):
        """dcsr_pminres with the preconditioner of the last setup (or none):
        (iterations, x, ||r|| at each preconditioner call)."""
        b = np.ascontiguousarray(b, np.float64).copy()
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
        hist = np.zeros(hist_cap)
        nh = ctypes.c_int()
        it = self.lib.ref_minres(_p(b), _p(x), ctypes.c_double(tol), maxit, stop_type,
                                 int(use_pc), _p(hist), hist_cap, ctypes.byref(nh))
        return it, x, hist[: min(nh.value, hist_cap)].copy()

    def gcg(self, b, x0=None, tol=1e-8, maxit=100, hist_cap=1024):
        """dcsr_pgcg with the preconditioner of the last setup:
        (iterations, x, ||r|| at each preconditioner call)."""
        b = np.ascontiguousarray(b, np.float64).copy()
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
        hist = np.zeros(hist_cap)
        nh = ctypes.c_int()
        it = self.lib.ref_gcg(_p(b), _p(x), ctypes.c_double(tol), maxit, 0, _p(hist),
                              hist_cap, ctypes.byref(nh))
        return it, x, hist[: min(nh.value, hist_cap)].copy()

    def level_P(self, l: int):
        """P of level l with its values."""
        n, _, nc, pnnz = self.level_info(l)[:4]
        ia = np.empty(n + 1, np.int32)
        ja = np.empty(pnnz, np.int32)
        val = np.empty(pnnz)
        self.lib.ref_level_P(l, _p(ia), _p(ja), _p(val))
        return ia, ja, val

    def cube_p1(self, ndiv):
        """The reference's own P1 stiffness on its cube mesh with ndiv
        divisions per edge (mesh_cube_init + call_assembly, Dirichlet rows
        set to identity): (ia, ja, val, vertex coordinates (nv, 3),
        Dirichlet flags)."""
        out = (ctypes.c_int * 3)()
        self.lib.ref_cube_p1(ndiv, out)
        nv, nnz = out[0], out[1]
        ia = np.empty(nv + 1, np.int32)
        ja = np.empty(nnz, np.int32)
        val = np.empty(nnz)
        xv = np.empty(3 * nv)
        d = np.empty(nv, np.int32)
        self.lib.ref_cube_p1_get(_p(ia), _p(ja), _p(val), _p(xv), _p(d))
        return ia, ja, val, xv.reshape(nv, 3), d

    def amli_coef(self, lambda_max, lambda_min, degree):
        c = np.zeros(degree + 1)
        self.lib.ref_amli_coef(ctypes.c_double(lambda_max), ctypes.c_double(lambda_min),
                               degree, _p(c))
        return c

    def free(self):
        self.lib.ref_free()

    # -- block (BSR) matrices: amg_setup_ua_bsr, precond_dbsr_amg ----------
    def srand(self, seed: int) -> None:
        """srand() in the reference's process (its HEC draws from rand())."""
        self.lib.ref_srand(ctypes.c_uint(seed))

    def bsr_setup(self, nb, ia, ja, val, params: AMGParams | None = None) -> int:
        params = params or AMGParams()
        ia = np.ascontiguousarray(ia, np.int32)
        ja = np.ascontiguousarray(ja, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        self._keep_bsr = (ia, ja, val)
        ip, dp = params.arrays()
        return self.lib.ref_bsr_setup(len(ia) - 1, int(ia[-1]), nb, _p(ia), _p(ja), _p(val),
                                      ip, dp)

    def bsr_num_levels(self) -> int:
        return self.lib.ref_bsr_num_levels()

    def bsr_level_A(self, l: int, nb: int):
        out = (ctypes.c_int * 2)()
        self.lib.ref_bsr_level_info(l, out)
        n, nnzb = out[0], out[1]
        ia = np.empty(n + 1, np.int32)
        ja = np.empty(nnzb, np.int32)
        val = np.empty(nnzb * nb * nb)
        self.lib.ref_bsr_level_A(l, _p(ia), _p(ja), _p(val))
        return ia, ja, val

    def bsr_level_agg(self, l: int):
        out = (ctypes.c_int * 2)()
        self.lib.ref_bsr_level_info(l, out)
        agg = np.empty(out[0], np.int32)
        self.lib.ref_bsr_level_agg(l, _p(agg))
        return agg

    def bsr_precond(self, r):
        r = np.ascontiguousarray(r, np.float64).copy()
        z = np.zeros_like(r)
        self.lib.ref_bsr_precond(_p(r), _p(z))
        return z

    def bsr_free(self):
        self.lib.ref_bsr_free()

    def bsr_krylov_amg(self, nb, ia, ja, val, b, type_, tol=1e-8, maxit=500, stop_type=1,
                       restart=25, params: AMGParams | None = None):
        """linear_solver_dbsr_krylov_amg from x = 0: (iterations, x)."""
        params = params or AMGParams()
        ia = np.ascontiguousarray(ia, np.int32)
        ja = np.ascontiguousarray(ja, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        b = np.ascontiguousarray(b, np.float64).copy()
        x = np.zeros_like(b)
        ip, dp = params.arrays()
        it = self.lib.ref_bsr_krylov_amg(len(ia) - 1, int(ia[-1]), nb, _p(ia), _p(ja), _p(val),
                                         _p(b), _p(x), type_, ctypes.c_double(tol), maxit,
                                         stop_type, restart, ip, dp)
        return it, x

    def mxv(self, ia, ja, val, x):
        n = len(ia) - 1
        y = np.empty(n)
        self.lib.ref_mxv(n, int(ia[-1]), _p(ia), _p(ja), _p(val), _p(x), _p(y))
        return y

    def aAxpy(self, alpha, ia, ja, val, x, y):
        y = np.array(y, np.float64)
        n = len(ia) - 1
        self.lib.ref_aAxpy(ctypes.c_double(alpha), n, int(ia[-1]), _p(ia), _p(ja),
                           _p(val), _p(x), _p(y))
        return y

    def smooth(self, smoother, pre, sweeps, ia, ja, val, b, x, relax=1.0, omega=None):
        assert omega is None
        x = np.array(x, np.float64)
        n = len(ia) - 1
        self.lib.ref_smooth(smoother, int(pre), sweeps, ctypes.c_double(relax), n,
                            int(ia[-1]), _p(ia), _p(ja), _p(val), _p(b), _p(x))
        return x

    def rap(self, ia, ja, val, nc, agg):
        n = len(ia) - 1
        agg = np.ascontiguousarray(agg, np.int32)
        cia = np.empty(nc + 1, np.int32)
        nnz = self.lib.ref_rap_agg(n, int(ia[-1]), _p(ia), _p(ja), _p(val), nc,
                                   _p(agg), _p(cia), None, None)
        cja = np.empty(nnz, np.int32)
        cv = np.empty(nnz)
        self.lib.ref_rap_agg(n, int(ia[-1]), _p(ia), _p(ja), _p(val), nc, _p(agg),
                             _p(cia), _p(cja), _p(cv))
        return cia, cja, cv


def port() -> Port:
    return Port()


def ref() -> Ref:
    return Ref()


def ref_available() -> bool:
    return os.path.exists(REF_SO)
