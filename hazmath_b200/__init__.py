"""hazmath_b200 -- B200-native UA-AMG preconditioned Krylov solve (HAZmath drop-in).

The product is the CUDA shared library ``libhazb200.so`` built from ``csrc/``
(sm_100a).  This module is its Python host mirror through ctypes: the
HAZmath structures (``dCSRmat``, ``dvector``, ``AMG_param``,
``linear_itsolver_param``, ``precond_data``, ``AMG_data``), the drop-in entry
points with HAZmath's names and argument meaning, and a thin ``Solver``
wrapper over the persistent device handle.  There is no CPU fallback: if the
library is missing or no GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhazb200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "hazmath_b200.h")

INT = C.c_int
SHORT = C.c_short
REAL = C.c_double

# constants of include/macro.h (same values)
SUCCESS = 0
ERROR_INPUT_PAR = -13
ERROR_MAT_SIZE = -15
ERROR_ALLOC_MEM = -20
ERROR_DATA_STRUCTURE = -21
ERROR_DATA_ZERODIAG = -22
ERROR_AMG_SMOOTH_TYPE = -31
ERROR_AMG_COARSEING = -33
ERROR_SOLVER_TYPE = -40
ERROR_SOLVER_STAG = -42
ERROR_SOLVER_SOLSTAG = -43
ERROR_SOLVER_TOLSMALL = -44
ERROR_SOLVER_MISC = -47
ERROR_SOLVER_MAXIT = -48
SOLVER_CG = 1
SOLVER_MinRes, SOLVER_VGMRES, SOLVER_VFGMRES, SOLVER_GCG = 2, 3, 4, 5
SOLVER_UMFPACK = 32
STOP_REL_RES, STOP_REL_PRECRES, STOP_MOD_REL_RES = 1, 2, 3
PREC_AMG = 2
UA_AMG, SA_AMG = 1, 2
VMB, HEC, HEM = 1, 4, 5
V_CYCLE, W_CYCLE, AMLI_CYCLE, NL_AMLI_CYCLE, ADD_CYCLE = 1, 2, 3, 4, 5
SMOOTHER_JACOBI, SMOOTHER_GS, SMOOTHER_SGS = 1, 2, 3
SMOOTHER_SOR, SMOOTHER_SSOR, SMOOTHER_GSOR, SMOOTHER_SGSOR = 5, 6, 7, 8
SMOOTHER_L1DIAG = 10
HZB_PREC_FP64, HZB_PREC_MIXED = 0, 1
HZB_GS_EXACT, HZB_GS_MULTICOLOR = 0, 1
HZB_MATCH_EXACT, HZB_MATCH_PARALLEL = 0, 1
# kernels hzb_time_kernel can time
HZB_K_SPMV64, HZB_K_SPMV32, HZB_K_RES64, HZB_K_L1_32, HZB_K_L1_64 = 0, 1, 2, 3, 4
HZB_K_BSR_RES, HZB_K_BSR_JAC, HZB_K_BSR_GS, HZB_K_GS64 = 5, 6, 7, 8
MAX_AMG_LVL = 20


class dCSRmat(C.Structure):
    _fields_ = [("row", INT), ("col", INT), ("nnz", INT), ("IA", C.POINTER(INT)),
                ("JA", C.POINTER(INT)), ("val", C.POINTER(REAL))]


class dBSRmat(C.Structure):
    _fields_ = [("ROW", INT), ("COL", INT), ("NNZ", INT), ("nb", INT),
                ("storage_manner", INT), ("val", C.POINTER(REAL)), ("IA", C.POINTER(INT)),
                ("JA", C.POINTER(INT))]


class dvector(C.Structure):
    _fields_ = [("row", INT), ("val", C.POINTER(REAL))]


class linear_itsolver_param(C.Structure):
    _fields_ = [("linear_itsolver_type", SHORT), ("linear_precond_type", SHORT),
                ("linear_stop_type", SHORT), ("linear_maxit", INT), ("linear_tol", REAL),
                ("linear_restart", INT), ("linear_print_level", SHORT),
                ("HX_smooth_iter", SHORT), ("AL_scaling_param", REAL)]


class AMG_param(C.Structure):
    _fields_ = [("AMG_type", SHORT), ("print_level", SHORT), ("maxit", INT), ("tol", REAL),
                ("max_levels", SHORT), ("coarse_dof", INT), ("cycle_type", SHORT),
                ("smoother", SHORT), ("presmooth_iter", SHORT), ("postsmooth_iter", SHORT),
                ("relaxation", REAL), ("polynomial_degree", SHORT), ("coarse_solver", SHORT),
                ("coarse_scaling", SHORT), ("amli_degree", SHORT),
                ("amli_coef", C.POINTER(REAL)), ("nl_amli_krylov_type", SHORT),
                ("aggregation_type", SHORT), ("strong_coupled", REAL),
                ("max_aggregation", INT), ("smooth_filter", SHORT),
                ("tentative_smooth", REAL), ("Schwarz_levels", INT),
                ("Schwarz_mmsize", INT), ("Schwarz_maxlvl", INT), ("Schwarz_type", INT),
                ("Schwarz_blksolver", INT), ("HAZDIR", C.c_char_p),
                ("Schwarz_on_blk", C.POINTER(INT)), ("Schwarz_patch_type", C.POINTER(INT)),
                ("damping_param", REAL), ("BSR_alpha", REAL), ("BSR_omega", REAL),
                ("fpwr", REAL), ("smoother_function", C.c_void_p)]


class precond(C.Structure):
    _fields_ = [("data", C.c_void_p),
                ("fct", C.CFUNCTYPE(None, C.POINTER(REAL), C.POINTER(REAL), C.c_void_p)),
                ("setup_time", REAL)]


class Schwarz_data(C.Structure):
    _fields_ = [("A", dCSRmat), ("nblk", INT), ("iblock", C.POINTER(INT)),
                ("jblock", C.POINTER(INT)), ("rhsloc1", dvector), ("xloc1", dvector),
                ("Schwarz_type", SHORT), ("blk_solver", INT), ("memt", INT),
                ("mask", C.POINTER(INT)), ("maxbs", INT), ("maxbnnz", INT),
                ("blk_data", C.c_void_p), ("numeric", C.c_void_p), ("swzparam", C.c_void_p)]


class AMG_data(C.Structure):
    _fields_ = [("max_levels", SHORT), ("num_levels", SHORT), ("A", dCSRmat), ("R", dCSRmat),
                ("P", dCSRmat), ("b", dvector), ("x", dvector), ("M", dCSRmat),
                ("Numeric", C.c_void_p), ("near_kernel_dim", INT),
                ("near_kernel_basis", C.c_void_p), ("Schwarz_levels", INT),
                ("Schwarz", Schwarz_data), ("w", dvector), ("cycle_type", INT),
                ("wdata", C.c_void_p)]


class precond_data(C.Structure):
    _fields_ = [("AMG_type", SHORT), ("print_level", SHORT), ("maxit", INT),
                ("max_levels", SHORT), ("tol", REAL), ("cycle_type", SHORT),
                ("smoother", SHORT), ("presmooth_iter", SHORT), ("postsmooth_iter", SHORT),
                ("relaxation", REAL), ("polynomial_degree", SHORT), ("coarse_solver", SHORT),
                ("coarse_scaling", SHORT), ("amli_degree", SHORT),
                ("nl_amli_krylov_type", SHORT), ("amli_coef", C.POINTER(REAL)),
                ("mgl_data", C.POINTER(AMG_data)), ("fpwr", REAL), ("A", C.c_void_p),
                ("A_nk", C.c_void_p), ("P_nk", C.c_void_p), ("R_nk", C.c_void_p),
                ("r", C.c_void_p), ("w", C.POINTER(REAL))]


class hzb_param(C.Structure):
    _fields_ = [("precision", SHORT), ("gs_schedule", SHORT), ("matching", SHORT),
                ("export_hierarchy", SHORT), ("use_omega", SHORT),
                ("omega", C.POINTER(C.c_float)), ("device", INT), ("fallback_check", SHORT),
                ("use_graph", SHORT), ("reserved", SHORT * 6)]


class hzb_stats(C.Structure):
    _fields_ = [("num_levels", INT), ("rows", INT * MAX_AMG_LVL), ("nnz", INT * MAX_AMG_LVL),
                ("iterations", INT), ("final_relres", REAL), ("setup_seconds", REAL),
                ("solve_seconds", REAL), ("strong_coupled", REAL), ("condest", REAL),
                ("omega_contraction", REAL * 2), ("omega_used", INT), ("launches", INT)]


_lib = None


def lib() -> C.CDLL:
    """Load libhazb200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m hazmath_b200.build`")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.hzb_last_error.restype = C.c_char_p
        L.amg_data_create.restype = P(AMG_data)
        L.amg_setup_ua.restype = SHORT
        L.amg_setup_sa.restype = SHORT
        L.hzb_create.argtypes = [P(C.c_void_p), P(AMG_param), P(linear_itsolver_param),
                                 P(hzb_param)]
        for name in ("hzb_setup_device", "hzb_solve_device", "hzb_precond_device",
                     "hzb_set_omega_device", "hzb_level_copy", "hzb_get_stats",
                     "hzb_setup_host", "hzb_solve_host", "hzb_destroy"):
            getattr(L, name).argtypes = None
        L.hzb_setup_device.argtypes = [C.c_void_p, INT, INT, C.c_void_p, C.c_void_p, C.c_void_p]
        L.hzb_solve_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.hzb_solve_host.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.hzb_setup_host.argtypes = [C.c_void_p, P(dCSRmat)]
        L.hzb_precond_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.hzb_set_omega_device.argtypes = [C.c_void_p, C.c_void_p]
        L.hzb_level_copy.argtypes = [C.c_void_p, INT, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
        L.hzb_get_stats.argtypes = [C.c_void_p, P(hzb_stats)]
        L.hzb_level_prolongation.argtypes = [C.c_void_p, INT, C.c_void_p, C.c_void_p,
                                             C.c_void_p, P(INT)]
        L.hzb_destroy.argtypes = [C.c_void_p]
        L.hzb_bsr_setup_host.argtypes = [C.c_void_p, P(dBSRmat)]
        L.hzb_bsr_setup_device.argtypes = [C.c_void_p, INT, INT, INT, C.c_void_p, C.c_void_p,
                                           C.c_void_p]
        L.hzb_bsr_level.argtypes = [C.c_void_p, INT, P(dBSRmat), C.c_void_p]
        for name in ("hzb_bsr_precond_device", "hzb_bsr_precond_host", "hzb_bsr_solve_device",
                     "hzb_bsr_solve_host"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.linear_solver_dbsr_krylov_amg.argtypes = [P(dBSRmat), P(dvector), P(dvector),
                                                    P(linear_itsolver_param), P(AMG_param)]
        L.hzb_time_kernel.argtypes = [C.c_void_p, INT, INT, INT, P(REAL), P(REAL)]
        L.hzb_batch_setup_device.argtypes = [C.c_void_p, INT, P(INT), INT, INT, C.c_void_p,
                                             C.c_void_p, C.c_void_p]
        L.hzb_batch_solve_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, P(INT),
                                             P(REAL), P(REAL)]
        L.hzb_dcsr_aAxpy_device.argtypes = [REAL, INT, INT, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p]
        L.hzb_smoother_device.argtypes = [SHORT, SHORT, INT, REAL, INT, INT, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.hzb_aggregation_hem_device.argtypes = [INT, INT, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, REAL, C.c_void_p, P(INT)]
        L.hzb_rap_agg_device.argtypes = [INT, INT, C.c_void_p, C.c_void_p, C.c_void_p, INT,
                                         C.c_void_p, P(INT), P(C.c_void_p), P(C.c_void_p),
                                         P(C.c_void_p)]
        L.hzb_rap_agg_device_noalloc.argtypes = [INT, INT, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, INT, C.c_void_p, INT,
                                                 C.c_void_p, C.c_void_p, C.c_void_p, P(INT)]
        L.hzb_copy_to_host.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.hzb_free_device.argtypes = [C.c_void_p]
        L.dcsr_pcg.argtypes = [P(dCSRmat), P(dvector), P(dvector), P(precond), REAL, INT,
                               SHORT, SHORT]
        for name in ("dcsr_pvgmres", "dcsr_pvfgmres"):
            getattr(L, name).argtypes = [P(dCSRmat), P(dvector), P(dvector), P(precond), REAL,
                                         INT, SHORT, SHORT, SHORT]
        for name in ("dcsr_pgcg", "dcsr_pminres"):
            getattr(L, name).argtypes = [P(dCSRmat), P(dvector), P(dvector), P(precond), REAL,
                                         INT, SHORT, SHORT]
        L.hzb_assemble_p1_kuhn_device.argtypes = [INT, C.c_void_p, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_void_p, P(INT)]
        L.amg_amli_coef.argtypes = [REAL, REAL, INT, P(REAL)]
        L.amg_amli_coef.restype = None
        for name in ("precond_amg", "precond_amli", "precond_nl_amli", "precond_amg_add"):
            getattr(L, name).restype = None
        for name in ("amli", "nl_amli", "mgcycle_add", "mgcycle"):
            getattr(L, name).restype = None
        L.python_wrapper_krylov_amg.argtypes = [P(INT), P(INT), C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.c_void_p, C.c_void_p, P(REAL),
                                                P(INT), P(INT)]
        _lib = L
    return _lib


def last_error() -> str:
    return lib().hzb_last_error().decode()


def declared_symbols(header: str = HEADER) -> list[str]:
    """Function names declared in include/hazmath_b200.h."""
    import re
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    # declarations start in column 0; struct fields are indented
    names = re.findall(r"^(?:const\s+)?[A-Za-z_][A-Za-z_0-9]*\s*\**\s*([A-Za-z_][A-Za-z_0-9]*)\s*\(",
                       text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "return")))


# ---------------------------------------------------------------------------
# parameter helpers (HAZmath's init functions, run in the library)
# ---------------------------------------------------------------------------
def amg_param(**kw) -> AMG_param:
    """AMG_param from param_amg_init, then keyword overrides."""
    p = AMG_param()
    lib().param_amg_init(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def itsolver_param(**kw) -> linear_itsolver_param:
    p = linear_itsolver_param()
    lib().param_linear_solver_init(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def b200_param(**kw) -> hzb_param:
    p = hzb_param()
    lib().hzb_param_init(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def bench_amg(**kw) -> AMG_param:
    """The UA-AMG setting of the benchmark configurations: HEM, theta = 0,
    V(1,1) Gauss-Seidel, coarse direct solve at <= 2000 rows."""
    base = dict(AMG_type=UA_AMG, cycle_type=V_CYCLE, smoother=SMOOTHER_GS,
                presmooth_iter=1, postsmooth_iter=1, aggregation_type=HEM,
                strong_coupled=0.0, max_aggregation=20, coarse_dof=2000, max_levels=20,
                coarse_solver=SOLVER_UMFPACK, maxit=1, tol=1e-6)
    base.update(kw)
    return amg_param(**base)


class _HostCSR:
    """Keeps numpy arrays alive behind a dCSRmat."""

    def __init__(self, ia, ja, val):
        self.ia = np.ascontiguousarray(ia, np.int32)
        self.ja = np.ascontiguousarray(ja, np.int32)
        self.val = np.ascontiguousarray(val, np.float64)
        n = len(self.ia) - 1
        self.mat = dCSRmat(n, n, int(self.ia[-1]), self.ia.ctypes.data_as(C.POINTER(INT)),
                           self.ja.ctypes.data_as(C.POINTER(INT)),
                           self.val.ctypes.data_as(C.POINTER(REAL)))


def _dvec(a: np.ndarray) -> dvector:
    return dvector(len(a), a.ctypes.data_as(C.POINTER(REAL)))


# ---------------------------------------------------------------------------
# drop-in calls on numpy arrays (host pointers, as the reference takes them)
# ---------------------------------------------------------------------------
def linear_solver_dcsr_krylov_amg(ia, ja, val, b, x, itparam, amgparam, b200=None):
    """itsolver.c:846 semantics; x (float64 array) is updated in place.
    Returns the iteration count or a negative ERROR_* code."""
    A = _HostCSR(ia, ja, val)
    assert x.dtype == np.float64 and x.flags.c_contiguous
    bb = np.ascontiguousarray(b, np.float64)
    if b200 is None:
        return lib().linear_solver_dcsr_krylov_amg(C.byref(A.mat), C.byref(_dvec(bb)),
                                                   C.byref(_dvec(x)), C.byref(itparam),
                                                   C.byref(amgparam))
    return lib().hzb_solver_dcsr_krylov_amg(C.byref(A.mat), C.byref(_dvec(bb)),
                                            C.byref(_dvec(x)), C.byref(itparam),
                                            C.byref(amgparam), C.byref(b200))


class _HostBSR:
    """Keeps numpy arrays alive behind a dBSRmat (blocks row-major)."""

    def __init__(self, nb, ia, ja, val):
        self.ia = np.ascontiguousarray(ia, np.int32)
        self.ja = np.ascontiguousarray(ja, np.int32)
        self.val = np.ascontiguousarray(val, np.float64)
        n = len(self.ia) - 1
        self.mat = dBSRmat(n, n, int(self.ia[-1]), int(nb), 0,
                           self.val.ctypes.data_as(C.POINTER(REAL)),
                           self.ia.ctypes.data_as(C.POINTER(INT)),
                           self.ja.ctypes.data_as(C.POINTER(INT)))


def linear_solver_dbsr_krylov_amg(nb, ia, ja, val, b, x, itparam, amgparam):
    """itsolver.c:2104 semantics on a block matrix of nb x nb blocks; x
    (float64 array, ROW * nb) is updated in place.  Returns the iteration
    count or a negative ERROR_* code."""
    A = _HostBSR(nb, ia, ja, val)
    assert x.dtype == np.float64 and x.flags.c_contiguous
    bb = np.ascontiguousarray(b, np.float64)
    return lib().linear_solver_dbsr_krylov_amg(C.byref(A.mat), C.byref(_dvec(bb)),
                                               C.byref(_dvec(x)), C.byref(itparam),
                                               C.byref(amgparam))


def linear_solver_amg(ia, ja, val, b, x, amgparam):
    A = _HostCSR(ia, ja, val)
    bb = np.ascontiguousarray(b, np.float64)
    return lib().linear_solver_amg(C.byref(A.mat), C.byref(_dvec(bb)), C.byref(_dvec(x)),
                                   C.byref(amgparam))


def python_wrapper_krylov_amg(ia, ja, val, b, u, tol=1e-8, maxit=500, print_lvl=0):
    ia = np.ascontiguousarray(ia, np.int32)
    ja = np.ascontiguousarray(ja, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    n, nnz = INT(len(ia) - 1), INT(int(ia[-1]))
    lib().python_wrapper_krylov_amg(C.byref(n), C.byref(nnz), ia.ctypes.data, ja.ctypes.data,
                                    val.ctypes.data, b.ctypes.data, u.ctypes.data,
                                    C.byref(REAL(tol)), C.byref(INT(maxit)),
                                    C.byref(INT(print_lvl)))


def assemble_p1_kuhn_device(N: int, kcell_ptr, ia_ptr, ja_ptr=None, val_ptr=None, K=None):
    """hzb_assemble_p1_kuhn_device on device pointers: the interior-dof P1
    stiffness on the Kuhn mesh of N^3 cubes.  Returns (status, nnz); ja/val
    are filled when both pointers are given."""
    nnz = INT()
    Kp = None
    if K is not None:
        Kh = np.ascontiguousarray(K, np.float64).reshape(9)
        Kp = Kh.ctypes.data_as(C.c_void_p)
    rc = lib().hzb_assemble_p1_kuhn_device(N, kcell_ptr, Kp, ia_ptr, ja_ptr, val_ptr,
                                           C.byref(nnz))
    return rc, nnz.value


# the preconditioner linear_solver_dcsr_krylov_amg picks for a cycle type
_PRECOND_OF_CYCLE = {AMLI_CYCLE: "precond_amli", NL_AMLI_CYCLE: "precond_nl_amli",
                     ADD_CYCLE: "precond_amg_add"}


def amli_coef(lambda_max: float, lambda_min: float, degree: int) -> np.ndarray:
    """amg_amli_coef: the degree + 1 coefficients of the AMLI polynomial."""
    c = np.zeros(degree + 1)
    lib().amg_amli_coef(lambda_max, lambda_min, degree, c.ctypes.data_as(C.POINTER(REAL)))
    return c


class AMGHierarchy:
    """amg_data_create + amg_setup_ua on a host matrix; the pieces a caller
    assembles itself (HAZNICS create_precond_amg style): the preconditioner
    of the cycle type (precond_amg, precond_amli, precond_nl_amli or
    precond_amg_add) for dcsr_pcg / dcsr_pgcg / dcsr_pv(f)gmres, the cycles,
    amg_data_free."""

    def __init__(self, ia, ja, val, amgparam: AMG_param, smoothed: bool = False):
        """smoothed: amg_setup_sa instead of amg_setup_ua."""
        self._A = _HostCSR(ia, ja, val)
        self.param = amgparam
        L = lib()
        self.mgl = L.amg_data_create(amgparam.max_levels)
        self.mgl[0].A = self._A.mat   # the caller's arrays, as dcsr_cp'd in the reference
        self._owned_A0 = True
        setup = L.amg_setup_sa if smoothed else L.amg_setup_ua
        self.status = setup(self.mgl, C.byref(amgparam))
        self.pcdata = precond_data()
        L.precond_data_null(C.byref(self.pcdata))
        L.param_amg_to_prec(C.byref(self.pcdata), C.byref(amgparam))
        self.pcdata.max_levels = self.mgl[0].num_levels
        self.pcdata.mgl_data = self.mgl
        self.pc = precond()
        self.pc.data = C.cast(C.pointer(self.pcdata), C.c_void_p)
        self.pc_name = _PRECOND_OF_CYCLE.get(amgparam.cycle_type, "precond_amg")
        self.pc.fct = C.cast(getattr(L, self.pc_name), type(self.pc.fct))

    @property
    def num_levels(self) -> int:
        return self.mgl[0].num_levels

    def level(self, l: int):
        A = self.mgl[l].A
        n, nnz = A.row, A.nnz
        ia = np.ctypeslib.as_array(A.IA, (n + 1,)).copy()
        ja = np.ctypeslib.as_array(A.JA, (nnz,)).copy()
        val = np.ctypeslib.as_array(A.val, (nnz,)).copy()
        return ia, ja, val

    def agg(self, l: int):
        P = self.mgl[l].P
        ia = np.ctypeslib.as_array(P.IA, (P.row + 1,))
        ja = np.ctypeslib.as_array(P.JA, (max(P.nnz, 1),))
        out = np.full(P.row, -1, np.int32)
        has = ia[1:] > ia[:-1]
        out[has] = ja[ia[:-1][has]]
        return out

    def precond(self, r):
        r = np.ascontiguousarray(r, np.float64).copy()
        z = np.zeros_like(r)
        getattr(lib(), self.pc_name)(r.ctypes.data_as(C.POINTER(REAL)),
                                     z.ctypes.data_as(C.POINTER(REAL)),
                                     C.cast(C.pointer(self.pcdata), C.c_void_p))
        return z

    def cycle(self, b, x):
        """One cycle of the setup's cycle type on mgl[0].b / mgl[0].x
        (mgcycle, amli, nl_amli or mgcycle_add); returns the new x."""
        n = self.mgl[0].A.row
        bb = np.ascontiguousarray(b, np.float64).copy()
        xx = np.ascontiguousarray(x, np.float64).copy()
        m0 = self.mgl[0]
        # copies: a ctypes field read is a view into mgl[0]
        sb, sx = dvector(m0.b.row, m0.b.val), dvector(m0.x.row, m0.x.val)
        self.mgl[0].b = _dvec(bb)
        self.mgl[0].x = _dvec(xx)
        ct = self.param.cycle_type
        L = lib()
        if ct == AMLI_CYCLE:
            L.amli(self.mgl, C.byref(self.param), 0)
        elif ct == NL_AMLI_CYCLE:
            L.nl_amli(self.mgl, C.byref(self.param), 0, self.num_levels)
        elif ct == ADD_CYCLE:
            L.mgcycle_add(self.mgl, C.byref(self.param))
        else:
            L.mgcycle(self.mgl, C.byref(self.param))
        self.mgl[0].b, self.mgl[0].x = sb, sx
        assert n == len(xx)
        return xx

    def minres(self, b, x, tol=1e-8, maxit=500, stop_type=STOP_REL_RES, prtlvl=0):
        """dcsr_pminres with the setup's preconditioner."""
        bb = np.ascontiguousarray(b, np.float64)
        return lib().dcsr_pminres(C.byref(self._A.mat), C.byref(_dvec(bb)), C.byref(_dvec(x)),
                                  C.byref(self.pc), tol, maxit, stop_type, prtlvl)

    def gcg(self, b, x, tol=1e-8, maxit=100, stop_type=STOP_REL_RES, prtlvl=0):
        """dcsr_pgcg with the setup's preconditioner."""
        bb = np.ascontiguousarray(b, np.float64)
        return lib().dcsr_pgcg(C.byref(self._A.mat), C.byref(_dvec(bb)), C.byref(_dvec(x)),
                               C.byref(self.pc), tol, maxit, stop_type, prtlvl)

    def pcg(self, b, x, tol=1e-8, maxit=500, stop_type=STOP_REL_RES, prtlvl=0):
        bb = np.ascontiguousarray(b, np.float64)
        return lib().dcsr_pcg(C.byref(self._A.mat), C.byref(_dvec(bb)), C.byref(_dvec(x)),
                              C.byref(self.pc), tol, maxit, stop_type, prtlvl)

    def gmres(self, b, x, tol=1e-8, maxit=500, restart=100, flexible=True,
              stop_type=STOP_REL_RES, prtlvl=0):
        """dcsr_pvfgmres (flexible) or dcsr_pvgmres with the setup's
        preconditioner."""
        bb = np.ascontiguousarray(b, np.float64)
        f = lib().dcsr_pvfgmres if flexible else lib().dcsr_pvgmres
        return f(C.byref(self._A.mat), C.byref(_dvec(bb)), C.byref(_dvec(x)),
                 C.byref(self.pc), C.c_double(tol), maxit, restart, stop_type, prtlvl)

    def free(self):
        if self.mgl:
            # level 0 A belongs to the caller here: detach before freeing
            self.mgl[0].A = dCSRmat()
            lib().amg_data_free(self.mgl, C.byref(self.param))
            self.mgl = None


class Solver:
    """Persistent device handle (hzb_create / hzb_setup_* / hzb_solve_*)."""

    def __init__(self, amg: AMG_param | None = None, it: linear_itsolver_param | None = None,
                 b200: hzb_param | None = None):
        self.amg = amg or bench_amg()
        self.it = it or itsolver_param(linear_itsolver_type=SOLVER_CG,
                                       linear_precond_type=PREC_AMG, linear_tol=1e-8,
                                       linear_maxit=500)
        self.b200 = b200 or b200_param()
        h = C.c_void_p()
        rc = lib().hzb_create(C.byref(h), C.byref(self.amg), C.byref(self.it),
                              C.byref(self.b200))
        if rc:
            raise RuntimeError(f"hzb_create: {rc} {last_error()}")
        self.h = h
        self._keep = None

    def setup_device(self, n, nnz, ia_ptr, ja_ptr, val_ptr) -> int:
        return lib().hzb_setup_device(self.h, n, nnz, ia_ptr, ja_ptr, val_ptr)

    def setup_host(self, ia, ja, val) -> int:
        self._keep = _HostCSR(ia, ja, val)
        return lib().hzb_setup_host(self.h, C.byref(self._keep.mat))

    def solve_device(self, b_ptr, x_ptr) -> int:
        return lib().hzb_solve_device(self.h, b_ptr, x_ptr)

    def solve_host(self, b, x) -> int:
        bb = np.ascontiguousarray(b, np.float64)
        return lib().hzb_solve_host(self.h, bb.ctypes.data, x.ctypes.data)

    def precond_device(self, r_ptr, z_ptr) -> int:
        return lib().hzb_precond_device(self.h, r_ptr, z_ptr)

    def batch_setup_device(self, off, nnz, ia_ptr, ja_ptr, val_ptr) -> int:
        """Hierarchy of the block-diagonal union of len(off) - 1 systems
        (rows of system k: off[k] .. off[k+1]-1)."""
        self._off = np.ascontiguousarray(off, np.int32)
        ns = len(self._off) - 1
        return lib().hzb_batch_setup_device(self.h, ns, self._off.ctypes.data_as(
            C.POINTER(INT)), int(self._off[-1]), nnz, ia_ptr, ja_ptr, val_ptr)

    def batch_solve_device(self, b_ptr, x_ptr):
        """Per-system flexible CG: (return code, iterations, relative
        residuals, seconds from the solve's start to each system's
        convergence)."""
        ns = len(self._off) - 1
        its = np.zeros(ns, np.int32)
        rel = np.zeros(ns)
        sec = np.zeros(ns)
        rc = lib().hzb_batch_solve_device(self.h, b_ptr, x_ptr,
                                          its.ctypes.data_as(C.POINTER(INT)),
                                          rel.ctypes.data_as(C.POINTER(REAL)),
                                          sec.ctypes.data_as(C.POINTER(REAL)))
        return rc, its, rel, sec

    def set_omega_device(self, omega_ptr) -> int:
        return lib().hzb_set_omega_device(self.h, omega_ptr)

    def stats(self) -> hzb_stats:
        st = hzb_stats()
        lib().hzb_get_stats(self.h, C.byref(st))
        return st

    def level(self, l: int):
        st = self.stats()
        n, nnz = st.rows[l], st.nnz[l]
        ia = np.empty(n + 1, np.int32)
        ja = np.empty(nnz, np.int32)
        val = np.empty(nnz)
        agg = np.empty(n, np.int32)
        rc = lib().hzb_level_copy(self.h, l, ia.ctypes.data, ja.ctypes.data, val.ctypes.data,
                                  agg.ctypes.data)
        if rc:
            raise RuntimeError(f"hzb_level_copy: {rc} {last_error()}")
        return ia, ja, val, agg

    def prolongation(self, l: int):
        """The smoothed prolongation of level l as (ia, ja, val), or None for
        an unsmoothed level."""
        n = self.stats().rows[l]
        nnz = INT()
        rc = lib().hzb_level_prolongation(self.h, l, None, None, None, C.byref(nnz))
        if rc:
            raise RuntimeError(f"hzb_level_prolongation: {rc} {last_error()}")
        if nnz.value == 0:
            return None
        ia = np.empty(n + 1, np.int32)
        ja = np.empty(nnz.value, np.int32)
        val = np.empty(nnz.value)
        lib().hzb_level_prolongation(self.h, l, ia.ctypes.data, ja.ctypes.data, val.ctypes.data,
                                     C.byref(nnz))
        return ia, ja, val

    # -- block (BSR) matrices -------------------------------------------
    def setup_bsr_host(self, nb, ia, ja, val) -> int:
        """amg_setup_ua_bsr on the device for a host block matrix."""
        self._keep_bsr = _HostBSR(nb, ia, ja, val)
        return lib().hzb_bsr_setup_host(self.h, C.byref(self._keep_bsr.mat))

    def setup_bsr_device(self, nrow, nnzb, nb, ia_ptr, ja_ptr, val_ptr) -> int:
        return lib().hzb_bsr_setup_device(self.h, nrow, nnzb, nb, ia_ptr, ja_ptr, val_ptr)

    def time_kernel(self, which: int, level: int, reps: int):
        """(ms per launch, algorithmic bytes per launch) of hzb_time_kernel."""
        ms, by = REAL(), REAL()
        rc = lib().hzb_time_kernel(self.h, which, level, reps, C.byref(ms), C.byref(by))
        if rc:
            raise RuntimeError(f"hzb_time_kernel: {rc} {last_error()}")
        return ms.value, by.value

    def bsr_level(self, l: int):
        """Block matrix of level l as (ia, ja, val) and its block
        aggregates (None on the coarsest level)."""
        m = dBSRmat()
        rc = lib().hzb_bsr_level(self.h, l, C.byref(m), None)
        if rc:
            raise RuntimeError(f"hzb_bsr_level: {rc} {last_error()}")
        n, nnzb, nb = m.ROW, m.NNZ, m.nb
        ia = np.empty(n + 1, np.int32)
        ja = np.empty(nnzb, np.int32)
        val = np.empty(nnzb * nb * nb)
        agg = np.empty(n, np.int32)
        m.IA = ia.ctypes.data_as(C.POINTER(INT))
        m.JA = ja.ctypes.data_as(C.POINTER(INT))
        m.val = val.ctypes.data_as(C.POINTER(REAL))
        last = l == self.stats().num_levels - 1
        rc = lib().hzb_bsr_level(self.h, l, C.byref(m), None if last else agg.ctypes.data)
        if rc:
            raise RuntimeError(f"hzb_bsr_level: {rc} {last_error()}")
        return ia, ja, val, (None if last else agg)

    def bsr_precond_host(self, r):
        rr = np.ascontiguousarray(r, np.float64)
        z = np.zeros_like(rr)
        rc = lib().hzb_bsr_precond_host(self.h, rr.ctypes.data, z.ctypes.data)
        if rc:
            raise RuntimeError(f"hzb_bsr_precond_host: {rc} {last_error()}")
        return z

    def bsr_precond_device(self, r_ptr, z_ptr) -> int:
        return lib().hzb_bsr_precond_device(self.h, r_ptr, z_ptr)

    def bsr_solve_device(self, b_ptr, x_ptr) -> int:
        return lib().hzb_bsr_solve_device(self.h, b_ptr, x_ptr)

    def bsr_solve_host(self, b, x) -> int:
        bb = np.ascontiguousarray(b, np.float64)
        return lib().hzb_bsr_solve_host(self.h, bb.ctypes.data, x.ctypes.data)

    def close(self):
        if self.h:
            lib().hzb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
