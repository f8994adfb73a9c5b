"""CPU checks of the drop-in boundary: the library loads and exports every
function include/hazmath_b200.h declares, the structures have the reference's
layout, and the host-only parameter functions keep HAZmath's defaults."""
import ctypes as C
import json
import os
import subprocess
import tempfile

import pytest

import hazmath_b200 as hz
from conftest import GOLDEN, ROOT


@pytest.fixture(scope="module")
def lib():
    from hazmath_b200 import build
    build.build()
    return hz.lib()


def test_exports_every_declared_symbol(lib):
    names = hz.declared_symbols()
    assert "linear_solver_dcsr_krylov_amg" in names and "hzb_solve_device" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_mirror_sizes():
    lay = json.load(open(os.path.join(GOLDEN, "layout.json")))
    for name, cls in [("dCSRmat", hz.dCSRmat), ("dvector", hz.dvector),
                      ("linear_itsolver_param", hz.linear_itsolver_param),
                      ("AMG_param", hz.AMG_param), ("precond", hz.precond),
                      ("Schwarz_data", hz.Schwarz_data), ("AMG_data", hz.AMG_data),
                      ("precond_data", hz.precond_data)]:
        assert C.sizeof(cls) == lay[f"sizeof({name})"], name


def test_header_layout_matches_reference():
    """Compile a probe against include/hazmath_b200.h and compare every
    sizeof/offsetof with the values recorded from the reference headers."""
    lay = json.load(open(os.path.join(GOLDEN, "layout.json")))
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "hazmath_b200.h"',
             "int main(){"]
    for key in lay:
        if key.startswith("sizeof("):
            t = key[7:-1]
            lines.append(f'printf("%s %zu\\n", "{key}", sizeof({t}));')
        else:
            t, f = key.split(".")
            lines.append(f'printf("%s %zu\\n", "{key}", offsetof({t},{f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "p.c"), os.path.join(d, "p")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    got = {k: int(v) for k, v in (ln.split() for ln in out.strip().splitlines())}
    assert got == lay


def test_param_defaults(lib):
    """param_amg_init / param_linear_solver_init / precond_data_null values
    of parameters.c:158-250 and data.c:22-55."""
    p = hz.amg_param()
    assert (p.AMG_type, p.maxit, p.tol, p.max_levels, p.coarse_dof, p.cycle_type) == \
        (1, 1, 1e-6, 10, 200, 2)
    assert (p.smoother, p.presmooth_iter, p.postsmooth_iter, p.coarse_solver) == (2, 1, 1, 0)
    assert (p.aggregation_type, p.strong_coupled, p.max_aggregation) == (4, 0.04, 20)
    it = hz.itsolver_param()
    assert (it.linear_itsolver_type, it.linear_precond_type, it.linear_stop_type,
            it.linear_maxit, it.linear_restart, it.linear_tol) == (4, 0, 1, 500, 100, 1e-6)
    d = hz.precond_data()
    lib.precond_data_null(C.byref(d))
    assert (d.maxit, d.max_levels, d.tol, d.cycle_type, d.relaxation, d.coarse_solver) == \
        (100, 20, 1e-8, 1, 1.2, 32)
    lib.param_amg_to_prec(C.byref(d), C.byref(p))
    assert (d.maxit, d.tol, d.cycle_type, d.coarse_solver) == (1, 1e-6, 2, 0)
    q = hz.amg_param(cycle_type=1, tol=5.0, maxit=7)
    lib.param_prec_to_amg(C.byref(q), C.byref(d))
    assert q.cycle_type == 2 and q.tol == 5.0 and q.maxit == 7   # tol, maxit not copied


def test_amg_data_create_free(lib):
    mgl = lib.amg_data_create(5)
    assert mgl[0].max_levels == 5 and mgl[4].max_levels == 5 and mgl[0].num_levels == 0
    p = hz.amg_param()
    lib.amg_data_free(mgl, C.byref(p))


def test_entry_points_fail_loudly_without_a_device(lib):
    """On a machine without a usable GPU the drop-in entry points return
    ERROR_SOLVER_MISC with the CUDA error text: there is no CPU path to fall
    back on."""
    import numpy as np
    import torch
    from hazmath_b200 import problems as P
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ia, ja, val = P.poisson2d_5pt(16)
    b = np.ones(len(ia) - 1)
    x = np.zeros_like(b)
    it = hz.itsolver_param(linear_itsolver_type=hz.SOLVER_CG)
    assert hz.linear_solver_dcsr_krylov_amg(ia, ja, val, b, x, it, hz.bench_amg()) == \
        hz.ERROR_SOLVER_MISC
    assert "CUDA" in hz.last_error()
    assert hz.linear_solver_dbsr_krylov_amg(1, ia, ja, val, b, x, it, hz.bench_amg()) == \
        hz.ERROR_SOLVER_MISC
    assert not x.any()
