"""The reference's own C driver, relinked against the drop-in.

examples/solvers/solvers.c of the reference (solvers.c:105-118 calls
linear_solver_dcsr_krylov_amg on the matrix and right-hand side it reads) is
compiled once and linked three ways by oracle/build_relink.sh: against the
reference library alone, with -lhazb200 before the shared reference library,
and with -lhazb200 before a copy of the static archive whose drop-in names
are made local.  Run on the reference's known-answer case (A.dat / b.dat:
the 128 x 128 five-point Laplacian) with a committed input.dat (CG, UA-AMG,
HEM, theta 0, V(1,1) Gauss-Seidel, direct coarsest solve, tol 1e-8), the
relinked drivers must print the reference's iteration table: the same
number of iterations (15) and the same residuals to the printed digits.

The reference-only driver ends with exit status 252 after its table: its CG
estimates the condition number through LAPACK, which this build lacks
(krylov.c:704).  The drop-in estimates it itself and returns 0, which also
shows that the relinked drivers ran libhazb200.so's entry point."""
import os
import re
import subprocess

import numpy as np
import pytest

from hazmath_b200 import problems as P

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
ROW = re.compile(r"^\s*(\d+) \|\s+([0-9.eE+-]+)\s+\|\s+([0-9.eE+-]+)\s+\|")


def write_case(d, golden):
    ia, ja, val = P.poisson2d_5pt(128)
    n = len(ia) - 1
    rows = np.repeat(np.arange(n), np.diff(ia))
    with open(os.path.join(d, "A.dat"), "w") as f:
        f.write(f"{n} {n} {len(ja)}\n")
        for i, j, v in zip(rows, ja, val):
            f.write(f"{i} {j} {v:.15e}\n")
    b = golden("fixture128.npz")["b"]
    with open(os.path.join(d, "b.dat"), "w") as f:
        f.write(f"{n}\n")
        for v in b:
            f.write(f"{v:.17g}\n")
    with open(os.path.join(ROOT, "tests", "golden", "solvers_input.dat")) as src, \
            open(os.path.join(d, "input.dat"), "w") as dst:
        dst.write(src.read())


def table(out):
    return [(int(m.group(1)), float(m.group(2)), float(m.group(3)))
            for m in (ROW.match(line) for line in out.splitlines()) if m]


def run(exe, d):
    # the driver prints a freed file-name buffer (solvers.c:73, :79), so its
    # output is not guaranteed to be valid UTF-8
    p = subprocess.run([os.path.join(REF_DIR, exe), "A.dat", "b.dat"], cwd=d,
                       capture_output=True, timeout=300)
    return p.returncode, p.stdout.decode("utf-8", errors="replace")


@pytest.mark.parametrize("exe", ["solvers_b200", "solvers_b200_static"])
def test_relinked_reference_driver(tmp_path, golden, exe):
    for b in ("solvers_ref", exe):
        if not os.path.exists(os.path.join(REF_DIR, b)):
            pytest.skip(f"oracle/_ref/{b} not built (oracle/build_relink.sh)")
    d = str(tmp_path)
    write_case(d, golden)
    rc_ref, out_ref = run("solvers_ref", d)
    rc, out = run(exe, d)
    assert rc_ref == 252, out_ref[-2000:]
    assert rc == 0, out[-2000:]
    t_ref, t = table(out_ref), table(out)
    assert len(t_ref) == 16 and t_ref[-1][0] == 15
    assert [r[0] for r in t] == [r[0] for r in t_ref]
    for (_, rel_a, abs_a), (_, rel_b, abs_b) in zip(t, t_ref):
        assert abs(rel_a - rel_b) <= 1e-6 * rel_b, (rel_a, rel_b)
        assert abs(abs_a - abs_b) <= 1e-6 * abs_b, (abs_a, abs_b)
