"""The FP32 cycle's sliced-ELL schedule against the staged row bundles.

Both sum every row of a level in CSR order in FP32, one thread per row (the
bundles from shared memory, the sliced copy from its column-major slices), so
the mixed solve takes the same iterates bit for bit whichever of the two the
levels run.  HZB_FP32_LANES forces the schedule of every level of at least
4096 rows ("sell") or the bundles everywhere ("0").  The coarse levels of the
Kuhn hierarchy have ragged rows (4 to ~30 entries), so the slices carry
padding that the kernels must not read."""
import numpy as np
import pytest
import scipy.sparse as sp

import hazmath_b200 as hz
from hazmath_b200 import problems as P

pytestmark = pytest.mark.gpu


def mixed_solve(monkeypatch, schedule, ia, ja, val, b):
    monkeypatch.setenv("HZB_FP32_LANES", schedule)
    S = hz.Solver(hz.bench_amg(smoother=hz.SMOOTHER_L1DIAG, presmooth_iter=2,
                               postsmooth_iter=2),
                  b200=hz.b200_param(precision=hz.HZB_PREC_MIXED))
    assert S.setup_host(ia, ja, val) == 0, hz.last_error()
    x = np.zeros(len(b))
    it = S.solve_host(b, x)
    st = S.stats()
    levels = [(int(st.rows[l]), int(st.nnz[l])) for l in range(st.num_levels)]
    S.close()
    return it, x, levels


@pytest.mark.parametrize("N,sigma", [(24, 1.0), (40, 1.5)])
def test_sell_matches_bundles_bitwise(monkeypatch, N, sigma):
    ia, ja, val = P.kuhn3d_p1(N, P.lognormal_field(N, sigma, 8.0, 7))
    b = P.rhs_uniform(len(ia) - 1, 8)
    it_s, x_s, lv_s = mixed_solve(monkeypatch, "sell", ia, ja, val, b)
    it_b, x_b, lv_b = mixed_solve(monkeypatch, "0", ia, ja, val, b)
    assert lv_s == lv_b
    assert sum(1 for n, _ in lv_s if n >= 4096) >= 2   # the sliced copy ran on 2+ levels
    assert it_s == it_b > 0
    assert np.array_equal(x_s, x_b)
    A = sp.csr_matrix((val, ja, ia), shape=(len(b), len(b)))
    assert np.linalg.norm(b - A @ x_s) / np.linalg.norm(b) < 1e-8
