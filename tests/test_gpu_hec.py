"""HEC aggregation on the device (aggregation_type 4, the reference's
default; aggregation_hec, amg_setup_ua.c:752-845): the row order comes from
glibc's rand() (iarray_shuffle, array.c:302-315), which the reference never
seeds, so a fresh process draws from srand(1).  Every setup here starts from
srand(1), and its hierarchy must be the reference's first setup in a fresh
process bit for bit (tests/golden/hec.npz, made with srand(1)): level sizes,
every aggregate map, every coarse operator (SHA-256), the adapted threshold.
Then a PCG solve with that hierarchy converges like the reference's
preconditioner does."""
import hashlib

import numpy as np
import pytest

import hazmath_b200 as hz
from hazmath_b200 import problems as P

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _matrix(golden, name):
    if name == "fix":
        return P.poisson2d_5pt(128)
    g = golden("gmres.npz")
    return g["kuhn/A_ia"], g["kuhn/A_ja"], g["kuhn/A_val"]


@pytest.mark.parametrize("name", ["fix", "kuhn"])
def test_hec_hierarchy_matches_fresh_process_reference(golden, name):
    g = golden("hec.npz")
    ia, ja, val = _matrix(golden, name)
    amg = hz.bench_amg(aggregation_type=hz.HEC, strong_coupled=0.04, coarse_dof=100)
    S = hz.Solver(amg)
    assert S.setup_host(ia, ja, val) == 0, hz.last_error()
    st = S.stats()
    info = g[f"{name}/info"]
    assert st.num_levels == len(info)
    for l in range(st.num_levels):
        assert (st.rows[l], st.nnz[l]) == (info[l][0], info[l][1]), l
        lia, lja, lval, agg = S.level(l)
        assert [sha(lia), sha(lja), sha(lval)] == list(g[f"{name}/A{l}_sha"]), l
        if l < st.num_levels - 1:
            assert np.array_equal(agg, g[f"{name}/agg{l}"]), l
    assert st.strong_coupled == float(g[f"{name}/theta_after"])
    b = P.rhs_uniform(len(ia) - 1, 5)
    x = np.zeros(len(b))
    it = S.solve_host(b, x)
    assert 0 < it < 200, (it, hz.last_error())
    assert S.stats().final_relres < 1e-8
    S.close()


def test_hec_each_setup_starts_from_srand1(golden):
    """A second setup draws its permutation from srand(1) again, so with the
    same threshold it repeats the first hierarchy bit for bit (a handle keeps
    the adapted threshold as the reference's caller-owned AMG_param does, so
    this uses theta = 0, which the adaptation leaves unchanged)."""
    ia, ja, val = _matrix(golden, "kuhn")
    amg = hz.bench_amg(aggregation_type=hz.HEC, strong_coupled=0.0, coarse_dof=100)
    S = hz.Solver(amg)
    maps = []
    for _ in range(2):
        assert S.setup_host(ia, ja, val) == 0, hz.last_error()
        st = S.stats()
        maps.append([S.level(l)[3] for l in range(st.num_levels - 1)])
    assert len(maps[0]) == len(maps[1]) >= 2
    for a, b in zip(*maps):
        assert np.array_equal(a, b)
    S.close()
