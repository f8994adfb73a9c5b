"""HEC aggregation (aggregation_type 4, the reference's default): the
reference draws its row order from the C library's rand() (iarray_shuffle,
array.c:302), so a run is reproducible once the stream is seeded.  The
oracle restates glibc's generator (or_srand / or_rand) and the HEC walk
(or_hec); these tests pin the generator to the system's rand() and the
aggregate maps of every level to the reference's (tests/golden/hec.npz,
made with srand(1), i.e. a fresh process)."""
import ctypes
import ctypes.util

import numpy as np
import pytest

import oracle
from conftest import small_case


def _libc():
    name = ctypes.util.find_library("c")
    return ctypes.CDLL(name) if name else None


def test_rand_stream_is_the_c_librarys():
    libc = _libc()
    if libc is None or "libc.so.6" not in str(ctypes.util.find_library("c")):
        pytest.skip("not a glibc system")
    P = oracle.port()
    for seed in (1, 0, 12345, 2 ** 31 + 7):
        libc.srand(ctypes.c_uint(seed))
        P.srand(seed)
        want = [libc.rand() for _ in range(2000)]
        assert [P.rand() for _ in range(2000)] == want, seed


def _levels(port, ia, ja, val, info, theta):
    """Run the oracle's HEC level by level on the coarse operators that the
    oracle's own Galerkin product makes from the maps, with the threshold
    adapting as amg_setup_ua does."""
    port.srand(1)
    got = []
    for l in range(len(info) - 1):
        nc, agg = port.hec(ia, ja, val, theta=theta)
        got.append(agg)
        n = len(ia) - 1
        if nc * 4 > n:
            theta /= 2
        elif nc * 1.25 < n:
            theta *= 2
        ia, ja, val = port.rap(ia, ja, val, nc, agg)
    return got, theta


@pytest.mark.parametrize("case", ["fix", "kuhn"])
def test_oracle_hec_matches_reference_every_level(golden, port, case):
    A = small_case(golden("gmres.npz"), case)
    v = small_case(golden("hec.npz"), case)
    info = v["info"]
    got, theta = _levels(port, A["A_ia"], A["A_ja"], A["A_val"], info, 0.04)
    for l, agg in enumerate(got):
        np.testing.assert_array_equal(agg, v[f"agg{l}"], err_msg=f"level {l}")
    assert theta == float(v["theta_after"])
