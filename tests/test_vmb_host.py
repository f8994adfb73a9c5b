"""The CPU oracle's VMB aggregation (oracle/hzoracle.c or_vmb, a restatement
of aggregation_vmb) against the reference's level-0 aggregate maps in
tests/golden/vmb.npz: the restatement is pinned, and the fixture the GPU
tests read is what the reference produced."""
import numpy as np
import pytest

from conftest import small_case

CAP = {"fix/vmb": 20, "fix/vmb4": 4, "kuhn/vmb": 20, "kuhn/vmb_t": 20, "kuhn/vmb_w": 9}


@pytest.mark.parametrize("key", sorted(CAP))
def test_oracle_vmb_matches_reference(golden, port, key):
    A = small_case(golden("gmres.npz"), key.split("/")[0])
    v = small_case(golden("vmb.npz"), key)
    assert int(v["params"][8]) == CAP[key]
    nc, agg = port.vmb(A["A_ia"], A["A_ja"], A["A_val"], theta=float(v["dparams"][0]),
                       max_aggregation=CAP[key])
    np.testing.assert_array_equal(agg, v["agg0"])
    assert nc == int(v["info"][1, 0])


def test_oracle_vmb_edge_cases(port):
    # a path graph 0-1-2-3-4 (negative couplings) and an isolated row 5
    n = 6
    rows = [[0, 1], [0, 1, 2], [1, 2, 3], [2, 3, 4], [3, 4], [5]]
    ia = np.cumsum([0] + [len(r) for r in rows]).astype(np.int32)
    ja = np.concatenate(rows).astype(np.int32)
    val = np.array([2.0 if (i == j) else -1.0 for i, r in enumerate(rows) for j in r])
    nc, agg = port.vmb(ia, ja, val)
    # step 1 descending: row 5 is isolated; row 4 opens {4, 3}; rows 3..2 see a
    # taken neighbour; row 1 opens {1, 0, 2}
    assert nc == 2
    assert list(agg) == [1, 1, 1, 0, 0, -1]
    # a cap of 2 leaves row 2 out of {1, 0}; step 2 finds both neighbouring
    # aggregates full, so step 3 opens a third one for it
    nc, agg = port.vmb(ia, ja, val, max_aggregation=2)
    assert nc == 3 and list(agg) == [1, 1, 2, 0, 0, -1]
    # a path 0..5, cap 4: step 1 opens {5, 4} and {2, 1, 3}; row 0 sees a
    # taken neighbour, and step 2 joins it to aggregate 1 (3 members < 4)
    rows = [[0, 1], [0, 1, 2], [1, 2, 3], [2, 3, 4], [3, 4, 5], [4, 5]]
    ia = np.cumsum([0] + [len(r) for r in rows]).astype(np.int32)
    ja = np.concatenate(rows).astype(np.int32)
    val = np.array([2.0 if (i == j) else -1.0 for i, r in enumerate(rows) for j in r])
    nc, agg = port.vmb(ia, ja, val, max_aggregation=4)
    assert nc == 2 and list(agg) == [1, 1, 1, 1, 0, 0]
