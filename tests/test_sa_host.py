"""The oracle's C restatement of smoothed aggregation (or_sa_setup: the UA
aggregates with the adaptive threshold, the filtered damped-Jacobi smoother,
dcsr_mxm, dcsr_trans, the general dcsr_rap, the coarsest transposed for the
direct solver) against the reference's hierarchies in tests/golden/sa.npz:
every coarse operator and every smoothed prolongation bit for bit (SHA-256),
and the adapted threshold."""
import hashlib

import numpy as np
import pytest

from conftest import small_case

VARIANTS = ["fix/sa", "fix/sa_nf", "kuhn/sa", "kuhn/sa_nf", "kuhn/sa_t", "kuhn/sa_w"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# the 128^2 variants' dense coarse levels take the oracle (like the reference)
# tens of seconds: their first three levels are compared, the Kuhn variants whole
LEVELS = {"fix/sa": 3, "fix/sa_nf": 3}


@pytest.mark.parametrize("key", VARIANTS)
def test_oracle_sa_hierarchy_matches_reference(golden, port, key):
    A = small_case(golden("gmres.npz"), key.split("/")[0])
    v = small_case(golden("sa.npz"), key)
    ip = [int(t) for t in v["params"]]
    dp = [float(t) for t in v["dparams"]]
    info = v["info"]
    nl = LEVELS.get(key, len(info))
    whole = nl == len(info)
    As, Ps, theta = port.sa_hierarchy(A["A_ia"], A["A_ja"], A["A_val"], theta=dp[0],
                                      coarse_dof=ip[1], max_levels=nl if not whole else ip[0],
                                      aggregation_type=ip[7], max_aggregation=ip[8],
                                      smooth_filter=ip[15], tentative_smooth=dp[3],
                                      coarse_solver=ip[6] if whole else 0)
    assert len(As) == nl
    for l, a in enumerate(As):
        assert [sha(x) for x in a] == list(v[f"A{l}_sha"]), f"A{l}"
    for l, p in enumerate(Ps):
        assert len(p[1]) == int(info[l, 3])
        assert [sha(x) for x in p] == list(v[f"P{l}_sha"]), f"P{l}"
    if whole:
        assert theta == float(v["theta_after"])
