import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return np.load(os.path.join(GOLDEN, name), allow_pickle=False)
    return load


@pytest.fixture(scope="session")
def port():
    import oracle
    if not os.path.exists(oracle.PORT_SO):
        oracle.build(ref=False)
    return oracle.port()


def small_case_names(z):
    return sorted({k.split("/")[0] for k in z.files})


def small_case(z, name):
    pre = name + "/"
    return {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}


def params_of(case):
    import oracle
    ip = [int(v) for v in case["params"]]
    dp = [float(v) for v in case["dparams"]]
    names = ["max_levels", "coarse_dof", "cycle_type", "smoother", "presmooth_iter",
             "postsmooth_iter", "coarse_solver", "aggregation_type", "max_aggregation",
             "coarse_scaling", "print_level", "maxit"]
    kw = dict(zip(names, ip))
    kw.update(strong_coupled=dp[0], relaxation=dp[1], tol=dp[2])
    return oracle.AMGParams(**kw)
