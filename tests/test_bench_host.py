"""bench.py's reference arm and argument checks on CPU: the JSON line of the
contract (metric, value, unit, impl, cpu_baseline, e2e) for a --variant of
the drop-in and for the bsr workload, and the variants' workload rule."""
import json
import os
import subprocess
import sys

import pytest

import oracle
from conftest import ROOT

KEYS = {"metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
        "cpu_baseline", "e2e"}


def _bench(*args, timeout=600):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                          capture_output=True, text=True, timeout=timeout)


def _line(r):
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("variant", ["gmres", "w"])
def test_reference_arm_variant_line(variant):
    d = _line(_bench("--impl", "reference", "--workload", "c1", "--variant", variant,
                     "--steps", "1", "--warmup", "3"))
    assert KEYS <= set(d)
    assert d["impl"] == "reference" and d["config"]["variant"] == variant
    assert d["value"] > 0 and d["iterations"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] == 1


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_reference_arm_bsr_line():
    d = _line(_bench("--impl", "reference", "--workload", "bsr", "--steps", "1",
                     "--warmup", "3"))
    assert KEYS <= set(d)
    assert d["iterations"] == 9 and d["config"]["dofs"] == 750141


def test_variant_needs_c1_or_c2():
    r = _bench("--impl", "reference", "--workload", "c5", "--variant", "gmres", timeout=120)
    assert r.returncode == 2 and "c1 and c2" in r.stderr


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_reference_arm_c1_line():
    """c1: the full workload every timed step; setup and solve seconds of the
    reference reported beside the total."""
    d = _line(_bench("--impl", "reference", "--workload", "c1", "--steps", "2",
                     "--warmup", "3"))
    assert KEYS <= set(d)
    assert d["steps"] == 2 and d["steps_requested"] == 2
    assert d["iterations"] == 25   # l1-Jacobi V(2,2) on the 255^2 Poisson problem
    assert d["setup_s"] > 0 and d["solve_s"] > 0


def test_solve_bytes_model():
    """The solve-level byte model of the mixed solve on a two-level
    hierarchy, term by term."""
    sys.path.insert(0, ROOT)
    import bench
    n0, nnz0, nz32, n1 = 1000, 7000, 5000, 400
    levels = [{"rows": n0, "nnz": nnz0, "nnz32": nz32}, {"rows": n1}]
    sweep = 8 * nz32 + 4 * (n0 + 1) + 12 * n0
    cyc = 12 * n0 + 3 * sweep + sweep + (4 * (n1 + 1) + 8 * n0 + 4 * n1) \
        + (12 * n0 + 4 * n1) + 8 * n1 * n1 + 8 * n1
    outer = 12 * nnz0 + 4 * (n0 + 1) + 16 * n0 + 112 * n0
    res0 = 12 * nnz0 + 4 * (n0 + 1) + 24 * n0
    assert bench.solve_bytes_mixed(levels, 10, False) == 10 * outer + 11 * cyc + 2 * res0
    # the learned weights add 4 bytes per fine row to the first and three full sweeps
    assert bench.solve_bytes_mixed(levels, 10, True) - bench.solve_bytes_mixed(
        levels, 10, False) == 11 * 4 * (4 * n0)


def test_clock_samples_after_mark():
    """The clock summary keeps the nvidia-smi samples taken after the start of
    the timed region (the sampler starts before the warm-up steps), falls back
    to all samples when none is later, and reports the throttle reasons seen."""
    import datetime
    sys.path.insert(0, ROOT)
    import bench
    rows = ["2026/12/04 01:00:00.000, 1500, 1965, 300.1, Not Active, Not Active, Not Active, "
            "Not Active\n",
            "2026/12/04 01:00:01.000, 1965, 1965, 900.0, Not Active, Not Active, Not Active, "
            "Active\n",
            "2026/12/04 01:00:01.200, 1905, 1965, 950.0, Not Active, Not Active, Not Active, "
            "Not Active\n",
            "garbled\n"]
    mark = datetime.datetime(2026, 12, 4, 1, 0, 0, 500000)
    s = bench.Clocks.summary(rows, mark)
    assert s["samples"] == 2 and s["sm_mhz"] == 1935.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    late = bench.Clocks.summary(rows, datetime.datetime(2027, 1, 1))
    assert late["samples"] == 3 and late["sm_mhz"] == 1905.0
    assert bench.Clocks.summary([], mark)["sm_mhz"] is None
