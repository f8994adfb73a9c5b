"""Kernel-level parity of the CUDA library against the reference's outputs
(golden fixtures) and the CPU oracle, through the C ABI on device arrays.
Integer outputs and every FP64 kernel are compared bit for bit."""
import ctypes as C

import numpy as np
import pytest

import hazmath_b200 as hz
from hazmath_b200 import problems as P
from gpu_util import DevCSR, dev, host, ptr

pytestmark = pytest.mark.gpu


def test_mxv_aAxpy_bit_exact(golden):
    g = golden("smoothers.npz")
    A = DevCSR(g["ia"], g["ja"], g["val"])
    x = dev(g["x0"])
    y = dev(np.zeros(A.n))
    assert hz.lib().hzb_dcsr_mxv_device(*A.args(), ptr(x), ptr(y)) == 0
    assert np.array_equal(host(y), g["mxv"])
    for alpha, key in ((-1.0, "aAxpy_m1"), (0.7, "aAxpy_07")):
        y = dev(g["b"])
        assert hz.lib().hzb_dcsr_aAxpy_device(alpha, *A.args(), ptr(x), ptr(y)) == 0
        assert np.array_equal(host(y), g[key])


@pytest.mark.parametrize("N", [9, 40])
def test_mxv_kuhn_vs_oracle(port, N):
    """15-point Kuhn pattern with explicit zeros; N = 40 exercises bundles
    of 128 rows x 15 entries staged in shared memory."""
    ia, ja, val = P.kuhn3d_p1(N, P.lognormal_field(N, 1.0, 4.0, 7))
    x = np.random.default_rng(1).uniform(-1, 1, len(ia) - 1)
    A = DevCSR(ia, ja, val)
    y = dev(np.zeros(A.n))
    assert hz.lib().hzb_dcsr_mxv_device(*A.args(), ptr(dev(x)), ptr(y)) == 0
    assert np.array_equal(host(y), port.mxv(ia, ja, val, x))


@pytest.mark.parametrize("sm", [1, 2, 3, 5, 6, 7, 8, 10])
@pytest.mark.parametrize("pre", [1, 0])
def test_smoothers_bit_exact(golden, sm, pre):
    """GS/SGS/SOR through the level-scheduled exact sweep; Jacobi and
    l1-Jacobi row-parallel: all equal to the reference's sequential loops."""
    g = golden("smoothers.npz")
    A = DevCSR(g["ia"], g["ja"], g["val"])
    x = dev(g["x0"])
    rc = hz.lib().hzb_smoother_device(sm, pre, 2, 1.2, *A.args(), ptr(dev(g["b"])), ptr(x))
    assert rc == 0, hz.last_error()
    assert np.array_equal(host(x), g[f"s{sm}_pre{pre}"])


@pytest.mark.parametrize("sm", [6, 7, 8])
@pytest.mark.parametrize("pre", [1, 0])
def test_combined_smoothers_vs_oracle(port, sm, pre):
    ia, ja, val = P.aniso2d_p1(23, 0.03, 0.4)
    rng = np.random.default_rng(sm * 10 + pre)
    b, x0 = rng.uniform(-1, 1, len(ia) - 1), rng.uniform(-1, 1, len(ia) - 1)
    A = DevCSR(ia, ja, val)
    x = dev(x0)
    assert hz.lib().hzb_smoother_device(sm, pre, 1, 1.15, *A.args(), ptr(dev(b)), ptr(x)) == 0
    assert np.array_equal(host(x), port.smooth(sm, pre, 1, ia, ja, val, b, x0, relax=1.15))


def _hem(ia, ja, val, theta):
    A = DevCSR(ia, ja, val)
    agg = dev(np.zeros(A.n, np.int32))
    nc = C.c_int()
    rc = hz.lib().hzb_aggregation_hem_device(*A.args(), theta, ptr(agg), C.byref(nc))
    assert rc == 0, hz.last_error()
    return nc.value, host(agg)


@pytest.mark.parametrize("case", ["aniso2d_31", "kuhn_12", "theta_p2d_40"])
def test_hem_matches_reference_level0(golden, case):
    z = golden("small_cases.npz")
    theta = float(z[f"{case}/dparams"][0])
    nc, agg = _hem(z[f"{case}/A_ia"], z[f"{case}/A_ja"], z[f"{case}/A_val"], theta)
    assert np.array_equal(agg, z[f"{case}/agg0"])
    assert nc == int(z[f"{case}/info"][0][2])


@pytest.mark.parametrize("seed", range(4))
def test_hem_random_vs_oracle(port, seed):
    rng = np.random.default_rng(seed)
    m = int(rng.integers(15, 60))
    ia, ja, val = P.aniso2d_p1(m, float(10 ** rng.uniform(-4, 0)), float(rng.uniform(0, np.pi)))
    theta = float(rng.choice([0.0, 0.1, 0.3]))
    nc, agg = _hem(ia, ja, val, theta)
    nc_o, agg_o = port.hem(ia, ja, val, theta)
    assert nc == nc_o and np.array_equal(agg, agg_o)


@pytest.mark.parametrize("path", [1, 2, 3, 4])
def test_hem_implementations_agree(golden, port, monkeypatch, path):
    # ranked lists + byte ring, ranked lists + bit ring, bit ring over the raw
    # rows, state in global memory: the same aggregates as the reference
    monkeypatch.setenv("HZB_HEM_PATH", str(path))
    z = golden("small_cases.npz")
    for case in ["aniso2d_31", "kuhn_12", "theta_p2d_40"]:
        theta = float(z[f"{case}/dparams"][0])
        nc, agg = _hem(z[f"{case}/A_ia"], z[f"{case}/A_ja"], z[f"{case}/A_val"], theta)
        assert np.array_equal(agg, z[f"{case}/agg0"]), case
        assert nc == int(z[f"{case}/info"][0][2])
    k = P.lognormal_field(14, 1.0, 3.0, 7)
    ia, ja, val = P.kuhn3d_p1(14, k)
    rows = np.repeat(np.arange(len(ia) - 1), np.diff(ia))
    val = val * (1.0 + 0.01 * ((rows + ja + path) % 3))   # symmetric ties and near-ties
    nc, agg = _hem(ia, ja, val, 0.05)
    nc_o, agg_o = port.hem(ia, ja, val, 0.05)
    assert nc == nc_o and np.array_equal(agg, agg_o)


def test_rap_bit_exact(golden):
    g = golden("rap.npz")
    A = DevCSR(g["ia"], g["ja"], g["val"])
    nc = int(g["nc"])
    nnz = C.c_int()
    pia, pja, pval = C.c_void_p(), C.c_void_p(), C.c_void_p()
    rc = hz.lib().hzb_rap_agg_device(*A.args(), nc, ptr(dev(g["agg"])), C.byref(nnz),
                                     C.byref(pia), C.byref(pja), C.byref(pval))
    assert rc == 0, hz.last_error()
    out = []
    for p, n, dt in ((pia, nc + 1, np.int32), (pja, nnz.value, np.int32),
                     (pval, nnz.value, np.float64)):
        h = np.empty(n, dt)
        assert hz.lib().hzb_copy_to_host(C.c_void_p(h.ctypes.data), p,
                                         C.c_size_t(h.nbytes)) == 0
        hz.lib().hzb_free_device(p)
        out.append(h)
    assert np.array_equal(out[0], g["cia"])
    assert np.array_equal(out[1], g["cja"])
    assert np.array_equal(out[2], g["cval"])

