"""The allocation-free Galerkin product, hzb_rap_agg_device_noalloc.

It exists for callers that cannot call cudaMalloc -- a process whose device
memory is reserved up front by its own allocator, or library code that must
not take the implicit device synchronisation of cudaMalloc/cudaFree: its
scratch is a fixed device array inside the library.  These tests call it
through the C ABI and compare its output with hzb_rap_agg_device's -- which
allocates -- on two calls in a row, bit for bit (same kernels, same order),
and check that bad inputs (an aggregate id out of range, row pointers that
end above the stated entry count) are turned into an error by the device
check before any kernel indexes by them.  The file is named so that pytest
collects it last."""
import ctypes as C

import numpy as np
import pytest

import hazmath_b200 as hz
from hazmath_b200 import problems as P
from gpu_util import DevCSR, dev, host, ptr

pytestmark = pytest.mark.gpu


def rap_alloc(A, nc, agg_d):
    nnz = C.c_int()
    pia, pja, pval = C.c_void_p(), C.c_void_p(), C.c_void_p()
    rc = hz.lib().hzb_rap_agg_device(*A.args(), nc, ptr(agg_d), C.byref(nnz), C.byref(pia),
                                     C.byref(pja), C.byref(pval))
    assert rc == 0, hz.last_error()
    out = []
    for p, m, dt in ((pia, nc + 1, np.int32), (pja, nnz.value, np.int32),
                     (pval, nnz.value, np.float64)):
        h = np.empty(m, dt)
        assert hz.lib().hzb_copy_to_host(h.ctypes.data, p, h.nbytes) == 0
        hz.lib().hzb_free_device(p)
        out.append(h)
    return out


def rap_noalloc(A, nc, agg_d, cap):
    import torch
    cia = torch.zeros(nc + 1, dtype=torch.int32, device="cuda")
    cja = torch.zeros(max(cap, 1), dtype=torch.int32, device="cuda")
    cval = torch.zeros(max(cap, 1), dtype=torch.float64, device="cuda")
    nnz = C.c_int()
    rc = hz.lib().hzb_rap_agg_device_noalloc(*A.args(), nc, ptr(agg_d), cap, ptr(cia),
                                             ptr(cja), ptr(cval), C.byref(nnz))
    return rc, nnz.value, host(cia), host(cja)[:nnz.value], host(cval)[:nnz.value]


def cases():
    g = np.load(__import__("os").path.join(__import__("conftest").GOLDEN, "rap.npz"))
    yield g["ia"], g["ja"], g["val"], int(g["nc"]), g["agg"]
    import oracle
    port = oracle.port()
    ia, ja, val = P.aniso2d_p1(150, 0.01, 0.6)
    nc, agg = port.hem(ia, ja, val, 0.0)
    yield ia, ja, val, nc, agg


@pytest.mark.parametrize("k", [0, 1])
def test_noalloc_matches_allocating_entry_point(k):
    ia, ja, val, nc, agg = list(cases())[k]
    A = DevCSR(ia, ja, val)
    agg_d = dev(np.int32(agg))
    ref_ia, ref_ja, ref_val = rap_alloc(A, nc, agg_d)
    for _call in range(2):   # the scratch keeps the previous call's contents
        rc, nnz, cia, cja, cval = rap_noalloc(A, nc, agg_d, len(ref_ja))
        assert rc == 0, hz.last_error()
        assert nnz == len(ref_ja)
        assert np.array_equal(cia, ref_ia)
        assert np.array_equal(cja, ref_ja)
        assert np.array_equal(cval, ref_val)


def test_noalloc_limits_and_capacity():
    ia, ja, val, nc, agg = list(cases())[0]
    A = DevCSR(ia, ja, val)
    agg_d = dev(np.int32(agg))
    # capacity too small: error, and the needed size is reported
    rc, nnz, _, _, _ = rap_noalloc(A, nc, agg_d, 3)
    assert rc == hz.ERROR_INPUT_PAR and nnz > 3
    # sizes beyond the static scratch are rejected before any device work
    big = hz.lib().hzb_rap_agg_device_noalloc(65537, 10, ptr(A.ia), ptr(A.ja), ptr(A.val), 5,
                                              ptr(agg_d), 10, ptr(A.ia), ptr(A.ja),
                                              ptr(A.val), C.byref(C.c_int()))
    assert big == hz.ERROR_MAT_SIZE
    big = hz.lib().hzb_rap_agg_device_noalloc(100, 1048577, ptr(A.ia), ptr(A.ja), ptr(A.val),
                                              5, ptr(agg_d), 10, ptr(A.ia), ptr(A.ja),
                                              ptr(A.val), C.byref(C.c_int()))
    assert big == hz.ERROR_MAT_SIZE


def test_bad_inputs_rejected_before_indexing():
    """An aggregate id >= nc, and an nnz that understates ia[n], return
    ERROR_INPUT_PAR from both entry points (the device check reads agg, ia
    and ja within the caller's stated sizes only), and a valid call after
    them still gives the exact product."""
    ia, ja, val, nc, agg = list(cases())[0]
    A = DevCSR(ia, ja, val)
    ref_ia, ref_ja, ref_val = rap_alloc(A, nc, dev(np.int32(agg)))
    bad = np.int32(agg).copy()
    bad[len(bad) // 2] = nc + 7
    bad_d = dev(bad)
    rc, _, _, _, _ = rap_noalloc(A, nc, bad_d, len(ref_ja))
    assert rc == hz.ERROR_INPUT_PAR
    assert "aggregate" in hz.last_error()
    nnz = C.c_int()
    pia, pja, pval = C.c_void_p(), C.c_void_p(), C.c_void_p()
    rc = hz.lib().hzb_rap_agg_device(*A.args(), nc, ptr(bad_d), C.byref(nnz), C.byref(pia),
                                     C.byref(pja), C.byref(pval))
    assert rc == hz.ERROR_INPUT_PAR
    # understated entry count: ia[n] no longer equals nnz
    import torch
    n, full = A.n, A.nnz
    cap = len(ref_ja)
    oia = torch.full((nc + 1,), -5, dtype=torch.int32, device="cuda")
    oja = torch.full((cap,), -5, dtype=torch.int32, device="cuda")
    oval = torch.zeros(cap, dtype=torch.float64, device="cuda")
    for under in (full - 1, full // 2):
        out = C.c_int()
        rc = hz.lib().hzb_rap_agg_device_noalloc(n, under, ptr(A.ia), ptr(A.ja), ptr(A.val),
                                                 nc, ptr(dev(np.int32(agg))), cap, ptr(oia),
                                                 ptr(oja), ptr(oval), C.byref(out))
        assert rc == hz.ERROR_INPUT_PAR
        assert "row pointers" in hz.last_error()
    assert bool((oia == -5).all()) and bool((oja == -5).all())    # nothing written
    rc, nnz2, cia, cja, cval = rap_noalloc(A, nc, dev(np.int32(agg)), len(ref_ja))
    assert rc == 0 and nnz2 == len(ref_ja)
    assert np.array_equal(cia, ref_ia) and np.array_equal(cja, ref_ja)
    assert np.array_equal(cval, ref_val)
