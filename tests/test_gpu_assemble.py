"""Device assembly of the Kuhn-mesh P1 stiffness (hzb_assemble_p1_kuhn_device)
against the host generator the parity fixtures and the benchmark use
(hazmath_b200.problems.kuhn3d_p1): the same row pointers, columns and values
bit for bit, for per-cube coefficients, constant anisotropic tensors and
boundary-dominated small meshes; against the reference's own assembly on
its own cube mesh (tests/golden/cube_p1.npz) to rounding; and the assembled
matrix solves like the host one."""
import numpy as np
import pytest

import hazmath_b200 as hz
from hazmath_b200 import problems as P
from gpu_util import dev, host, ptr, torch_cuda

pytestmark = pytest.mark.gpu


def assemble(N, kcell=None, K=None):
    torch = torch_cuda()
    m = N - 1
    ia = torch.empty(m ** 3 + 1, dtype=torch.int32, device="cuda")
    kd = dev(np.ascontiguousarray(kcell, np.float64)) if kcell is not None else None
    kp = ptr(kd) if kd is not None else None
    rc, nnz = hz.assemble_p1_kuhn_device(N, kp, ptr(ia), K=K)
    assert rc == 0, hz.last_error()
    ja = torch.empty(nnz, dtype=torch.int32, device="cuda")
    val = torch.empty(nnz, dtype=torch.float64, device="cuda")
    rc, nnz2 = hz.assemble_p1_kuhn_device(N, kp, ptr(ia), ptr(ja), ptr(val), K=K)
    assert rc == 0 and nnz2 == nnz
    torch.cuda.synchronize()
    return host(ia), host(ja), host(val)


def same(got, want):
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])
    assert got[2].tobytes() == np.ascontiguousarray(want[2], np.float64).tobytes()


@pytest.mark.parametrize("N", [2, 3, 4, 9, 33])
def test_lognormal_cells_bit_exact(N):
    k = P.lognormal_field(N, 1.5, 2.0, 40 + N) if N > 2 else np.array([[[2.0, 3.0], [5.0, 7.0]],
                                                                        [[11.0, 13.0], [17.0, 19.0]]])
    want = P.kuhn3d_p1(N, k)
    got = assemble(N, k)
    same(got, want)


def test_unit_coefficient_bit_exact():
    want = P.kuhn3d_p1(24)
    same(assemble(24), want)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_anisotropic_tensor_bit_exact(seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(3)
    a /= np.linalg.norm(a)
    th, eps = rng.uniform(0, np.pi), 10 ** rng.uniform(-3, 0)
    c, s = np.cos(th), np.sin(th)
    A = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    R = np.eye(3) * c + s * A + (1 - c) * np.outer(a, a)
    K = R @ np.diag([1.0, 1.0, eps]) @ R.T
    k = P.lognormal_field(12, 1.0, 2.0, seed)
    same(assemble(12, k, K), P.kuhn3d_p1(12, k, K))


def test_diagonal_tensor_bit_exact():
    """A diagonal K takes the kernel that leaves out the entries every
    diagonal tensor zeroes."""
    K = np.diag([1.0, 0.3, 2.5])
    k = P.lognormal_field(10, 1.0, 2.0, 5)
    same(assemble(10, k, K), P.kuhn3d_p1(10, k, K))


def test_full_size_bit_exact():
    """128^3 cubes, the 2,048,383-row, 30,340,171-entry configuration."""
    N = 128
    k = P.lognormal_field(N, 1.0, 8.0, 2)
    got = assemble(N, k)
    assert len(got[0]) == 127 ** 3 + 1 and len(got[1]) == 30340171
    same(got, P.kuhn3d_p1(N, k))


def test_assembled_matrix_solves_like_host_one():
    N = 40
    k = P.lognormal_field(N, 1.0, 4.0, 9)
    ia, ja, val = assemble(N, k)
    b = P.rhs_uniform(len(ia) - 1, 3)
    it = hz.itsolver_param(linear_itsolver_type=hz.SOLVER_CG, linear_precond_type=hz.PREC_AMG,
                           linear_tol=1e-8, linear_maxit=200)
    out = []
    for arrs in ((ia, ja, val), P.kuhn3d_p1(N, k)):
        S = hz.Solver(hz.bench_amg(), it)
        assert S.setup_host(*arrs) == 0
        x = np.zeros(len(b))
        out.append((S.solve_host(b, x), x))
        S.close()
    assert out[0][0] == out[1][0] > 0
    assert out[0][1].tobytes() == out[1][1].tobytes()


def test_rejects_bad_sizes():
    torch = torch_cuda()
    ia = torch.empty(8, dtype=torch.int32, device="cuda")
    assert hz.assemble_p1_kuhn_device(1, None, ptr(ia))[0] == hz.ERROR_MAT_SIZE
    assert hz.assemble_p1_kuhn_device(600, None, ptr(ia))[0] == hz.ERROR_MAT_SIZE


@pytest.mark.parametrize("ndiv", [4, 8, 12])
def test_matches_reference_assembly(golden, ndiv):
    """Against the reference's own assembly on its own cube mesh (unit
    coefficient): same pattern, values to rounding."""
    from conftest import small_case
    ref = small_case(golden("cube_p1.npz"), f"n{ndiv}")
    ia, ja, val = assemble(ndiv)
    np.testing.assert_array_equal(ia, ref["ia"])
    np.testing.assert_array_equal(ja, ref["ja"])
    np.testing.assert_allclose(val, ref["val"], rtol=0, atol=1e-14 * np.abs(ref["val"]).max())


def test_unaligned_outputs_take_the_scalar_copy():
    """ja / val that are not 16-byte aligned (views one element in) get the
    same arrays through the element-wise copy-out."""
    torch = torch_cuda()
    N = 20
    k = P.lognormal_field(N, 1.0, 3.0, 17)
    want = P.kuhn3d_p1(N, k)
    m, nnz = N - 1, int(want[0][-1])
    kd = dev(k)
    ia = torch.empty(m ** 3 + 1, dtype=torch.int32, device="cuda")
    ja = torch.zeros(nnz + 1, dtype=torch.int32, device="cuda")
    va = torch.zeros(nnz + 1, dtype=torch.float64, device="cuda")
    rc, got = hz.assemble_p1_kuhn_device(N, ptr(kd), ptr(ia), ptr(ja[1:]), ptr(va[1:]))
    assert rc == 0 and got == nnz
    torch.cuda.synchronize()
    same((host(ia), host(ja[1:]), host(va[1:])), want)
    assert int(host(ja)[0]) == 0 and host(va)[0] == 0.0
