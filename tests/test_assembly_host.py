"""The Kuhn-mesh P1 generator (hazmath_b200.problems.kuhn3d_p1), which the
device assembly reproduces bit for bit, against the reference's own
assembly on its own cube mesh (tests/golden/cube_p1.npz: mesh_cube_init with
uniform refinement + the elliptic_p1 example's call_assembly, unit
coefficient, interior vertices renumbered lexicographically): the same
15-point pattern, and values equal to the reference's to rounding (the
reference computes each simplex's gradients by a small matrix inversion)."""
import numpy as np
import pytest

from conftest import small_case
from hazmath_b200 import problems as P

VTOL = 1e-14   # relative to max |a_ij| (h = 1/12 is not a power of two)


@pytest.mark.parametrize("ndiv", [4, 8, 12])
def test_generator_matches_reference_assembly(golden, ndiv):
    ref = small_case(golden("cube_p1.npz"), f"n{ndiv}")
    ia, ja, val = P.kuhn3d_p1(ndiv)
    np.testing.assert_array_equal(ia, ref["ia"])
    np.testing.assert_array_equal(ja, ref["ja"])
    np.testing.assert_allclose(val, ref["val"], rtol=0, atol=VTOL * np.abs(ref["val"]).max())


def test_generator_stores_the_exact_zero_couplings(golden):
    """The reference's symbolic assembly keeps every vertex pair of a simplex;
    the 8 couplings that vanish for the unit coefficient stay stored as
    exact zeros on both sides."""
    ref = small_case(golden("cube_p1.npz"), "n8")
    ia, ja, val = P.kuhn3d_p1(8)
    assert (val == 0.0).sum() > 0
    assert np.all(np.abs(ref["val"][val == 0.0]) < 1e-15)
