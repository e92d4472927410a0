"""The reciprocal-based division of the stencil kernels against the IEEE quotient.

The diffusion and divergence-damping stencils divide by a column's sub-triangle areas at every
level; they take 1/area rounded to nearest once per column and form each quotient from it with
fused multiply-adds (Markstein's theorem), which must give the IEEE quotient bit for bit, so the
FP64 form keeps its operation-for-operation parity with the reference. Checked here on the
device over random pairs (wide exponent range and near-exact quotients) in double and float.
"""
import pytest

import thor_b200


@pytest.mark.gpu
def test_reciprocal_division_is_the_ieee_quotient():
    for seed in (1, 20260101):
        bad_d, bad_f = thor_b200.check_division(1 << 27, seed)
        assert (bad_d, bad_f) == (0, 0), (seed, bad_d, bad_f)


@pytest.mark.gpu
def test_reciprocal_division_check_rejects_bad_arguments():
    with pytest.raises(thor_b200.ThorxError):
        thor_b200.check_division(-1)
    assert thor_b200.check_division(0) == (0, 0)
