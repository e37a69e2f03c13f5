"""The grid engine's division by a fixed divisor (x * RN(1/d) refined once by
the exact FMA remainder, Markstein's correction, for |x| in [2^-90, 2^90] and
zeros; IEEE division elsewhere) against IEEE division, over every one of the
2^32 float bit patterns of x. The engine divides by the product only for a
divisor whose count is 0; the counts here come from the same check it runs at
sheet creation."""
import pytest

import silt_b200 as S

pytestmark = pytest.mark.gpu

# The divisors the coarse (0.2 m) and tire (0.02 m) sheets divide by:
# 2 cell, cell^2, 231, cell.
ENGINE_DIVISORS = [0.4, 0.04, 231.0, 0.2, 0.02, 0.0004]


@pytest.mark.parametrize("d", ENGINE_DIVISORS)
def test_fixed_division_matches_ieee_for_every_float(d):
    counts = S.check_fixed_division(d)
    assert counts[0] == sum(counts[1:]), counts
    assert counts[0] == 0, f"d={d}: mismatches by class {counts}"


def test_check_finds_mismatches_of_an_overflowing_product():
    # With d = 1e-30 the product x * (1 / d) overflows inside the guarded
    # range (2^90 * 1e30 > FLT_MAX), so the check must report mismatches and
    # the engine would keep such a divisor on IEEE division.
    counts = S.check_fixed_division(1e-30)
    assert counts[0] == sum(counts[1:]), counts
    assert counts[0] > 1000, counts
