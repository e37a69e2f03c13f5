"""The grid engine's division by a fixed divisor (x * RN(1/d) refined once by
the exact FMA remainder, Markstein's correction, for |x| in [2^-90, 2^90] and
zeros; IEEE division elsewhere) against IEEE division, over every one of the
2^32 float bit patterns of x. The engine divides by the product only for a
divisor whose count is 0; the counts here come from the same check it runs at
sheet creation."""
import pytest

import silt_b200 as S

pytestmark = pytest.mark.gpu

# The divisors the coarse (0.2 m) and tire (0.02 m) sheets divide by,
# 2 cell, cell^2, 231 and cell as the float products the step forms
# (0.2f * 0.2f is 0.040000003, not the float nearest 0.04): the library
# takes these as checked without running the check, so each is checked here.
ENGINE_DIVISORS = [0.4, 0.2 * 0.2, 231.0, 0.2, 0.04, 0.0004, 0.02]


def test_known_divisors_are_the_engine_divisors():
    import numpy as np

    f = np.float32
    want = sorted({float(f(2) * f(c)) for c in (0.2, 0.02)} | {float(f(c) * f(c)) for c in (0.2, 0.02)}
                  | {231.0, float(f(0.2)), float(f(0.02))})
    assert sorted(S.known_exact_divisors()) == want


@pytest.mark.parametrize("k", range(7))
def test_fixed_division_matches_ieee_for_every_float(k):
    d = S.known_exact_divisors()[k]
    counts = S.check_fixed_division(d)
    assert counts[0] == sum(counts[1:]), counts
    assert counts[0] == 0, f"d={d!r}: mismatches by class {counts}"


def test_check_finds_mismatches_of_an_overflowing_product():
    # With d = 1e-30 the product x * (1 / d) overflows inside the guarded
    # range (2^90 * 1e30 > FLT_MAX), so the check must report mismatches and
    # the engine would keep such a divisor on IEEE division.
    counts = S.check_fixed_division(1e-30)
    assert counts[0] == sum(counts[1:]), counts
    assert counts[0] > 1000, counts
