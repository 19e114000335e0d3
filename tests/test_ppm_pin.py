"""The oracle's PPM edges (no reference counterpart) pinned to Colella & Woodward (1984) by cases
worked by hand from the paper's equations: eq. 1.6 with the limited slopes of eq. 1.8 gives the
interface values, eq. 1.10 flattens an extremum and pulls an overshooting edge in. The GPU's PPM
is held to this oracle by the parity tests."""
import math

import pytest

from oracle.oracle import ppm_edges


def _cubic_averages(c, centres):
    # cell averages over [x - 1/2, x + 1/2] of p(x) = c0 + c1 x + c2 x^2 + c3 x^3
    def prim(x):
        return c[0] * x + c[1] * x ** 2 / 2 + c[2] * x ** 3 / 3 + c[3] * x ** 4 / 4
    return [prim(x + 0.5) - prim(x - 0.5) for x in centres]


def test_smooth_monotone_cubic_gives_exact_interfaces():
    # unlimited there (monotone, slopes within a factor of the neighbours'), eq. 1.6 is the
    # fourth-order interface value 7/12 (a_j + a_j+1) - 1/12 (a_j-1 + a_j+2): exact for a cubic
    c = (1.0, 0.3, 0.05, 0.01)
    lo, hi = ppm_edges(*_cubic_averages(c, [-2, -1, 0, 1, 2]))

    def p(x):
        return c[0] + c[1] * x + c[2] * x ** 2 + c[3] * x ** 3
    assert hi == pytest.approx(p(0.5), rel=1e-12)
    assert lo == pytest.approx(p(-0.5), rel=1e-12)


def test_extremum_is_flattened():
    # (a_R - a)(a - a_L) <= 0: both edges take the cell's value (eq. 1.10, first case)
    assert ppm_edges(0.0, 1.0, 2.0, 1.0, 0.0) == (2.0, 2.0)
    # a one-sided step with a flat side: the same test holds with a zero product
    assert ppm_edges(0.0, 0.0, 0.0, 1.0, 1.0) == (0.0, 0.0)


def test_overshooting_edge_is_pulled_in():
    # slopes (eq. 1.8): at a_j-1 = 0.1 the mean 0.1; at a_j = 0.2 min(0.45, 2 x 0.1) = 0.2; at
    # a_j+1 = 1 zero (a_j+2 - a_j+1 = 0). Eq. 1.6: a_L = 0.15 - 0.1/6, a_R = 0.6 + 0.2/6.
    # da = a_R - a_L = 0.5, a6 = 6 (a - (a_L + a_R)/2) = -1.1: -da^2 > da a6, so the upper
    # edge is pulled in to 3 a - 2 a_L (eq. 1.10).
    lo, hi = ppm_edges(0.0, 0.1, 0.2, 1.0, 1.0)
    al = 0.15 - 0.1 / 6
    assert lo == pytest.approx(al, rel=1e-13)
    assert hi == pytest.approx(3 * 0.2 - 2 * al, rel=1e-13)
    # the mirror image pulls the lower edge in
    lo2, hi2 = ppm_edges(1.0, 1.0, 0.2, 0.1, 0.0)
    assert hi2 == pytest.approx(al, rel=1e-13) and lo2 == pytest.approx(3 * 0.2 - 2 * al, rel=1e-13)


def test_steep_slope_is_limited_to_twice_the_smaller_difference():
    # a_j-1 = 0, a_j = 1, a_j+1 = 10: the centred slope 5 exceeds 2 min(1, 9) = 2 (eq. 1.8)
    lo, hi = ppm_edges(0.0, 0.0, 1.0, 10.0, 19.0)
    dm, d0, dp = 0.0, 2.0, 9.0  # slopes at a_j-1 (one side flat), a_j, a_j+1 (min(9, 2 x 9))
    al = 0.5 * (0.0 + 1.0) - (d0 - dm) / 6
    ar = 0.5 * (1.0 + 10.0) - (dp - d0) / 6
    da, a6 = ar - al, 6 * (1.0 - 0.5 * (al + ar))
    if da * a6 > da * da:
        al = 3 * 1.0 - 2 * ar
    elif -da * da > da * a6:
        ar = 3 * 1.0 - 2 * al
    assert (lo, hi) == pytest.approx((al, ar), rel=1e-13)
    assert math.isfinite(lo) and lo <= 1.0 <= hi
