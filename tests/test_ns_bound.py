"""The bound behind the Newton-Schulz finish's last step (polar.cpp newton_schulz_finish): a
step X <- X (3I - X^T X)/2 maps each d_i = sigma_i^2 - 1 to -3/4 d_i^2 (1 - d_i/3), so with
e = ||d||_2 / sqrt(n) the next e is at most 3/4 e^2 sqrt(n) (1 + e sqrt(n)/3); the finish
skips the confirming Gram when that bound is below a tenth of the rounding floor.  Checked
here in exact arithmetic on the singular values (rational numbers, no rounding)."""
from fractions import Fraction
import math

import numpy as np
import pytest


def ns_map(d):
    # sigma^2 = 1 + d ; sigma' = sigma (3 - sigma^2) / 2 ; d' = sigma'^2 - 1
    s2 = 1 + d
    return s2 * (3 - s2) * (3 - s2) / 4 - 1


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("n", [4, 64, 512])
def test_step_map_and_bound(seed, n):
    rng = np.random.default_rng(seed)
    for scale in (1e-2, 1e-5, 1e-9):
        d = [Fraction(float(x)) for x in rng.uniform(-scale, scale, n)]
        dn = [ns_map(x) for x in d]
        for x, y in zip(d, dn):
            assert y == -Fraction(3, 4) * x * x * (1 - x / 3)  # the map, exactly
        e = math.sqrt(float(sum(x * x for x in d)) / n)
        e_next = math.sqrt(float(sum(y * y for y in dn)) / n)
        rn = math.sqrt(n)
        assert e_next <= 0.75 * e * e * rn * (1.0 + e * rn / 3.0) * (1 + 1e-12)


def test_skip_threshold_is_past_the_floor():
    """At n = 8192 and the floor 1e-14 the skip applies from e of about 3.8e-9 down, where a
    step's bound is at most a tenth of the floor, and not above."""
    n, floor = 8192, 1e-14
    rn = math.sqrt(n)

    def bound(e):
        return 0.75 * e * e * rn * (1.0 + e * rn / 3.0)
    assert bound(3.5e-9) <= 0.1 * floor
    assert bound(4.5e-9) > 0.1 * floor
