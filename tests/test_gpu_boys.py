"""The device Boys function against arbitrary precision (B200).

The reference pins its Boys function to mpmath at BOYS_REL_TOL = 1e-14
(tests/unit/test_boys.py:14-38, tests/tolerances.py:14); the same check runs
here on the device evaluation every integral kernel uses (md.cuh ``boys``):
the arguments of that test, every point of the 0.05 Taylor grid and the
points between them up to the switch at t = 36, the range around the switch,
and every order the kernels evaluate (0..9).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
BOYS_REL_TOL = 1e-14
MAX_ORDER = 9


def reference(n: int, t: float) -> float:
    import mpmath

    mpmath.mp.dps = 30
    if t == 0.0:
        return 1.0 / (2 * n + 1)
    half = mpmath.mpf(n) + mpmath.mpf(1) / 2
    return float(mpmath.gammainc(half, 0, t) / (2 * mpmath.mpf(t) ** half))


@pytest.fixture(scope="module")
def context():
    from hafnium_b200 import _lib

    return _lib.Context(0)


def check(context, ts):
    values = context.boys(ts, MAX_ORDER)
    worst = 0.0
    for i, t in enumerate(ts):
        for n in range(MAX_ORDER + 1):
            expected = reference(n, float(t))
            worst = max(worst, abs(values[i, n] - expected) / expected)
    return worst


def test_reference_arguments(context):
    ts = [0.0, 1e-9, 0.05, 0.7, 3.0, 12.5, 34.999, 35.0, 36.0, 60.0, 250.0, 1e4]
    assert check(context, ts) <= BOYS_REL_TOL


def test_grid_points_and_midpoints(context):
    grid = np.arange(0, 721) * 0.05
    ts = np.concatenate([grid[::7], grid[3::11] + 0.025, grid[5::13] + 0.0124])
    assert check(context, ts[ts >= 0.0]) <= BOYS_REL_TOL


def test_around_the_switch_to_the_large_argument_form(context):
    ts = np.concatenate([np.linspace(35.0, 37.0, 41), [36.0 - 1e-12, 36.0 + 1e-12]])
    assert check(context, ts) <= BOYS_REL_TOL


def test_rejects_negative_arguments_and_orders_beyond_the_kernels(context):
    from hafnium_b200.errors import InputError

    with pytest.raises(InputError, match="non-negative"):
        context.boys([-0.5], 2)
    with pytest.raises(InputError, match="non-negative"):
        context.boys([float("nan")], 2)
    with pytest.raises(InputError, match="orders 0..9"):
        context.boys([1.0], 10)
