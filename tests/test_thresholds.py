"""The engine compares floats with float bounds where the reference widens them
to double (src/mc3d_types.h:11-13); the float bounds decide identically."""
from __future__ import annotations

import numpy as np
import pytest

CASES = [  # (double literal, reference operator, float bound, engine operator)
    (0.1, "lt", float.fromhex("0x1.99999ap-4"), "lt"),      # epsilon < SURVIVAL_CHANCE
    (0.0001, "lt", float.fromhex("0x1.a36e2ep-14"), "le"),  # W < W_THRESHOLD
    (0.99999, "le", float.fromhex("0x1.fffeb0p-1"), "le"),  # fabsf(uz) <= UZ_THRESH
]


def cmp(a, b, op):
    return a < b if op == "lt" else a <= b


@pytest.mark.parametrize("lit,ref_op,bound,op", CASES)
def test_float_bounds_equivalent(lit, ref_op, bound, op):
    b = np.float32(bound)
    around = [b]
    up = down = b
    for _ in range(2000):
        up = np.nextafter(up, np.float32(np.inf))
        down = np.nextafter(down, np.float32(-np.inf))
        around += [up, down]
    rng = np.random.default_rng(0)
    around += list(np.float32(rng.uniform(0, 2 * lit, 20000))) + [np.float32(np.nan)]
    for v in around:
        assert bool(cmp(v, b, op)) == bool(cmp(float(v), lit, ref_op)), (lit, v)
