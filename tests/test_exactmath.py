"""Accuracy of the reproducible series functions (mc3d_exactmath.h) against
double-precision libm, on the domains the photon loop uses them."""
from __future__ import annotations

import math

import numpy as np


def ulp_err(got: float, exact: float) -> float:
    f = np.float32(exact)
    ulp = float(np.spacing(np.abs(f))) if f != 0 else float(np.spacing(np.float32(1e-30)))
    return abs(got - exact) / ulp


def sample(lo, hi, n, seed=0):
    rng = np.random.default_rng(seed)
    return np.float32(rng.uniform(lo, hi, n))


def test_logf(orc):
    L = orc.lib()
    xs = np.concatenate([sample(2 ** -24, 1.0, 20000), np.float32(2.0) ** -np.arange(25),
                         np.float32(1) - np.float32(2.0) ** -np.arange(1, 25)])
    worst = max(ulp_err(L.orc_logf(float(x)), math.log(float(x))) for x in xs if x > 0)
    assert worst <= 3.0, worst
    assert L.orc_logf(1.0) == 0.0


def test_sincospif(orc):
    L = orc.lib()
    s, c = C_float(), C_float()
    worst = 0.0
    for x in np.concatenate([sample(0, 2, 20000), np.float32([0, 0.25, 0.5, 1, 1.5, 1.75])]):
        L.orc_sincospif(float(x), s.ref, c.ref)
        ex_s, ex_c = math.sin(math.pi * float(x)), math.cos(math.pi * float(x))
        # absolute error relative to a unit-magnitude result
        worst = max(worst, abs(s.v - ex_s) / 2 ** -24, abs(c.v - ex_c) / 2 ** -24)
    assert worst <= 4.0, worst


def test_acos_and_sin(orc):
    L = orc.lib()
    worst_a = max(ulp_err(L.orc_acosf(float(c)), math.acos(float(c)))
                  for c in np.concatenate([sample(0, 1, 20000), np.float32([0, 0.5, 1])]))
    assert worst_a <= 4.0, worst_a
    worst_s = max(ulp_err(L.orc_sinf(float(a)), math.sin(float(a)))
                  for a in sample(1e-3, math.pi / 2, 20000))
    assert worst_s <= 3.0, worst_s
    assert L.orc_acosf(1.0) == 0.0 and L.orc_sinf(0.0) == 0.0


class C_float:
    def __init__(self):
        import ctypes
        self._c = ctypes.c_float()
        self.ref = ctypes.byref(self._c)

    @property
    def v(self):
        return self._c.value
