"""RNG parity on the GPU: the engine's multiply-with-carry draws and stream seeds
against the reference's own rand_MWC_co (compiled from gpumcml_rng/gpumcml_rng.cu,
run in a kernel) and against the oracle's init_RNG restatement."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

REF_RNG = ROOT / "oracle" / "_ref" / "libref_rng.so"


def ref_rng():
    assert REF_RNG.exists(), "oracle/_ref/libref_rng.so missing: run oracle/build_ref.py"
    h = C.CDLL(str(REF_RNG))
    h.ref_mwc_draws.restype = C.c_int
    h.ref_mwc_draws.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    h.ref_conversion_mismatches.restype = C.c_longlong
    h.ref_conversion_mismatches.argtypes = [C.c_ulonglong, C.c_ulonglong]
    return h


def test_draws_bit_exact_vs_reference_kernel(engine, orc, table):
    x, a = orc.init_rng(table, 12345, 4096)
    ours = engine.mwc_draws(x, a, 1000)
    ref = np.zeros_like(ours)
    assert ref_rng().ref_mwc_draws(x.ctypes.data, a.ctypes.data, len(x), 1000,
                                   ref.ctypes.data) == 0
    assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32))
    for g in range(0, 4096, 512):
        assert np.array_equal(orc.rand_co(int(x[g]), int(a[g]), 1000).view(np.uint32),
                              ours[g].view(np.uint32))


def test_float_conversion_exhaustive():
    """rand_MWC_co's __fdividef(__uint2float_rz(u), 2^32) equals the engine's
    __uint2float_rz(u) * 2^-32 for every 32-bit u."""
    assert ref_rng().ref_conversion_mismatches(0, 1 << 32) == 0


@pytest.mark.parametrize("seed", [1, 12345, 1796308352, (1 << 32) - 2, (77 << 32) + 5])
def test_stream_seeds_match_init_rng(engine, orc, table, seed):
    job = engine.Job(photons=10 ** 8, seed=seed)
    n = 300_000
    x, a = engine.stream_seeds(job, 0, n, table)
    ox, oa = orc.init_rng(table, seed, n)
    assert np.array_equal(x, ox) and np.array_equal(a, oa)


def test_stream_seeds_deep_and_wrapping(engine, orc, table):
    """streams far into a job, beyond the table length (multipliers wrap)"""
    short = table[:1001]
    job = engine.Job(photons=10 ** 8, seed=424242)
    first = 4_000_000
    x, a = engine.stream_seeds(job, first, 2000, short)
    ox, oa = orc.init_rng(short, 424242, first + 2000)
    assert np.array_equal(x, ox[first:]) and np.array_equal(a, oa[first:])


def test_stream_seeds_with_rejections(engine, orc):
    """tiny multipliers make init_RNG reject attempts often; every later stream
    shifts by the rejected attempts"""
    small = np.array([4294967118] + [3, 5, 7, 11, 13, 2, 17] * 300, np.uint32)
    job = engine.Job(photons=50_000, seed=987654321)
    x, a = engine.stream_seeds(job, 0, 50_000, small)
    ox, oa = orc.init_rng(small, 987654321, 50_000)
    assert np.array_equal(x, ox) and np.array_equal(a, oa)
