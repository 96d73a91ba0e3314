"""The oracle's restatement of the reference RNG against the reference's own
init_RNG (gpumcml_rng/gpumcml_rng.cu:59-118, compiled into oracle/_ref), plus the
jump-ahead identity the engine's parallel seeding rests on."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import ROOT

REF_RNG = ROOT / "oracle" / "_ref" / "libref_rng.so"
BEGIN_DEFAULT = 4294967118


def ref_lib():
    if not REF_RNG.exists():
        pytest.skip("reference RNG not built (oracle/build_ref.py needs the reference checkout)")
    h = C.CDLL(str(REF_RNG))
    h.ref_init_rng.restype = C.c_int
    h.ref_init_rng.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_char_p, C.c_uint64]
    return h


def write_table(path, table):
    with open(path, "w") as f:
        for a in table:
            p = (int(a) << 32) - 1
            f.write(f"{int(a)} {p >> 32} {p & 0xffffffff}\n")


def ref_init(tmp_path, table, seed, n):
    path = tmp_path / "safeprimes_base32.txt"
    write_table(path, table)
    x = np.zeros(n, np.uint64)
    a = np.zeros(n, np.uint32)
    rc = ref_lib().ref_init_rng(x.ctypes.data, a.ctypes.data, n, str(path).encode(), seed)
    return rc, x, a


@pytest.mark.parametrize("seed", [1, 12345, 1796308352, (1 << 32) - 2, (123 << 32) + 99])
def test_init_rng_matches_reference(tmp_path, orc, table, seed):
    n = 230_400  # the reference's slot count, src/mc3d_gpu.cu:434
    rc, x, a = ref_init(tmp_path, table[: n + 1], seed, n)
    assert rc == 0
    ox, oa = orc.init_rng(table[: n + 1], seed, n)
    assert np.array_equal(x, ox) and np.array_equal(a, oa)


def test_init_rng_rejections_match_reference(tmp_path, orc):
    """multipliers 2..17 make the validity loop (gpumcml_rng.cu:100) reject often"""
    small = np.array([BEGIN_DEFAULT] + [3, 5, 7, 11, 13, 2, 17] * 2000, np.uint32)
    n = len(small) - 1
    rc, x, a = ref_init(tmp_path, small, 987654321, n)
    assert rc == 0
    ox, oa = orc.init_rng(small, 987654321, n)
    assert np.array_equal(x, ox) and np.array_equal(a, oa)
    # and some streams did retry: their states differ from a no-retry seeding
    begin, m = BEGIN_DEFAULT, (BEGIN_DEFAULT << 32) - 1
    naive = [(987654321 * pow(begin, 2 * i + 2, m)) % m & 0xffffffff for i in range(50)]
    assert any(int(ox[i]) & 0xffffffff != naive[i] for i in range(50))


@pytest.mark.parametrize("seed", [0, (BEGIN_DEFAULT - 1) << 32, 0xffffffff])
def test_invalid_seeds_rejected_like_reference(tmp_path, orc, table, seed):
    rc, _, _ = ref_init(tmp_path, table[:11], seed, 10)
    assert rc == 1
    with pytest.raises(ValueError):
        orc.init_rng(table[:11], seed, 10)


def test_mwc_is_lcg_modulo_a_2_32_minus_1(orc):
    """x_{n+1} = a x_n mod (a 2^32 - 1) for the packed state: the identity behind
    the engine's jump-ahead seeding"""
    rng = np.random.default_rng(5)
    for _ in range(20):
        a = int(rng.integers(1 << 30, 1 << 32))
        m = (a << 32) - 1
        x0 = int(rng.integers(1, a - 1)) << 32 | int(rng.integers(0, 1 << 32 - 1))
        x = x0
        for n in range(1, 200):
            x = (x & 0xffffffff) * a + (x >> 32)
            assert x == x0 * pow(a, n, m) % m


def test_rand_co_restatement(orc, table):
    x, a = orc.init_rng(table, 4242, 16)
    for g in range(16):
        got = orc.rand_co(int(x[g]), int(a[g]), 500)
        st, m = int(x[g]), int(a[g])
        exp = np.zeros(500, np.float32)
        for d in range(500):
            st = (st & 0xffffffff) * m + (st >> 32)
            u = st & 0xffffffff
            if u >= 1 << 24:  # truncate to 24 significant bits (toward zero)
                drop = u.bit_length() - 24
                u = (u >> drop) << drop
            exp[d] = np.float32(u) * np.float32(2.0 ** -32)
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))
