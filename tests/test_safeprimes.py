"""The safe-prime table generator: Marsaglia's MWC condition, order, file format
(readable by the reference's init_RNG, whose file is not distributed)."""
from __future__ import annotations

import numpy as np


def is_prime(n: int) -> bool:
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    d, r = n - 1, 0
    while d % 2 == 0:
        d //= 2
        r += 1
    for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(r - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def test_condition_and_order(engine):
    t = engine.safeprime_table(300)
    assert t[0] == 4294967118  # largest a < 2^32 with a*2^32-1 and a*2^31-1 prime
    assert np.all(np.diff(t.astype(np.int64)) < 0)
    for a in t[::7]:
        a = int(a)
        assert is_prime((a << 32) - 1) and is_prime((a << 31) - 1)


def test_no_multiplier_skipped(engine):
    """every a between two consecutive table entries fails the condition"""
    t = engine.safeprime_table(6)
    have = set(int(a) for a in t)
    for a in range(int(t[-1]), int(t[0]) + 1):
        ok = is_prime((a << 32) - 1) and is_prime((a << 31) - 1)
        assert ok == (a in have), a


def test_bound_and_threads_deterministic(engine):
    a = engine.safeprime_table(2000, threads=1)
    b = engine.safeprime_table(2000, threads=8)
    assert np.array_equal(a, b)
    c = engine.safeprime_table(50, below=int(a[10]))
    assert np.array_equal(c, a[11:61])


def test_text_round_trip(engine, tmp_path, table):
    path = tmp_path / "safeprimes_base32.txt"
    engine.write_safeprimes(path, table[:1000])
    back = engine.read_safeprimes(path, cap=5000)
    assert np.array_equal(back, table[:1000])
    first = path.read_text().splitlines()[0].split()
    a = int(first[0])
    assert (int(first[1]) << 32 | int(first[2])) == (a << 32) - 1
