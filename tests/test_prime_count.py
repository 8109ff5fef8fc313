"""Exact prime counts on the host (cz_prime_count; runs without a GPU).

The library sizes interval buffers from pi(hi - 1) - pi(lo - 1) (the role of
the reference's Meissel-Lehmer count, src/census/prime_count.cpp:11-24).
Checked against a numpy sieve on short intervals, against published values of
pi(x) and against the shipped sample blocks' prime counts.
"""
import numpy as np
import pytest

from rabung_atlas32_b200.census import prime_count


def sieve_count(lo, hi):
    s = np.ones(hi, dtype=bool)
    s[:2] = False
    for q in range(2, int(hi ** 0.5) + 1):
        if s[q]:
            s[q * q::q] = False
    return int(s[lo:hi].sum())


@pytest.mark.parametrize("lo,hi", [(0, 0), (0, 2), (0, 3), (2, 3), (3, 3), (0, 100), (97, 98), (98, 100),
                                   (1000, 2000), (10 ** 6, 10 ** 6 + 12345), (2 ** 20, 2 ** 20 + 8192)])
def test_short_intervals_vs_sieve(lo, hi):
    assert prime_count(lo, hi) == sieve_count(lo, hi)


def test_long_intervals_vs_sieve():
    # intervals longer than the short-interval sieve: the Lucy-Hedgehog path
    for lo, hi in [(0, 10 ** 7), (12345, 9 * 10 ** 6 + 7), (2 ** 22 + 1, 2 ** 24 - 3)]:
        assert prime_count(lo, hi) == sieve_count(lo, hi), (lo, hi)


def test_published_values():
    # pi(10^k), pi(2^32), pi(2^33)
    assert prime_count(0, 10 ** 6 + 1) == 78498
    assert prime_count(0, 10 ** 9 + 1) == 50847534
    assert prime_count(0, 2 ** 32) == 203280221
    assert prime_count(0, 2 ** 33) == 393615806


def test_sample_block_counts(golden):
    for blk in ("00000", "49900"):
        recs, meta, _ = golden[blk]
        assert prime_count(meta["lo"], meta["hi"]) == len(recs) == meta["count"]
