"""Host segmented sieve for interval requests (the reference's bounded sieve,
src/census/prime_sieve.cpp:8-22, without its 2e6 width limit)."""
from __future__ import annotations

import numpy as np


def _base_primes(limit: int) -> np.ndarray:
    s = np.ones(limit + 1, dtype=bool)
    s[:2] = False
    for q in range(2, int(limit ** 0.5) + 1):
        if s[q]:
            s[q * q::q] = False
    return np.nonzero(s)[0]


def primes_in(lo: int, hi: int) -> list:
    """Primes in [lo, hi), hi <= 2^32."""
    if hi > 2 ** 32 or lo < 0:
        raise ValueError("interval outside [0, 2^32]")
    if hi <= lo:
        return []
    top = int(np.sqrt(hi)) + 1
    mark = np.ones(hi - lo, dtype=bool)
    for q in _base_primes(top):
        q = int(q)
        first = max(q * q, (lo + q - 1) // q * q)
        if first < hi:
            mark[first - lo::q] = False
    if lo <= 1:
        mark[: 2 - lo] = False
    return [int(x) + lo for x in np.nonzero(mark)[0]]


def primes_from(start: int, count: int) -> list:
    """The first `count` primes >= start."""
    out, lo = [], start
    width = 1 << 16
    while len(out) < count:
        hi = min(2 ** 32, lo + width)
        out += primes_in(lo, hi)
        if hi == 2 ** 32:
            break
        lo, width = hi, width * 2
    return out[:count]


def primes_ending(top: int, count: int) -> list:
    """The last `count` primes <= top."""
    out, hi = [], top + 1
    width = 1 << 16
    while len(out) < count and hi > 2:
        lo = max(0, hi - width)
        out = primes_in(lo, hi) + out
        hi, width = lo, width * 2
    return out[-count:]
