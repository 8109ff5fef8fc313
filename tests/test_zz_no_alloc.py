"""The allocation-free dense census entry point (cz_census_dense_noalloc).

It exists for callers that cannot call cudaMalloc (plugins in a host process
that owns the device memory budget, allocator-free services that must not grow
their device footprint after start-up): its only device scratch is a fixed
2 MiB array inside the library, and the call is synchronous.  This file is collected last so that a
run stopping at the first failure has already run every other test.  The
records must equal those of the regular entry point (cz_census, dense mode)
exactly -- integer results, zero tolerance -- on two calls in a row (the
array keeps the previous call's contents), and requests beyond the fixed
limits must be refused.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def _primes():
    from rabung_atlas32_b200 import sieve
    small = sieve.primes_in(2, 200)                      # 46 primes, p = 2 included
    big = sieve.primes_from(4_000_000, 18)               # near the 4,194,304 limit
    return small + big


def _noalloc(lib, ps):
    from rabung_atlas32_b200 import _lib
    arr = (ctypes.c_uint32 * len(ps))(*ps)
    nprof = lib.cz_count_profiles(arr, len(ps))
    out = (_lib.cz_profile * max(1, nprof))()
    rc = lib.cz_census_dense_noalloc(arr, len(ps), out, nprof, None)
    return rc, [(o.p, o.r, o.M, o.L, o.witness, o.status, o.K) for o in out[:nprof]]


def _regular(ps):
    from rabung_atlas32_b200.census import Census
    with Census() as c:
        out, _, _ = c.raw(ps, mode="dense", a4=False)
        n = c.count_profiles(ps)
        return [(o.p, o.r, o.M, o.L, o.witness, o.status, o.K) for o in out[:n]]


def test_noalloc_matches_regular_entry_twice():
    from rabung_atlas32_b200 import _lib
    lib = _lib.load()
    ps = _primes()
    assert len(ps) <= 64
    want = _regular(ps)
    rc1, got1 = _noalloc(lib, ps)
    assert rc1 == _lib.CZ_OK
    assert got1 == want
    # second call: the shared array still holds the first call's contents
    rc2, got2 = _noalloc(lib, ps[::-1])
    assert rc2 == _lib.CZ_OK
    assert got2 == _regular(ps[::-1])
    rc3, got3 = _noalloc(lib, ps)
    assert rc3 == _lib.CZ_OK and got3 == want


def test_noalloc_refuses_beyond_limits():
    from rabung_atlas32_b200 import _lib, sieve
    lib = _lib.load()
    rc, _ = _noalloc(lib, sieve.primes_from(1000, 65))          # more than 64 primes
    assert rc == _lib.CZ_ELIMIT
    rc, _ = _noalloc(lib, [4_194_319])                          # p above the limit
    assert rc == _lib.CZ_ELIMIT
    rc, _ = _noalloc(lib, [4_000_001])                          # composite: refused
    assert rc == _lib.CZ_EREFUSED
