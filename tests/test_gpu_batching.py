"""Device sieve, waves and uneven multi-block batches (bit-exact)."""
import numpy as np
import pytest

from rabung_atlas32_b200 import sieve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from rabung_atlas32_b200.census import Census
    with Census() as c:
        yield c


def tup(recs):
    return [(r.p, [(v.r, v.M, v.L, v.witness, v.K) for v in r.profiles], r.a4) for r in recs]


def test_device_sieve_matches_host(eng):
    reqs = [(0, 10), (2, 1), (3, 5), (4096, 4096), (1 << 20, 100), (16777259, 4096),
            (4294967000, 20), (4294875371, 4096), (2 ** 32 - 10, 5)]
    got = eng.sieve(reqs)
    for (lo, cnt), g in zip(reqs, got):
        assert g == sieve.primes_from(lo, cnt), (lo, cnt)


def uneven_blocks(nblocks, size, seed=20261203):
    rng = np.random.default_rng(seed)
    starts = np.exp2(rng.uniform(16, 32, nblocks)).astype(np.int64)
    return [sieve.primes_from(int(s), size) for s in sorted(starts)]


def test_uneven_batch_equals_per_block(eng):
    """C4 form at reduced size: one batched call == one call per block."""
    blocks = uneven_blocks(8, 512)
    flat = [p for b in blocks for p in b]
    batched = eng.profiles(flat, mode="auto", a4=True)
    per = [r for b in blocks for r in eng.profiles(b, mode="auto", a4=True)]
    assert tup(batched) == tup(per)


def test_waves_equal_single_call():
    """A plane budget small enough to force several waves changes no record."""
    from rabung_atlas32_b200.census import Census, Tuning
    ps = sieve.primes_ending(4294967291, 200) + sieve.primes_from(1 << 22, 100)
    with Census() as c:
        one = tup(c.profiles(ps, mode="auto", a4=True))
        assert c.last_stats["waves"] == 1
    with Census(tuning=Tuning(plane_budget_mb=64)) as c:
        many = tup(c.profiles(ps, mode="auto", a4=True))
        assert c.last_stats["waves"] > 1
    assert one == many
