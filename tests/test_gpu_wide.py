"""The 33-bit domain (primes below 2^33) through cz_census64, bit-exact
against the reference's data for that domain: the 2 x 1024 holdout primes of
its 33-bit engine (profiles_full), its GPU dense-oracle records between 2^32
and 2^33, and A4 from its own point counter (elliptic4_mestre.cpp); below
2^32 the wide build must reproduce the 32-bit records (block 49900's frame)."""
import ctypes

import pytest

import oracle
from conftest import load_gz
from rabung_atlas32_b200 import codec, sieve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wide():
    from rabung_atlas32_b200.census import Census64
    with Census64() as c:
        yield c


def rows(recs):
    return [(r.p, [(v.r, v.M, v.L, v.K, v.witness) for v in r.profiles]) for r in recs]


@pytest.mark.parametrize("w", [0, 1])
def test_holdout33_windows_sparse_and_a4(wide, w):
    d = load_gz("wide33.json.gz")
    win = d["holdout"][w]
    ps = [row[0] for row in win["rows"]]
    assert all(2 ** 32 < p < 2 ** 33 for p in ps)
    got = wide.profiles(ps, mode="sparse", a4=True, verify=True)
    assert rows(got) == [(p, [tuple(v) for v in prof]) for p, prof in win["rows"]]
    assert [r.a4 for r in got] == [d["a4"][str(p)] for p in ps]


def test_dense_oracle33_records(wide):
    recs = load_gz("wide33.json.gz")["dense_oracle"]
    got = wide.profiles([p for p, _ in recs], mode="auto", a4=False)
    assert rows(got) == [(p, [tuple(v) for v in prof]) for p, prof in recs]


def test_wide_dense_equals_wide_sparse():
    """The dense half-interval scan in 64-bit words agrees with the anchor filter
    on primes at both ends of (2^32, 2^33)."""
    from rabung_atlas32_b200.census import Census64
    ps = [4294967311, 5389000007, 8589934583]
    with Census64() as c:
        dense = rows(c.profiles(ps, mode="dense", a4=False))
        sparse = rows(c.profiles(ps, mode="sparse", a4=False))
    assert dense == sparse


def test_wide_build_reproduces_32bit_records(wide, golden):
    """Below 2^32 the 64-bit build reproduces block 49900 (anchor filter, frames
    byte for byte) and the C oracle on small primes (dense)."""
    recs, meta, _ = golden["49900"]
    got = wide.profiles([r.p for r in recs], mode="sparse", a4=True)
    from conftest import GOLDEN
    assert codec.encode_scan_frame(meta["lo"], meta["hi"], got) == (GOLDEN / "scan-49900.vdw").read_bytes()
    assert codec.encode_a4_frame(meta["lo"], meta["hi"], got) == (GOLDEN / "quadruplets-49900.a4").read_bytes()
    small = sieve.primes_in(3, 3000)
    for r in wide.profiles(small, mode="dense", a4=True):
        exp = oracle.profiles(r.p)
        assert [(v.r, v.M, v.L, v.witness, v.K) for v in r.profiles] == \
               [(v["r"], v["max"], v["prefix"], v["witness"], v["K"]) for v in exp], r.p
        assert r.a4 == oracle.a4(r.p), r.p


def test_wide_refusals(wide):
    """A composite is refused as a whole request; p >= 2^33 is out of domain."""
    from rabung_atlas32_b200 import _lib
    from rabung_atlas32_b200.census import CensusError
    with pytest.raises(CensusError):
        wide.profiles([5389000007, 5389000013], mode="sparse", a4=False)   # 37 x 83 x 1754803
    lib = _lib.load()
    arr = (ctypes.c_uint64 * 1)(2 ** 33 + 17)
    out = (_lib.cz_profile64 * 8)()
    assert lib.cz_census64(wide.h, arr, 1, _lib.CZ_AUTO, out, 8, None, None) == _lib.CZ_EINVAL
