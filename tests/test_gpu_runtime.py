"""Native runtime entry points on the GPU: the interval census
(cz_census_interval) and the serving runtime (cz_server_open / cz_submit /
cz_next_done / cz_poll).  Records must equal the reference's sample frames and
cz_census's own records bit for bit; a refused request in a merged batch must
be the only one refused."""
import ctypes

import pytest

from conftest import GOLDEN
from rabung_atlas32_b200 import codec, sieve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from rabung_atlas32_b200.census import Census
    with Census() as c:
        yield c


@pytest.mark.parametrize("block,lo,hi", [("00000", 1, 38891), ("49900", 4294915433, 1 << 32)])
def test_interval_census_equals_sample_frames(eng, block, lo, hi):
    primes, recs = eng.interval(lo, hi, mode="auto", a4=True, max_primes=4096)
    assert codec.encode_scan_frame(lo, hi, recs) == (GOLDEN / f"scan-{block}.vdw").read_bytes()
    assert codec.encode_a4_frame(lo, hi, recs) == (GOLDEN / f"quadruplets-{block}.a4").read_bytes()
    assert primes == [r.p for r in recs]


def test_interval_limits_and_empty(eng):
    from rabung_atlas32_b200 import _lib
    L, h = eng.lib, eng.h
    ps = (ctypes.c_uint32 * 10)()
    out = (_lib.cz_profile * 80)()
    npr, nprof = ctypes.c_uint32(), ctypes.c_uint32()
    # 25 primes below 100 do not fit 10 slots: CZ_ELIMIT with the needed count
    rc = L.cz_census_interval(h, 1, 100, _lib.CZ_AUTO, ps, 10, ctypes.byref(npr), out, 80, ctypes.byref(nprof),
                              None, None)
    assert rc == _lib.CZ_ELIMIT and npr.value == 25
    # a gap between primes holds none
    rc = L.cz_census_interval(h, 24, 29, _lib.CZ_AUTO, ps, 10, ctypes.byref(npr), out, 80, ctypes.byref(nprof),
                              None, None)
    assert rc == _lib.CZ_OK and npr.value == 0 and nprof.value == 0
    # profiles that do not fit: the needed count comes back
    ps64 = (ctypes.c_uint32 * 64)()
    rc = L.cz_census_interval(h, 1 << 24, (1 << 24) + 200, _lib.CZ_AUTO, ps64, 64, ctypes.byref(npr), out, 2,
                              ctypes.byref(nprof), None, None)
    want = sieve.primes_in(1 << 24, (1 << 24) + 200)
    assert rc == _lib.CZ_ELIMIT and npr.value == len(want) and nprof.value == eng.count_profiles(want)


def _server(slots=2, budget_mb=2048):
    from rabung_atlas32_b200 import _lib
    L = _lib.load()
    cfg = _lib.cz_config()
    L.cz_default_config(ctypes.byref(cfg))
    h = ctypes.c_void_p()
    assert L.cz_server_open(ctypes.byref(cfg), slots, budget_mb << 20, ctypes.byref(h)) == _lib.CZ_OK
    return L, h


def test_server_refusal_reaches_only_its_request(eng):
    from rabung_atlas32_b200 import _lib
    from rabung_atlas32_b200.census import to_records
    L, h = _server(slots=1)
    try:
        good = [sieve.primes_from(1 << 26, 40), sieve.primes_ending(4294967291, 24), sieve.primes_in(3, 500)]
        bad = sieve.primes_from(1 << 25, 8) + [(1 << 25) + 1]            # one composite
        ids = []
        for ps in good[:2] + [bad] + good[2:]:
            arr = (ctypes.c_uint32 * len(ps))(*ps)
            rid = ctypes.c_uint64()
            assert L.cz_submit(h, 0, len(ps), arr, _lib.CZ_AUTO | _lib.CZ_A4, ctypes.byref(rid)) == _lib.CZ_OK
            ids.append((rid.value, ps))
        for rid, ps in ids:
            out = (_lib.cz_profile * (8 * len(ps)))()
            a4 = (ctypes.c_uint32 * len(ps))()
            got = (ctypes.c_uint32 * len(ps))()
            npr, nprof = ctypes.c_uint32(), ctypes.c_uint32()
            rc = L.cz_poll(h, rid, 60000, got, len(ps), ctypes.byref(npr), out, 8 * len(ps), ctypes.byref(nprof), a4)
            if ps is bad:
                assert rc == _lib.CZ_EREFUSED and b"not prime" in L.cz_server_last_error(h)
                continue
            assert rc == _lib.CZ_OK and list(got[:npr.value]) == ps
            recs = to_records(ps, out, list(a4[:len(ps)]))
            alone = eng.profiles(ps, mode="auto", a4=True)
            assert [(r.p, [(v.r, v.M, v.L, v.witness, v.K) for v in r.profiles], r.a4) for r in recs] == \
                   [(r.p, [(v.r, v.M, v.L, v.witness, v.K) for v in r.profiles], r.a4) for r in alone]
        # nothing left: an idle server times out, an unknown id is refused
        rid = ctypes.c_uint64()
        assert L.cz_next_done(h, 0, ctypes.byref(rid)) == _lib.CZ_EPENDING     # polled ids are not announced
        assert L.cz_poll(h, 10 ** 9, 0, None, 0, None, None, 0, None, None) == _lib.CZ_EINVAL
    finally:
        L.cz_server_close(h)


def test_server_sieved_requests_and_next_done(eng):
    from rabung_atlas32_b200.serving import Server
    srv = Server(slots=2, slot_budget_mb=1024)
    try:
        reqs = [(1 << 20, 300), (4294967000, 50), (7, 1), (1 << 31, 2000)]
        ids = {srv.submit(lo, n): (lo, n) for lo, n in reqs}
        seen = set()
        while len(seen) < len(ids):
            rid = srv.next_done(60000)
            assert rid in ids and rid not in seen
            seen.add(rid)
            lo, n = ids[rid]
            primes, recs = srv.fetch(rid, n)
            exp = sieve.primes_in(lo, 1 << 32)[:n] if lo > (1 << 32) - 10 ** 6 else sieve.primes_from(lo, n)
            assert primes == exp
            alone = eng.profiles(primes, mode="auto", a4=True)
            assert [(r.p, [(v.r, v.M, v.L, v.witness) for v in r.profiles], r.a4) for r in recs] == \
                   [(r.p, [(v.r, v.M, v.L, v.witness) for v in r.profiles], r.a4) for r in alone]
        assert srv.next_done(10) is None
        assert srv.batches >= 1
    finally:
        srv.close()


def test_server_tight_plane_budget(eng):
    """Admission by device memory: with a 96 MiB plane budget, a request whose
    colour planes alone exceed it runs on the second handle in waves, while
    requests that fit only one or two at a time wait for space; every record
    equals cz_census's."""
    from rabung_atlas32_b200 import _lib
    from rabung_atlas32_b200.census import to_records
    L, h = _server(slots=1, budget_mb=96)
    try:
        big = sieve.primes_ending(4294967291, 200)          # ~200 x 2 MiB of planes near 2^32
        small = [sieve.primes_ending(4294967291 - k * 10 ** 6, 16) for k in range(6)]
        ids = []
        for ps in [big] + small:
            arr = (ctypes.c_uint32 * len(ps))(*ps)
            rid = ctypes.c_uint64()
            assert L.cz_submit(h, 0, len(ps), arr, _lib.CZ_AUTO | _lib.CZ_A4, ctypes.byref(rid)) == _lib.CZ_OK
            ids.append((rid.value, ps))
        for rid, ps in ids:
            out = (_lib.cz_profile * (8 * len(ps)))()
            a4 = (ctypes.c_uint32 * len(ps))()
            npr, nprof = ctypes.c_uint32(), ctypes.c_uint32()
            # A4's capacity is primes_cap: too small a one is CZ_ELIMIT and keeps the request
            rc = L.cz_poll(h, rid, 120000, None, 0, ctypes.byref(npr), out, 8 * len(ps), ctypes.byref(nprof), a4)
            assert rc == _lib.CZ_ELIMIT and npr.value == len(ps)
            rc = L.cz_poll(h, rid, 0, None, len(ps), ctypes.byref(npr), out, 8 * len(ps), ctypes.byref(nprof), a4)
            assert rc == _lib.CZ_OK
            recs = to_records(ps, out, list(a4[:len(ps)]))
            alone = eng.profiles(ps, mode="auto", a4=True)
            assert [(r.p, [(v.r, v.M, v.L, v.witness, v.K) for v in r.profiles], r.a4) for r in recs] == \
                   [(r.p, [(v.r, v.M, v.L, v.witness, v.K) for v in r.profiles], r.a4) for r in alone]
    finally:
        L.cz_server_close(h)


def test_server_speculation_misses_rerun_exact(eng):
    """Speculative thresholds at floor(log_r p) (margin 0) miss often; the
    server re-runs each missed prime on the anchor filter without speculation
    (no dense re-scan), and every record equals cz_census's."""
    from rabung_atlas32_b200.census import Tuning
    from rabung_atlas32_b200.serving import Server
    srv = Server(slots=1, slot_budget_mb=2048, tuning=Tuning(speculate=1, spec_margin10=(0,) * 10))
    try:
        reqs = [(4294967291 - 3 * 10 ** 6, 48), (1 << 31, 32)]
        ids = {srv.submit(lo, n): (lo, n) for lo, n in reqs}
        for rid, (lo, n) in ids.items():
            primes, recs = srv.fetch(rid, n)
            alone = eng.profiles(primes, mode="auto", a4=True)
            assert [(r.p, [(v.r, v.M, v.L, v.witness, v.K) for v in r.profiles], r.a4) for r in recs] == \
                   [(r.p, [(v.r, v.M, v.L, v.witness, v.K) for v in r.profiles], r.a4) for r in alone]
        st = srv.stats()
        assert st["respec_primes"] > 0
    finally:
        srv.close()
