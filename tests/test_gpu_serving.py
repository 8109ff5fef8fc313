"""Serving: continuous batching changes no record -- every request's result is
the same served in the mix as computed alone."""
import pytest

from rabung_atlas32_b200 import sieve

pytestmark = pytest.mark.gpu


def test_each_request_same_alone_and_in_mix():
    from rabung_atlas32_b200.census import Census
    from rabung_atlas32_b200.serving import Server, make_trace
    trace = make_trace(48, rate=400.0, seed=7)
    srv = Server(slots=2, slot_budget_mb=2048)
    try:
        srv.run(trace)
    finally:
        srv.close()
    assert srv.batches >= 2
    mixed = {r.rid: r for r in trace}
    with Census() as c:
        for r in trace:
            assert r.done >= r.arrival
            assert r.primes == sieve.primes_from(r.lo, r.count)
            alone = c.profiles(r.primes, mode="auto", a4=True)
            got = mixed[r.rid].records
            assert [(x.p, [(v.r, v.M, v.L, v.witness, v.K) for v in x.profiles], x.a4) for x in got] == \
                   [(x.p, [(v.r, v.M, v.L, v.witness, v.K) for v in x.profiles], x.a4) for x in alone]


def test_arrivals_join_the_running_filter():
    """Requests that arrive while the filter is running a large request are
    merged into that work: the running launch yields between work items (the
    scheduler's yield counter rises) and is relaunched over the old and new
    profiles together, and every record equals the request computed alone."""
    import time
    from rabung_atlas32_b200.census import Census
    from rabung_atlas32_b200.serving import Server
    srv = Server(slots=1, slot_budget_mb=8192)
    try:
        big = (4290000000, 2048)                        # ~6,800 profiles near 2^32: ~0.4 s of filter
        small = [((1 << 26) + 10 ** 5 * k, 8) for k in range(4)]
        ids = {srv.submit(*big): big}
        time.sleep(0.1)                                 # past its admission, inside its filter launch
        for lo, n in small:
            ids[srv.submit(lo, n)] = (lo, n)
        got = {rid: srv.fetch(rid, n) for rid, (lo, n) in ids.items()}
        st = srv.stats()
    finally:
        srv.close()
    assert st["yields"] >= 1 and st["launches"] >= 2
    with Census() as c:
        for rid, (lo, n) in ids.items():
            primes, recs = got[rid]
            assert primes == sieve.primes_from(lo, n)
            alone = c.profiles(primes, mode="auto", a4=True)
            assert [(x.p, [(v.r, v.M, v.L, v.witness, v.K) for v in x.profiles], x.a4) for x in recs] == \
                   [(x.p, [(v.r, v.M, v.L, v.witness, v.K) for v in x.profiles], x.a4) for x in alone]
