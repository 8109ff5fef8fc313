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
