"""GPU parity of the census engine, called through the C ABI.

Every M, L, witness, K and A4 is compared record for record with the
reference's shipped sample blocks, its holdout profiles, its dense-oracle
records and the outputs of its own CPU programs (fixtures in tests/golden),
and the sparse anchor filter is compared with the dense kernel.  All
integer results: the bar is bit-exact equality.
"""
import random

import pytest

import oracle
from conftest import load_gz
from rabung_atlas32_b200 import codec, sieve

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from rabung_atlas32_b200.census import Census
    with Census() as c:
        yield c


def tup(recs):
    return [(r.p, [(v.r, v.M, v.L, v.witness, v.K) for v in r.profiles]) for r in recs]


def golden_tup(recs):
    return [(r.p, [(v.r, v.M, v.L, v.witness, codec.minimum_k(r.p, v.r, v.M, v.L)) for v in r.profiles])
            for r in recs]


def test_first_256_primes_dense(eng, golden):
    """C1: the first 256 primes (2..1619), dense path, vs block 0."""
    recs, _, _ = golden["00000"]
    got = eng.profiles([r.p for r in recs[:256]], mode="dense", a4=True, verify=True)
    assert tup(got) == golden_tup(recs[:256])
    assert [r.a4 for r in got] == [r.a4 for r in recs[:256]]
    assert sum(r.a4 for r in got) == 23605


def test_block0_dense_frames(eng, golden):
    """Block 0 (4096 primes): profiles, A4 and both frames byte for byte."""
    recs, meta, _ = golden["00000"]
    got = eng.profiles([r.p for r in recs], mode="dense", a4=True)
    assert tup(got) == golden_tup(recs)
    from conftest import GOLDEN
    assert codec.encode_scan_frame(meta["lo"], meta["hi"], got) == (GOLDEN / "scan-00000.vdw").read_bytes()
    assert codec.encode_a4_frame(meta["lo"], meta["hi"], got) == (GOLDEN / "quadruplets-00000.a4").read_bytes()


def test_block49900_sparse_frames(eng, golden):
    """Block 49900 (2313 primes up to 4294967291): anchor filter, frames byte for byte."""
    recs, meta, _ = golden["49900"]
    got = eng.profiles([r.p for r in recs], mode="sparse", a4=True, verify=True)
    assert tup(got) == golden_tup(recs)
    assert [r.a4 for r in got] == [r.a4 for r in recs]
    from conftest import GOLDEN
    assert codec.encode_scan_frame(meta["lo"], meta["hi"], got) == (GOLDEN / "scan-49900.vdw").read_bytes()
    assert codec.encode_a4_frame(meta["lo"], meta["hi"], got) == (GOLDEN / "quadruplets-49900.a4").read_bytes()


@pytest.mark.parametrize("w", [0, 1, 2, 3])
def test_holdout_windows_sparse(eng, w):
    """4 x 1024 holdout primes at 0.257/1.337/2.971/4.237e9 (profiles_full)."""
    win = load_gz("holdout32.json.gz")[w]
    ps = [row[0] for row in win["rows"]]
    got = eng.profiles(ps, mode="sparse", a4=False)
    exp = [(p, [tuple(v) for v in prof]) for p, prof in win["rows"]]
    assert [(r.p, [(v.r, v.M, v.L, v.K, v.witness) for v in r.profiles]) for r in got] == exp


def test_dense_oracle_records(eng):
    """The reference GPU dense-oracle records below 2^32, by the sparse path."""
    recs = load_gz("dense_oracle.json.gz")
    ps = [p for p, _ in recs]
    got = eng.profiles(ps, mode="auto", a4=False)
    for (p, prof), r in zip(recs, got):
        assert [(v.r, v.M, v.L, v.K, v.witness) for v in r.profiles] == [tuple(v) for v in prof], p


def test_2p24_block_dense_vs_reference_and_sparse(eng):
    """C2: 4096 primes from 2^24: dense vs the reference full-walk program and
    moment_worker, and sparse == dense on every profile."""
    d = load_gz("refcpu_2p24.json.gz")
    ps = d["primes"]
    dense = eng.profiles(ps, mode="dense", a4=True)
    assert [r.a4 for r in dense] == d["a4"]
    by = {(r.p, v.r): (v.M, v.L, v.witness) for r in dense for v in r.profiles}
    for p, r, M, L, w in d["independent"]:
        assert by[(p, r)] == (M, L, w)
    sparse = eng.profiles(ps, mode="sparse", a4=False)
    assert tup(sparse) == tup(dense)


def test_top_block_sparse_vs_reference_cpu(eng, golden):
    """C3, all 13,660 profiles: 4096 primes ending at 4294967291 by the anchor
    filter, every record certified on the device.  The 1783 primes below
    block 49900 (5914 profiles) against the reference's own CPU sparse engines
    run on every one of their (p, r) pairs -- `target` for the coupled pairs
    {2, 4} and {3, 6}, `advance` for the other orders -- and the 2313 primes of
    block 49900 against its shipped frame; A4 against moment_worker for all."""
    d = load_gz("refcpu_top_block.json.gz")
    ps = d["primes"]
    got = eng.profiles(ps, mode="sparse", a4=True, verify=True)
    assert [r.a4 for r in got] == d["a4"]
    ref = {(p, r): (M, L, w) for p, r, M, L, w in d["advance"] + d["target"]}
    recs, _, _ = golden["49900"]
    top = {r.p: r for r in got}
    lower = [r for r in got if r.p < recs[0].p]
    n = 0
    for rec in lower:
        for v in rec.profiles:
            assert ref[(rec.p, v.r)] == (v.M, v.L, v.witness), (rec.p, v.r)
            n += 1
    assert n == len(ref) == 5914
    assert tup([top[r.p] for r in recs]) == golden_tup(recs)
    assert n + sum(len(r.profiles) for r in recs) == 13660


def test_top_block_dense_judge_1pct(eng):
    """C3 judge: the dense kernel re-runs a seeded 1% of (p, r) pairs of the top
    block; the anchor filter must agree on every one."""
    ps = sieve.primes_ending(4294967291, 4096)
    rng = random.Random(20261203)
    pick = sorted(rng.sample(ps, 41))
    sparse = eng.profiles(pick, mode="sparse", a4=False)
    dense = eng.profiles(pick, mode="dense", a4=False)
    assert tup(sparse) == tup(dense)


def test_small_primes_oracle(eng):
    """Every prime below 5000 (dense path; p=2 has no profile) vs the CPU oracle."""
    ps = sieve.primes_in(2, 5000)
    got = eng.profiles(ps, mode="auto", a4=True)
    for r in got:
        exp = oracle.profiles(r.p) if r.p > 2 else []
        assert [(v.r, v.M, v.L, v.witness, v.K) for v in r.profiles] == \
               [(v["r"], v["max"], v["prefix"], v["witness"], v["K"]) for v in exp], r.p
        assert r.a4 == (oracle.a4(r.p) if r.p > 2 else 0), r.p


def test_sparse_threshold_region_vs_oracle(eng):
    """Primes just above the sparse routing threshold: sparse == CPU oracle walk."""
    ps = sieve.primes_from(1 << 20, 48)
    got = eng.profiles(ps, mode="sparse", a4=True)
    for r in got:
        exp = oracle.profiles(r.p)
        assert [(v.r, v.M, v.L, v.witness) for v in r.profiles] == \
               [(v["r"], v["max"], v["prefix"], v["witness"]) for v in exp], r.p
        assert r.a4 == oracle.a4(r.p)


def test_refusal_on_composite(eng):
    """A non-prime is refused, and cheaply: setup marks it, and the table,
    filter and A4 kernels do no work for it (every colour window of a
    non-prime would match, so filtering it runs for tens of seconds)."""
    import time
    from rabung_atlas32_b200.census import CensusError
    with pytest.raises(CensusError):
        eng.profiles([4294967291, 4294967293], mode="sparse", a4=False)
    t0 = time.perf_counter()
    with pytest.raises(CensusError, match="status"):
        eng.profiles(sieve.primes_from(1 << 25, 8) + [(1 << 25) + 1], mode="sparse", a4=True)
    assert time.perf_counter() - t0 < 5.0


def test_filter_counters_cover_the_plane_pool(eng):
    """The in-run traffic figure (cz_stats.staged_bytes, the bench's
    roofline.traffic) counts every tile the filter copies into shared memory:
    tiles cover every word of both views of every profile, so one sparse call
    stages at least its whole plane pool; the filter's work counters are
    positive and the tests are at least one stage per counted lane-word."""
    ps = sieve.primes_ending(4294967291, 32)
    _, _, st = eng.raw(ps, mode="sparse", a4=False)
    pool = eng.plane_bytes(ps, mode="sparse")
    assert pool > 0 and st["staged_bytes"] >= pool
    assert st["words"] > 0 and st["tests"] >= st["words"] and st["completions"] > 0


def test_replay_bit_identical(eng):
    ps = sieve.primes_ending(4294967291, 64)
    a = eng.profiles(ps, mode="sparse", a4=False)
    st = eng.replay()
    assert st["n_profiles"] == sum(len(r.profiles) for r in a)
    b = eng.profiles(ps, mode="sparse", a4=False)
    assert tup(a) == tup(b)


def test_anchor_stages_do_not_change_records():
    """The per-order anchor stage counts trade filter work for screen and
    completion work; the records are certified either way and must not move."""
    import dataclasses
    from rabung_atlas32_b200.census import Census, Tuning
    ps = sieve.primes_ending(4294967291, 64)
    with Census(tuning=Tuning()) as c0:
        want = tup(c0.profiles(ps, mode="sparse", a4=False))
    for at in [(0, 0, 2, 2, 2, 2, 2, 2, 2, 2), (0, 0, 16, 10, 9, 8, 7, 7, 6, 6), (0,) * 10]:
        with Census(tuning=dataclasses.replace(Tuning(), anchor_t=at)) as c1:
            assert tup(c1.profiles(ps, mode="sparse", a4=False)) == want, at


def test_speculation_miss_rerun_exact():
    """Speculative thresholds at floor(log_r p) (margin 0) miss often; every miss
    is re-run without speculation and the records equal the unspeculated ones."""
    from rabung_atlas32_b200.census import Census, Tuning
    ps = sieve.primes_ending(4294967291, 96)
    with Census(tuning=Tuning(speculate=0)) as c0:
        want = tup(c0.profiles(ps, mode="sparse", a4=False))
    with Census(tuning=Tuning(speculate=1, spec_margin10=(0,) * 10)) as c1:
        got = tup(c1.profiles(ps, mode="sparse", a4=False))
        assert c1.last_stats["n_respec"] > 0
    assert got == want


def test_refusal_leaves_no_stale_state(eng):
    """A refused call (a composite: its A4 is not certified) followed, on the
    same handle, by an all-dense call with A4 must succeed: no status of the
    refused call survives into the next one."""
    from rabung_atlas32_b200.census import CensusError
    with pytest.raises(CensusError):
        eng.profiles(sieve.primes_from(1 << 25, 4) + [(1 << 25) + 1], mode="auto", a4=True)
    small = sieve.primes_in(3, 500)
    got = eng.profiles(small, mode="auto", a4=True)
    assert [r.a4 for r in got] == [oracle.a4(p) for p in small]


def test_reference_c_abi_baseline_profile(golden):
    """The reference's own in-process C ABI (baseline_init / baseline_profile,
    src/census/engine32/src/baseline_bridge.cu:7,21-27), called through ctypes
    as a reference maintainer would bind it: M into out[r] and L into
    prefix[r] equal block 49900's records; with full = 0 only the masks
    1, 5, 18, 19, 23 are served and any other returns 2, as there."""
    import ctypes
    from rabung_atlas32_b200 import _lib
    lib = _lib.load()
    lib.baseline_init(0xFFFFFFFF)
    recs, _, _ = golden["49900"]
    rng = random.Random(20261203)
    served = {1: {2}, 5: {2, 4}, 18: {3, 6}, 19: {2, 3, 6}, 23: {2, 3, 4, 6}}
    checked = 0
    for rec in rng.sample(recs, 40):
        adm = {v.r for v in rec.profiles}
        mask_all = sum(1 << (r - 2) for r in adm)
        by = {v.r: (v.M, v.L) for v in rec.profiles}
        out = (ctypes.c_uint * 10)()
        pre = (ctypes.c_uint * 10)()
        assert lib.baseline_profile(rec.p, mask_all, out, pre, 1) == 0
        for r in adm:
            assert (out[r], pre[r]) == by[r], (rec.p, r)
            checked += 1
        for mask, rs in served.items():
            out2 = (ctypes.c_uint * 10)()
            pre2 = (ctypes.c_uint * 10)()
            rc = lib.baseline_profile(rec.p, mask, out2, pre2, 0)
            if rs <= adm:
                assert rc == 0
                assert all((out2[r], pre2[r]) == by[r] for r in rs), (rec.p, mask)
            else:
                assert rc == 2, (rec.p, mask)
        # a mask outside the five without `full` is refused even when admissible
        if {2, 3} <= adm:
            assert lib.baseline_profile(rec.p, 0b11, out, pre, 0) == 2
            assert lib.baseline_profile(rec.p, 0b11, out, pre, 1) == 0
    assert checked > 100


def test_epoch_rows_do_not_change_records():
    """Rows per threshold epoch (one row per epoch up to one epoch per profile)
    only change when the filter's threshold rises; the records are certified
    either way and must not move."""
    import dataclasses
    from rabung_atlas32_b200.census import Census, Tuning
    ps = sieve.primes_ending(4294967291, 48) + sieve.primes_from(1 << 24, 48)
    with Census(tuning=Tuning()) as c0:
        want = tup(c0.profiles(ps, mode="sparse", a4=False))
    for er in (1, 7, 64, 256, 1 << 20):
        with Census(tuning=dataclasses.replace(Tuning(), epoch_rows=er)) as c1:
            assert tup(c1.profiles(ps, mode="sparse", a4=False)) == want, er


def test_small_tiles_do_not_change_records(tmp_path):
    """A library built with 16 KiB shared-memory tiles (instead of 80 KiB) cuts
    every view into many tiles (up to ~20 per view here), so bands, halos and
    tile edges are crossed everywhere; its records must equal the default
    build's, with no prime sent back to the dense path."""
    from rabung_atlas32_b200 import _lib, build
    from rabung_atlas32_b200.census import Census, Tuning
    ps = sieve.primes_from(1 << 26, 40) + sieve.primes_from(1 << 28, 40) + sieve.primes_ending(1 << 30, 24)
    with Census(tuning=Tuning()) as c0:
        want = tup(c0.profiles(ps, mode="sparse", a4=False))
    so = tmp_path / "librabung_census_tile4k.so"
    build.compile_library(so, extra=["-DCZ_TILE_WORDS=4096"])
    lib = _lib.load(so)
    saved = _lib._lib
    try:
        _lib._lib = lib
        with Census(tuning=Tuning()) as c1:
            got = c1.profiles(ps, mode="sparse", a4=False)
            assert c1.last_stats["n_fallback"] == 0
            assert tup(got) == want
    finally:
        _lib._lib = saved
