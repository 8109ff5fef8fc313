"""Pins the CPU oracle (oracle/census_oracle.c) to the reference's own
golden vectors: the shipped sample blocks, the holdout profiles and the
outputs of the reference CPU programs built into oracle/_ref."""
import random

import pytest

import oracle
from conftest import load_gz


def test_block0_profiles_and_a4(golden):
    recs, meta, _ = golden["00000"]
    for rec in recs:
        if rec.p < 3:
            assert rec.a4 == 0 and not rec.profiles
            continue
        got = [(v["r"], v["max"], v["prefix"], v["witness"]) for v in oracle.profiles(rec.p)]
        assert got == [(v.r, v.M, v.L, v.witness) for v in rec.profiles], rec.p
        assert oracle.a4(rec.p) == rec.a4, rec.p


def test_block49900_a4(golden):
    recs, _, _ = golden["49900"]
    for rec in recs[::7]:
        assert oracle.a4(rec.p) == rec.a4


def test_block49900_prefix(golden):
    recs, _, _ = golden["49900"]
    for rec in recs[::29]:
        for v in rec.profiles:
            assert oracle.prefix(rec.p, v.r) == v.L


def test_worked_example_p101():
    (v,) = oracle.profiles(101, 1)
    assert (v["max"], v["prefix"], v["K"], v["witness"]) == (7, 1, 8, 19)


def test_dense_vs_independent_2p24():
    d = load_gz("refcpu_2p24.json.gz")
    for p, r, M, L, w in d["independent"][:6]:
        (v,) = oracle.profiles(p, 1 << (r - 2))
        assert (v["max"], v["prefix"], v["witness"]) == (M, L, w)
    for p, a in list(zip(d["primes"], d["a4"]))[::97]:
        assert oracle.a4(p) == a


def test_a4_dense_equals_elliptic():
    rng = random.Random(7)
    primes = [p for p in range(1009, 40000) if oracle.is_prime(p)]
    for p in rng.sample(primes, 25):
        assert oracle.a4(p) == oracle.a4_dense(p)


def test_primality_and_sieve():
    ps = oracle.sieve(4294967000, 4294967296)
    assert ps[-1] == 4294967291
    assert all(oracle.is_prime(p) for p in ps)
    assert [p for p in range(4294967000, 4294967296) if oracle.is_prime(p)] == ps
    assert not oracle.is_prime(3215031751)   # strong pseudoprime to 2,3,5,7
