"""Atlas writer (packs, ledgers, chains) on CPU, fed with the reference's own
sample blocks decoded from the committed golden frames: the packs must hold
those frames byte for byte, the ledger rows must carry the sample manifest's
commitments, and the verifier must re-derive everything from the stored bytes.
Crash recovery, atomic commits, resume and pack roll-over are exercised with
faults made on the host (a torn pack tail, an aborting ledger insert)."""
import json
import random
import sqlite3
import subprocess
import sys

import pytest

from conftest import GOLDEN, ROOT
from rabung_atlas32_b200 import codec, ledger


def sample(block):
    recs, meta = codec.decode_scan_frame((GOLDEN / f"scan-{block}.vdw").read_bytes())
    vals, _ = codec.decode_a4_frame((GOLDEN / f"quadruplets-{block}.a4").read_bytes())
    for r, v in zip(recs, vals):
        r.a4 = v
    return recs, meta


@pytest.fixture(scope="module")
def blocks():
    return {"00000": sample("00000"), "49900": sample("49900")}


def test_sample_blocks_byte_identical_and_committed(tmp_path, blocks):
    manifest = {b["block"]: b for b in json.loads((GOLDEN / "manifest.json").read_text())["blocks"]}
    with ledger.Atlas(tmp_path, contiguous=False) as at:
        for name, bid in (("00000", 0), ("49900", 49900)):
            recs, meta = blocks[name]
            info = at.append(meta["lo"], meta["hi"], recs, block=bid)
            assert info["prime_hash"] == manifest[bid]["prime_hash"]
            assert info["science_hash"] == manifest[bid]["science_hash"]
            assert info["values_hash"] == manifest[bid]["values_hash"]
        for name, bid in (("00000", 0), ("49900", 49900)):
            assert at.frame("scan", bid) == (GOLDEN / f"scan-{name}.vdw").read_bytes()
            assert at.frame("quadruplets", bid) == (GOLDEN / f"quadruplets-{name}.a4").read_bytes()
        res = at.verify()
        sc, ac = codec.CHAIN_ZERO, codec.CHAIN_ZERO
        for name in ("00000", "49900"):
            recs, meta = blocks[name]
            sc, ac = codec.chain_step(sc, ac, meta["lo"], meta["hi"], recs)
        assert (res["profile_chain"], res["A4_chain"]) == (sc.hex(), ac.hex())
        assert res["primes"] == 4096 + 2313
        assert res["sum_A4"] == 9362607 + 1241775084440
        best = {r: (M, p) for r, M, p in at.db.execute("SELECT r, M, p FROM best")}
        allp = [(pr.r, pr.M, -rec.p) for name in blocks for rec in blocks[name][0] for pr in rec.profiles]
        for r in range(2, 10):
            M, negp = max((m, q) for rr, m, q in allp if rr == r)
            assert best[r] == (M, -negp)


def split_block0(blocks, cut):
    recs, meta = blocks["00000"]
    return [(1, recs[cut].p, recs[:cut]), (recs[cut].p, meta["hi"], recs[cut:])]


def test_contiguity_resume_and_rollover(tmp_path, blocks):
    parts = split_block0(blocks, 1500)
    with ledger.Atlas(tmp_path, pack_bytes=30000) as at:
        lo, hi, recs = parts[0]
        at.append(lo, hi, recs)
        with pytest.raises(ledger.LedgerError):
            at.append(hi + 2, hi + 100, parts[1][2][:1])           # gap: refused
    with ledger.Atlas(tmp_path, pack_bytes=30000) as at:           # reopen: resume point persisted
        assert at.next_lo == parts[1][0] and at.next_block == 1
        lo, hi, recs = parts[1]
        at.append(lo, hi, recs)
        packs = sorted(p.name for p in (tmp_path / "scan").glob("*.pack"))
        assert packs == ["facts-00000.pack", "facts-00001.pack"]     # rolled over at 30000 bytes
        res = at.verify()
        assert res["primes"] == 4096 and res["next_lo"] == 38891
        rows = []
        for bid in (0, 1):
            rows += codec.decode_scan_frame(at.frame("scan", bid))[0]
        assert [r.p for r in rows] == [r.p for r in blocks["00000"][0]]


def test_torn_pack_tail_is_cut_on_reopen(tmp_path, blocks):
    parts = split_block0(blocks, 2000)
    with ledger.Atlas(tmp_path) as at:
        at.append(*parts[0])
    # a run that died after writing its frames but before committing
    for f in ("scan/facts-00000.pack", "quadruplets/A4-00000.pack"):
        with (tmp_path / f).open("ab") as s:
            s.write(b"\xa5" * 777)
    with ledger.Atlas(tmp_path) as at:
        assert sorted(at.recovered) == [("quadruplets/A4-00000.pack", 777), ("scan/facts-00000.pack", 777)]
        at.verify()
        at.append(*parts[1])
        assert at.verify()["primes"] == 4096


def test_commit_is_atomic_across_both_ledgers(tmp_path, blocks):
    parts = split_block0(blocks, 1000)
    with ledger.Atlas(tmp_path) as at:
        at.append(*parts[0])
        before = (at.meta(), at.meta("a4"))
        # plant a fault in the A4 ledger: its block insert aborts after the
        # scan ledger's insert of the same block has run
        at.db.execute("CREATE TRIGGER a4.planted BEFORE INSERT ON blocks BEGIN SELECT RAISE(ABORT, 'planted'); END")
        with pytest.raises(sqlite3.IntegrityError):
            at.append(*parts[1])
        assert at.db.execute("SELECT count(*) FROM main.blocks").fetchone()[0] == 1
        assert (at.meta(), at.meta("a4")) == before
        at.db.execute("DROP TRIGGER a4.planted")
    with ledger.Atlas(tmp_path) as at:                              # the orphan frames are cut
        assert len(at.recovered) == 2
        at.verify()
        at.append(*parts[1])
        at.verify()


def test_verify_detects_a_flipped_byte(tmp_path, blocks):
    recs, meta = blocks["00000"]
    with ledger.Atlas(tmp_path) as at:
        at.append(meta["lo"], meta["hi"], recs)
    pack = tmp_path / "scan" / "facts-00000.pack"
    data = bytearray(pack.read_bytes())
    data[len(data) // 2] ^= 0x10
    pack.write_bytes(bytes(data))
    with ledger.Atlas(tmp_path) as at:
        with pytest.raises(Exception):
            at.verify()


def test_a4_point_audit_accepts_golden_rejects_planted(blocks):
    rng = random.Random(7)
    recs = blocks["49900"][0][:400] + blocks["00000"][0][-200:]
    assert all(ledger.a4_point_audit(r.p, r.a4, rng) for r in recs)
    assert not any(ledger.a4_point_audit(r.p, r.a4 + 1, rng) for r in recs if r.p > 1000)


def test_cli_verify_and_status(tmp_path, blocks):
    recs, meta = blocks["00000"]
    with ledger.Atlas(tmp_path) as at:
        at.append(meta["lo"], meta["hi"], recs)
    for cmd in ("verify", "status"):
        out = subprocess.run([sys.executable, "-m", "rabung_atlas32_b200.ledger", cmd, "--root", str(tmp_path)],
                             cwd=ROOT, capture_output=True, text=True, check=True).stdout
        d = json.loads(out)
        assert str(d["next_lo"]) == "38891"


class FakeCensus:
    """Stands in for the GPU census on CPU: records of the reference's block 0
    (decoded from the golden frames) and a host sieve.  `planted` changes the
    dense re-check of one prime, as a faulty census would."""

    def __init__(self, blocks, planted=None):
        self.recs = {r.p: r for r in blocks["00000"][0]}
        self.planted = planted
        self.calls = []
        self.verify_flags = []

    def sieve(self, requests):
        from rabung_atlas32_b200 import sieve
        return [sieve.primes_from(lo, n) for lo, n in requests]

    def profiles(self, primes, mode="auto", a4=True, verify=False):
        import copy
        self.calls.append(mode)
        self.verify_flags.append((mode, verify))
        out = [copy.deepcopy(self.recs[p]) for p in primes]
        for r in out:
            if mode == "dense" and r.p == self.planted:
                r.profiles[0].M += 1
            if not a4:
                r.a4 = 0
        return out


def test_supervisor_cuts_blocks_resumes_and_audits(tmp_path, blocks):
    fake = FakeCensus(blocks)
    with ledger.Atlas(tmp_path) as at:
        first = ledger.run(at, fake, 1, 38891, block_primes=1000, audit_every=2, max_blocks=2, log=lambda s: None)
        assert [d["primes"] for d in first] == [1000, 1000]
    with ledger.Atlas(tmp_path) as at:                                # resumes at next_lo
        rest = ledger.run(at, fake, 1, 38891, block_primes=1000, audit_every=2, log=lambda s: None)
        assert rest[0]["lo"] == first[-1]["hi"] and [d["primes"] for d in rest] == [1000, 1000, 96]
        assert rest[-1]["hi"] == 38891
        res = at.verify()
        assert res["primes"] == 4096 and res["GPU_audits"] == res["A4_certificate_audits"] == 3
        got = [r.p for b in range(5) for r in codec.decode_scan_frame(at.frame("scan", b))[0]]
        assert got == [r.p for r in blocks["00000"][0]]
    # every committed block's records were certified on the device
    assert all(v for m, v in fake.verify_flags if m != "dense")
    # a whole-block run reproduces the sample frames
    with ledger.Atlas(tmp_path / "one") as at:
        ledger.run(at, FakeCensus(blocks), 1, 38891, audit_every=1, log=lambda s: None)
        assert at.frame("scan", 0) == (GOLDEN / "scan-00000.vdw").read_bytes()
        assert at.frame("quadruplets", 0) == (GOLDEN / "quadruplets-00000.a4").read_bytes()


def test_supervisor_stops_before_committing_a_failed_audit(tmp_path, blocks):
    # every prime of the first block is in the audit sample when it holds 8 primes
    recs = blocks["00000"][0]
    fake = FakeCensus(blocks, planted=recs[3].p)
    with ledger.Atlas(tmp_path) as at:
        with pytest.raises(ledger.LedgerError, match="audit failed"):
            ledger.run(at, fake, 1, 38891, block_primes=8, audit_every=1, audit_primes=8, log=lambda s: None)
        assert at.next_lo == 1 and at.next_block == 0
    with ledger.Atlas(tmp_path) as at:
        assert at.recovered == [] and at.verify()["blocks"] == 0


def test_verify_catches_a_block_missing_a_prime(tmp_path, blocks):
    """A sieve that silently drops a prime yields a block whose count is short
    of the exact prime count of its interval; verify() refuses the atlas."""
    class DroppingCensus(FakeCensus):
        def sieve(self, requests):
            out = super().sieve(requests)
            return [[p for p in ps if p != 1009] for ps in out]

    with ledger.Atlas(tmp_path) as at:
        ledger.run(at, DroppingCensus(blocks), 1, 38891, block_primes=1000, audit_every=0, max_blocks=1,
                   log=lambda s: None)
        with pytest.raises(ledger.LedgerError, match="primes, \\[lo, hi\\) holds"):
            at.verify()
