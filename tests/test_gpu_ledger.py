"""Census supervisor on the GPU: device sieve -> census -> frames -> packs and
ledgers, with audits.  Block 0 and the last block of the domain, cut the way
the reference cuts them, must come out byte for byte as the reference's
sample frames; a multi-block run near 2^24 must verify and resume."""
import pytest

from conftest import GOLDEN
from rabung_atlas32_b200 import ledger

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from rabung_atlas32_b200.census import Census
    with Census() as c:
        yield c


def test_block0_supervised_equals_sample(tmp_path, eng):
    with ledger.Atlas(tmp_path) as at:
        done = ledger.run(at, eng, 1, 38891, audit_every=1, audit_primes=8, log=lambda s: None)
        assert [(d["lo"], d["hi"], d["primes"]) for d in done] == [(1, 38891, 4096)]
        assert at.frame("scan", 0) == (GOLDEN / "scan-00000.vdw").read_bytes()
        assert at.frame("quadruplets", 0) == (GOLDEN / "quadruplets-00000.a4").read_bytes()
        kinds = sorted((k, s) for k, s in at.db.execute(
            "SELECT kind, status FROM main.audits UNION ALL SELECT kind, status FROM a4.audits"))
        assert kinds == [("a4_point_check", "PASS"), ("dense_recheck", "PASS")]
        at.verify()


def test_last_block_supervised_equals_sample(tmp_path, eng):
    with ledger.Atlas(tmp_path, contiguous=False) as at:
        done = ledger.run(at, eng, 4294915433, 1 << 32, audit_every=0, log=lambda s: None)
        assert [(d["lo"], d["hi"], d["primes"]) for d in done] == [(4294915433, 1 << 32, 2313)]
        assert at.frame("scan", 0) == (GOLDEN / "scan-49900.vdw").read_bytes()
        assert at.frame("quadruplets", 0) == (GOLDEN / "quadruplets-49900.a4").read_bytes()
        at.verify()


def test_contiguous_start_from_one(tmp_path, eng):
    with ledger.Atlas(tmp_path) as at:
        ledger.run(at, eng, 1, 4000, audit_every=0, log=lambda s: None)
        assert at.next_lo == 4000 and at.verify()["primes"] == 550
        with pytest.raises(ledger.LedgerError):
            ledger.run(at, eng, 5000, 6000, log=lambda s: None)           # a gap is refused


def test_multiblock_run_resumes(tmp_path, eng):
    from rabung_atlas32_b200 import sieve
    lo, hi = 1 << 24, (1 << 24) + 60000
    with ledger.Atlas(tmp_path, pack_bytes=20000, contiguous=False) as at:
        first = ledger.run(at, eng, lo, hi, block_primes=1024, audit_every=2, max_blocks=3, log=lambda s: None)
        assert len(first) == 3 and first[0]["lo"] == lo
    with ledger.Atlas(tmp_path, pack_bytes=20000, contiguous=False) as at:  # resume where it stopped
        rest = ledger.run(at, eng, lo, hi, block_primes=1024, audit_every=2, log=lambda s: None)
        assert rest[0]["lo"] == first[-1]["hi"] and rest[-1]["hi"] == hi
        res = at.verify()
        assert res["primes"] == len(sieve.primes_in(lo, hi)) and res["next_lo"] == hi
        assert res["GPU_audits"] == res["A4_certificate_audits"] == 2
