"""Line-protocol workers: drop-in processes for the reference's census worker
and A4 worker, computing on the B200 through the C ABI.

Census worker (src/census/worker32.cu:10-45, docs/REPRODUCTION.md:29-39):
  stdout  {"type":"ready","domain_bits":32}
  stdin   "<batch_id> p1 ... pk"   batch ids strictly sequential from 0,
                                   1 <= k <= --max-batch, primes checked
          "QUIT"                   -> {"type":"bye"}
  stdout  per prime {"type":"measurement","status":"PASS","p","mask","total_ms",
          "profiles":[{"r","max","prefix","K","witness"}, ...]}, then
          {"type":"batch_done","id","count","wall_ms"}
  failure stderr "VDW_CAMPAIGN_FAILURE: <msg>", exit status 2; a batch is
          never partially accepted.

A4 worker (--a4; src/census/moment_worker.cpp:19-52):
  stdout  {"type":"ready","algorithm":"qualified_mestre_A4","maximum_batch":4096}
  stdin   "batch_id audit_index n p1 ... pn" (strictly increasing primes < 2^32)
  stdout  binary "A4BATCH1", id u64, n u32, certificate length u32, nanoseconds
          u64, sum u64, max attempt u32, small count u32, first u64, last u64,
          u32[n] values, certificate JSON (the audited prime's point count).

    python -m rabung_atlas32_b200.worker [--a4] [--min-p 1000] [--max-batch 128]
"""
from __future__ import annotations

import argparse
import json
import struct
import sys
import time

from . import codec
from .census import Census, CensusError


def fail(msg: str, tag: str = "VDW_CAMPAIGN_FAILURE") -> None:
    sys.stderr.write(f"{tag}: {msg}\n")
    sys.stderr.flush()
    sys.exit(2)


def census_worker(eng: Census, min_p: int, max_batch: int, mode: str) -> None:
    out = sys.stdout
    out.write(json.dumps({"type": "ready", "domain_bits": 32}, separators=(",", ":")) + "\n")
    out.flush()
    expected = 0
    for line in sys.stdin:
        line = line.strip()
        if line == "QUIT":
            out.write('{"type":"bye"}\n')
            out.flush()
            return
        toks = line.split()
        if not toks or not toks[0].isdigit() or int(toks[0]) != expected:
            fail("batch sequence")
        primes = []
        for t in toks[1:]:
            if not t.isdigit():
                fail("prime token")
            v = int(t)
            if not min_p <= v < 2 ** 32:
                fail("worker prime range")
            primes.append(v)
        if not 1 <= len(primes) <= max_batch:
            fail("worker batch size")
        t0 = time.perf_counter()
        try:
            recs = eng.profiles(primes, mode=mode, a4=False, verify=True)
        except CensusError as e:
            fail(str(e))
        total = 1000 * (time.perf_counter() - t0)
        per = total / len(primes)
        for rec in recs:
            out.write(json.dumps({"type": "measurement", "status": "PASS", "p": rec.p, "mask": rec.mask,
                                  "total_ms": round(per, 6),
                                  "profiles": [{"r": v.r, "max": v.M, "prefix": v.L, "K": v.K,
                                                "witness": v.witness} for v in rec.profiles]},
                                 separators=(",", ":")) + "\n")
        out.write(json.dumps({"type": "batch_done", "id": expected, "count": len(primes),
                              "wall_ms": round(1000 * (time.perf_counter() - t0), 6)},
                             separators=(",", ":")) + "\n")
        out.flush()
        expected += 1


def a4_worker(eng: Census) -> None:
    out = sys.stdout.buffer
    sys.stdout.write(json.dumps({"type": "ready", "algorithm": "qualified_mestre_A4", "maximum_batch": 4096},
                                separators=(",", ":")) + "\n")
    sys.stdout.flush()
    for line in sys.stdin:
        line = line.strip()
        if line == "QUIT":
            return
        toks = line.split()
        try:
            bid, audit, n = int(toks[0]), int(toks[1]), int(toks[2])
        except (ValueError, IndexError):
            fail("batch header", "A4")
        if n > 4096 or audit < -1 or audit >= n or len(toks) != 3 + n:
            fail("batch header", "A4")
        primes = [int(t) for t in toks[3:]]
        if any(b <= a for a, b in zip(primes, primes[1:])) or (primes and primes[-1] >= 2 ** 32):
            fail("ordered prime batch", "A4")
        t0 = time.perf_counter_ns()
        try:
            vals = eng.a4(primes) if primes else []
        except CensusError as e:
            fail(str(e), "A4")
        ns = time.perf_counter_ns() - t0
        cert = b""
        if audit >= 0:
            p, a = primes[audit], vals[audit]
            if p < 1000:
                cert = json.dumps({"status": "PASS", "p": p, "r": 2, "quadruples": a,
                                   "certificate": "small_dense"}, separators=(",", ":")).encode()
            else:
                chi = lambda x: 1 if pow(x % p, (p - 1) // 2, p) == 1 else -1
                b = 4 * chi(2) + 2 * chi(6) + 2 * chi(3) + 2 * chi(p - 1) + 2 * chi(p - 2)
                cert = json.dumps({"status": "PASS", "p": p, "r": 2, "quadruples": a,
                                   "elliptic_points": 8 * a + 12 + b,
                                   "certificate": "unique_lcm_multiple_in_Hasse"}, separators=(",", ":")).encode()
        small = sum(1 for p in primes if p < 1000)
        out.write(b"A4BATCH1")
        out.write(struct.pack("<QIIQQII", bid, n, len(cert), ns, sum(vals), 0, small))
        out.write(struct.pack("<QQ", primes[0] if primes else 0, primes[-1] if primes else 0))
        out.write(struct.pack("<" + "I" * n, *vals))
        out.write(cert)
        out.flush()


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--a4", action="store_true", help="speak the A4 worker protocol")
    ap.add_argument("--min-p", type=int, default=1000, help="least accepted prime (reference GPU worker: 1000)")
    ap.add_argument("--max-batch", type=int, default=128, help="primes per batch line (reference: 128)")
    ap.add_argument("--mode", default="auto", choices=["auto", "dense", "sparse"])
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    try:
        eng = Census(device=a.device)
    except Exception as e:  # no device: refuse like the reference (exit 2)
        fail(str(e))
    if a.a4:
        a4_worker(eng)
    else:
        census_worker(eng, a.min_p, a.max_batch, a.mode)


if __name__ == "__main__":
    main()
