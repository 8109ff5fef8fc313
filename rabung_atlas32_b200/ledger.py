"""Atlas writer: scan and A4 packs, SQLite ledgers, hash chains, and the
census supervisor that fills them block by block.

Layout under an atlas root -- the reference's published layout, as its readers
use it (docs/DATA_FORMAT.md:7-77; scripts/atlas_io.py:34-50;
scripts/verify_atlas.py:48-116):

  scan/facts-NNNNN.pack        VDWSM1 frames, concatenated
  scan/ledger.sqlite           blocks(id, lo, hi, n, pack, offset, size,
                               prime_hash, science_hash, summary), meta,
                               audits, best, milestones
  quadruplets/A4-NNNNN.pack    VDWA4V1 frames, concatenated
  quadruplets/ledger.sqlite    blocks(id, lo, hi, n, pack, offset, size,
                               prime_hash, profile_hash, values_hash, summary),
                               meta, audits

Hashes are stored as hex text; `summary` is zlib-compressed JSON ({"primes",
"hist_max", "hist_prefix", "hist_K"} per r for the scan, {"primes", "sum_A4"}
for A4); meta holds next_lo, next_block, prime_count, chain (and aggregate /
sum_A4).  Both chains start at 32 zero bytes and advance per block in id order:
scan = SHA256(prev || prime_hash || profile_hash || u64 lo || u64 hi),
A4 = SHA256(prev || prime_hash || profile_hash || values_hash || u64 lo || u64 hi).

Crash consistency: a block's two frames are appended to their packs and
fsync'd first, then both ledgers are updated in ONE SQLite transaction (the A4
ledger is ATTACHed to the scan connection, rollback journal, so the commit is
atomic across the two files).  On open, every pack is cut back to the end of
its last indexed frame, which drops a frame written by a run that died before
its commit.  A supervisor restarted on the same root resumes at meta next_lo.

    python -m rabung_atlas32_b200.ledger run --root DIR --lo 1 --hi 1000000
    python -m rabung_atlas32_b200.ledger verify --root DIR
    python -m rabung_atlas32_b200.ledger status --root DIR
"""
from __future__ import annotations

import argparse
import collections
import hashlib
import json
import os
import random
import sqlite3
import struct
import time
import zlib
from pathlib import Path

from . import codec
from .census import prime_count

PACK_BYTES = 64 << 20          # a new pack file starts past this size
BLOCK_PRIMES = 4096            # primes per block (the frame maximum)
TOP = 1 << 32                  # end of the 32-bit domain

SCAN_SCHEMA = """
CREATE TABLE IF NOT EXISTS main.blocks (
  id INTEGER PRIMARY KEY, lo INTEGER NOT NULL, hi INTEGER NOT NULL, n INTEGER NOT NULL,
  pack TEXT NOT NULL, offset INTEGER NOT NULL, size INTEGER NOT NULL,
  prime_hash TEXT NOT NULL, science_hash TEXT NOT NULL, summary BLOB NOT NULL);
CREATE TABLE IF NOT EXISTS main.meta (key TEXT PRIMARY KEY, value TEXT NOT NULL);
CREATE TABLE IF NOT EXISTS main.audits (
  id INTEGER PRIMARY KEY, block INTEGER NOT NULL, kind TEXT NOT NULL, items INTEGER NOT NULL,
  status TEXT NOT NULL, detail TEXT NOT NULL);
CREATE TABLE IF NOT EXISTS main.best (
  r INTEGER PRIMARY KEY, M INTEGER NOT NULL, p INTEGER NOT NULL, L INTEGER NOT NULL,
  K INTEGER NOT NULL, witness INTEGER NOT NULL, block INTEGER NOT NULL);
CREATE TABLE IF NOT EXISTS main.milestones (
  r INTEGER NOT NULL, M INTEGER NOT NULL, p INTEGER NOT NULL, L INTEGER NOT NULL,
  K INTEGER NOT NULL, witness INTEGER NOT NULL, block INTEGER NOT NULL, PRIMARY KEY (r, M));
"""
A4_SCHEMA = """
CREATE TABLE IF NOT EXISTS a4.blocks (
  id INTEGER PRIMARY KEY, lo INTEGER NOT NULL, hi INTEGER NOT NULL, n INTEGER NOT NULL,
  pack TEXT NOT NULL, offset INTEGER NOT NULL, size INTEGER NOT NULL,
  prime_hash TEXT NOT NULL, profile_hash TEXT NOT NULL, values_hash TEXT NOT NULL, summary BLOB NOT NULL);
CREATE TABLE IF NOT EXISTS a4.meta (key TEXT PRIMARY KEY, value TEXT NOT NULL);
CREATE TABLE IF NOT EXISTS a4.audits (
  id INTEGER PRIMARY KEY, block INTEGER NOT NULL, kind TEXT NOT NULL, items INTEGER NOT NULL,
  status TEXT NOT NULL, detail TEXT NOT NULL);
"""
ZERO = "00" * 32


class LedgerError(RuntimeError):
    pass


def block_summary(records) -> dict:
    """Per-order histograms of M, L and K for one block (string keys, as JSON)."""
    hists = {name: collections.defaultdict(collections.Counter) for name in ("hist_max", "hist_prefix", "hist_K")}
    for rec in records:
        for pr in rec.profiles:
            k = codec.minimum_k(rec.p, pr.r, pr.M, pr.L)
            hists["hist_max"][str(pr.r)][str(pr.M)] += 1
            hists["hist_prefix"][str(pr.r)][str(pr.L)] += 1
            hists["hist_K"][str(pr.r)][str(k)] += 1
    out = {"primes": len(records)}
    for name, orders in hists.items():
        out[name] = {r: dict(sorted(c.items())) for r, c in sorted(orders.items())}
    return out


def _pack_json(obj) -> bytes:
    return zlib.compress(json.dumps(obj, sort_keys=True, separators=(",", ":")).encode(), 6)


def _unpack_json(blob: bytes):
    return json.loads(zlib.decompress(blob))


class Atlas:
    """An atlas root opened for appending (and reading)."""

    def __init__(self, root, pack_bytes: int = PACK_BYTES, contiguous: bool = True):
        self.root = Path(root)
        self.pack_bytes = int(pack_bytes)
        self.contiguous = contiguous
        (self.root / "scan").mkdir(parents=True, exist_ok=True)
        (self.root / "quadruplets").mkdir(parents=True, exist_ok=True)
        self.db = sqlite3.connect(str(self.root / "scan" / "ledger.sqlite"), isolation_level=None)
        self.db.execute("PRAGMA journal_mode=DELETE")
        self.db.execute("ATTACH DATABASE ? AS a4", (str(self.root / "quadruplets" / "ledger.sqlite"),))
        self.db.execute("PRAGMA a4.journal_mode=DELETE")
        self.db.execute("BEGIN IMMEDIATE")
        try:
            for stmt in (SCAN_SCHEMA + A4_SCHEMA).split(";"):
                if stmt.strip():
                    self.db.execute(stmt)
            init = {"next_lo": "1", "next_block": "0", "prime_count": "0", "chain": ZERO}
            for k, v in {**init, "aggregate": json.dumps({}), "profile_count": "0"}.items():
                self.db.execute("INSERT OR IGNORE INTO main.meta(key, value) VALUES (?, ?)", (k, v))
            for k, v in {**init, "sum_A4": "0"}.items():
                self.db.execute("INSERT OR IGNORE INTO a4.meta(key, value) VALUES (?, ?)", (k, v))
            self.db.execute("COMMIT")
        except BaseException:
            self.db.execute("ROLLBACK")
            raise
        self.recovered = self._recover()

    # ---- state -------------------------------------------------------------
    def meta(self, group: str = "main") -> dict:
        return dict(self.db.execute(f"SELECT key, value FROM {group}.meta"))

    @property
    def next_lo(self) -> int:
        return int(self.meta()["next_lo"])

    @property
    def next_block(self) -> int:
        return int(self.meta()["next_block"])

    def close(self):
        if self.db is not None:
            self.db.close()
            self.db = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- packs -------------------------------------------------------------
    def _extents(self, group: str) -> dict:
        return {pack: end for pack, end in self.db.execute(
            f"SELECT pack, MAX(offset + size) FROM {group}.blocks GROUP BY pack")}

    def _recover(self) -> list:
        """Cut every pack back to its last indexed frame; returns what was cut."""
        cut = []
        for group, sub, prefix in (("main", "scan", "facts-"), ("a4", "quadruplets", "A4-")):
            ends = self._extents(group)
            for f in sorted((self.root / sub).glob(prefix + "*.pack")):
                end = ends.get(f.name, 0)
                size = f.stat().st_size
                if size > end:
                    with f.open("r+b") as s:
                        s.truncate(end)
                        s.flush()
                        os.fsync(s.fileno())
                    cut.append((f"{sub}/{f.name}", size - end))
        return cut

    def _target_pack(self, group: str, sub: str, prefix: str, nbytes: int) -> tuple:
        row = self.db.execute(f"SELECT pack, offset + size FROM {group}.blocks ORDER BY id DESC LIMIT 1").fetchone()
        if row is None:
            return f"{prefix}00000.pack", 0
        pack, end = row
        if end + nbytes > self.pack_bytes and end > 0:
            idx = int(pack[len(prefix):-len(".pack")]) + 1
            return f"{prefix}{idx:05d}.pack", 0
        return pack, end

    def _write(self, sub: str, pack: str, offset: int, data: bytes) -> None:
        path = self.root / sub / pack
        with path.open("ab") as s:
            if s.tell() != offset:
                raise LedgerError(f"{sub}/{pack}: expected to append at {offset}, file ends at {s.tell()}")
            s.write(data)
            s.flush()
            os.fsync(s.fileno())

    def frame(self, group: str, block: int) -> bytes:
        """Frame bytes of `block` in 'scan' or 'quadruplets', read through the index."""
        schema, sub = ("main", "scan") if group == "scan" else ("a4", "quadruplets")
        row = self.db.execute(f"SELECT pack, offset, size FROM {schema}.blocks WHERE id=?", (block,)).fetchone()
        if row is None:
            raise LedgerError(f"unknown block {block}")
        pack, offset, size = row
        with (self.root / sub / pack).open("rb") as s:
            s.seek(offset)
            data = s.read(size)
        if len(data) != size:
            raise LedgerError("truncated pack")
        return data

    # ---- append ------------------------------------------------------------
    def append(self, lo: int, hi: int, records, block: int | None = None, audits=()) -> dict:
        """Append one block: both frames, both ledger rows, chains, histograms,
        best/milestones and audit rows.  `records` are codec.Record with A4 set."""
        m, am = self.meta(), self.meta("a4")
        next_lo, next_block = int(m["next_lo"]), int(m["next_block"])
        bid = next_block if block is None else int(block)
        if bid < next_block:
            raise LedgerError(f"block id {bid} below the next free id {next_block}")
        if self.contiguous and (lo != next_lo or bid != next_block):
            raise LedgerError(f"block [{lo}, {hi}) id {bid} does not continue at [{next_lo}, ...) id {next_block}")
        if not (next_lo <= lo < hi <= TOP) or not 0 < len(records) <= BLOCK_PRIMES:
            raise LedgerError(f"block [{lo}, {hi}) with {len(records)} primes out of range")
        if any(not lo <= rec.p < hi for rec in records):
            raise LedgerError("prime outside its block")
        scan = codec.encode_scan_frame(lo, hi, records)
        a4f = codec.encode_a4_frame(lo, hi, records)
        ph, sh = codec.prime_hash(records), codec.science_hash(records)
        vh = hashlib.sha256(codec.a4_values_raw(records)).digest()
        chain_s, chain_a = codec.chain_step(bytes.fromhex(m["chain"]), bytes.fromhex(am["chain"]), lo, hi, records)
        summ = block_summary(records)
        sum_a4 = sum(rec.a4 for rec in records)
        agg = json.loads(m["aggregate"])
        for name in ("hist_max", "hist_prefix", "hist_K"):
            dst = agg.setdefault(name, {})
            for r, vals in summ[name].items():
                row = dst.setdefault(r, {})
                for v, c in vals.items():
                    row[v] = row.get(v, 0) + c
        nprof = sum(len(rec.profiles) for rec in records)

        spack, soff = self._target_pack("main", "scan", "facts-", len(scan))
        apack, aoff = self._target_pack("a4", "quadruplets", "A4-", len(a4f))
        self._write("scan", spack, soff, scan)
        self._write("quadruplets", apack, aoff, a4f)

        db = self.db
        db.execute("BEGIN IMMEDIATE")
        try:
            db.execute("INSERT INTO main.blocks VALUES (?,?,?,?,?,?,?,?,?,?)",
                       (bid, lo, hi, len(records), spack, soff, len(scan), ph.hex(), sh.hex(), _pack_json(summ)))
            db.execute("INSERT INTO a4.blocks VALUES (?,?,?,?,?,?,?,?,?,?,?)",
                       (bid, lo, hi, len(records), apack, aoff, len(a4f), ph.hex(), sh.hex(), vh.hex(),
                        _pack_json({"primes": len(records), "sum_A4": sum_a4})))
            best = {r: M for r, M in db.execute("SELECT r, M FROM main.best")}
            for rec in records:
                for pr in rec.profiles:
                    if pr.M > best.get(pr.r, 0):
                        best[pr.r] = pr.M
                        row = (pr.r, pr.M, rec.p, pr.L, codec.minimum_k(rec.p, pr.r, pr.M, pr.L), pr.witness, bid)
                        db.execute("INSERT OR REPLACE INTO main.best VALUES (?,?,?,?,?,?,?)", row)
                        db.execute("INSERT OR IGNORE INTO main.milestones VALUES (?,?,?,?,?,?,?)", row)
            for a in audits:
                schema = "a4" if a["kind"].startswith("a4") else "main"
                db.execute(f"INSERT INTO {schema}.audits(block, kind, items, status, detail) VALUES (?,?,?,?,?)",
                           (bid, a["kind"], a["items"], a["status"], json.dumps(a.get("detail", {}), sort_keys=True)))
            upd = {"next_lo": str(hi), "next_block": str(bid + 1),
                   "prime_count": str(int(m["prime_count"]) + len(records)), "chain": chain_s.hex(),
                   "aggregate": json.dumps(agg, sort_keys=True), "profile_count": str(int(m["profile_count"]) + nprof)}
            for k, v in upd.items():
                db.execute("UPDATE main.meta SET value=? WHERE key=?", (v, k))
            upda = {"next_lo": str(hi), "next_block": str(bid + 1),
                    "prime_count": str(int(am["prime_count"]) + len(records)), "chain": chain_a.hex(),
                    "sum_A4": str(int(am["sum_A4"]) + sum_a4)}
            for k, v in upda.items():
                db.execute("UPDATE a4.meta SET value=? WHERE key=?", (v, k))
            db.execute("COMMIT")
        except BaseException:
            db.execute("ROLLBACK")
            raise
        return {"block": bid, "lo": lo, "hi": hi, "primes": len(records), "profiles": nprof,
                "prime_hash": ph.hex(), "science_hash": sh.hex(), "values_hash": vh.hex(),
                "scan_chain": chain_s.hex(), "a4_chain": chain_a.hex()}

    # ---- verify ------------------------------------------------------------
    def verify(self, decode: bool = True) -> dict:
        """Re-derive every commitment from the stored bytes: frame extents are
        contiguous per pack and end at the pack's size, frames decode under
        the strict codec and hash to their index rows, chains, histograms,
        sums and counts equal meta.  Raises LedgerError on the first fault."""
        db = self.db

        def check(cond, msg):
            if not cond:
                raise LedgerError(msg)

        for schema in ("main", "a4"):
            check(db.execute(f"PRAGMA {schema}.integrity_check").fetchone()[0] == "ok", f"{schema} integrity")
        m, am = self.meta(), self.meta("a4")
        srows = db.execute("SELECT id,lo,hi,n,pack,offset,size,prime_hash,science_hash,summary FROM main.blocks "
                           "ORDER BY id").fetchall()
        arows = db.execute("SELECT id,lo,hi,n,pack,offset,size,prime_hash,profile_hash,values_hash,summary "
                           "FROM a4.blocks ORDER BY id").fetchall()
        check(len(srows) == len(arows), "ledgers hold different block counts")
        sc, ac = bytes(32), bytes(32)
        lo_expect, prev_id = 1, -1
        offsets = {}
        primes = profiles = total_a4 = 0
        agg = {name: collections.defaultdict(collections.Counter) for name in ("hist_max", "hist_prefix", "hist_K")}
        for s, a in zip(srows, arows):
            check(s[:4] == a[:4] and s[7] == a[7] and s[8] == a[8], f"block {s[0]}: ledgers disagree")
            check(s[0] > prev_id and s[1] < s[2] and 0 < s[3] <= BLOCK_PRIMES, f"block {s[0]}: bad identity")
            if self.contiguous:
                check(s[0] == prev_id + 1 and s[1] == lo_expect, f"block {s[0]}: not contiguous")
            check(s[1] >= lo_expect, f"block {s[0]}: overlaps its predecessor")
            # the block holds every prime of its interval: its count equals the
            # exact host count pi(hi - 1) - pi(lo - 1)
            check(prime_count(s[1], s[2]) == s[3], f"block {s[0]}: {s[3]} primes, [lo, hi) holds "
                                                  f"{prime_count(s[1], s[2])}")
            for sub, row in (("scan", s), ("quadruplets", a)):
                key = f"{sub}/{row[4]}"
                check(row[5] == offsets.get(key, 0) and row[6] > 0, f"block {s[0]}: {key} extent not contiguous")
                offsets[key] = row[5] + row[6]
            bound = struct.pack("<QQ", s[1], s[2])
            sc = hashlib.sha256(sc + bytes.fromhex(s[7]) + bytes.fromhex(s[8]) + bound).digest()
            ac = hashlib.sha256(ac + bytes.fromhex(a[7]) + bytes.fromhex(a[8]) + bytes.fromhex(a[9]) + bound).digest()
            ss, aa = _unpack_json(s[9]), _unpack_json(a[10])
            check(ss["primes"] == s[3] == aa["primes"], f"block {s[0]}: summary counts")
            for name in agg:
                for r, vals in ss[name].items():
                    agg[name][r].update({k: int(v) for k, v in vals.items()})
            if decode:
                recs, sm = codec.decode_scan_frame(self.frame("scan", s[0]))
                vals, amd = codec.decode_a4_frame(self.frame("quadruplets", s[0]))
                check((sm["lo"], sm["hi"], sm["count"]) == (s[1], s[2], s[3]), f"block {s[0]}: scan frame identity")
                check((amd["lo"], amd["hi"], amd["count"]) == (s[1], s[2], s[3]), f"block {s[0]}: A4 frame identity")
                check(codec.prime_hash(recs).hex() == s[7] == amd["prime_hash"], f"block {s[0]}: prime hash")
                check(codec.science_hash(recs).hex() == s[8] == amd["profile_science_hash"], f"block {s[0]}: science hash")
                check(amd["values_sha256"] == a[9], f"block {s[0]}: values hash")
                check(sum(vals) == aa["sum_A4"], f"block {s[0]}: A4 sum")
                check(block_summary(recs) == ss, f"block {s[0]}: histograms")
                for rec, v in zip(recs, vals):
                    check(v == 0 if rec.p == 2 else 0 <= v <= (rec.p - 3) // 2, f"p={rec.p}: A4 bound")
            primes += s[3]
            profiles += sum(sum(v.values()) for v in ss["hist_max"].values())
            total_a4 += aa["sum_A4"]
            lo_expect, prev_id = s[2], s[0]
        for sub, prefix in (("scan", "facts-"), ("quadruplets", "A4-")):
            for f in (self.root / sub).glob(prefix + "*.pack"):
                check(f.stat().st_size == offsets.get(f"{sub}/{f.name}", 0), f"{sub}/{f.name}: size != last extent")
        check(sc.hex() == m["chain"] and ac.hex() == am["chain"], "chain")
        for meta in (m, am):
            check(int(meta["next_lo"]) == lo_expect and int(meta["next_block"]) == prev_id + 1, "next_lo / next_block")
            check(int(meta["prime_count"]) == primes, "prime_count")
        check(int(am["sum_A4"]) == total_a4, "sum_A4")
        if self.contiguous:
            check(primes == prime_count(1, lo_expect), "prime_count differs from pi(next_lo - 1)")
        check(int(m["profile_count"]) == profiles, "profile_count")
        calc = {name: {r: dict(c) for r, c in orders.items()} for name, orders in agg.items()}
        stored = json.loads(m["aggregate"])
        check(all(calc[name] == stored.get(name, {}) for name in calc), "aggregate histograms")
        return {"blocks": len(srows), "primes": primes, "profiles": profiles, "sum_A4": total_a4,
                "next_lo": lo_expect, "profile_chain": sc.hex(), "A4_chain": ac.hex(),
                "GPU_audits": db.execute("SELECT count(*) FROM main.audits").fetchone()[0],
                "A4_certificate_audits": db.execute("SELECT count(*) FROM a4.audits").fetchone()[0]}


# ---- audits ------------------------------------------------------------------

def _legendre(a: int, p: int) -> int:
    a %= p
    if a == 0:
        return 0
    return 1 if pow(a, (p - 1) // 2, p) == 1 else -1


def _ec_mul(k: int, P, p: int):
    """[k]P on y^2 = x(x-1)(x-9) = x^3 - 10x^2 + 9x over F_p, affine, None = O."""
    def add(A, B):
        if A is None:
            return B
        if B is None:
            return A
        (x1, y1), (x2, y2) = A, B
        if x1 == x2 and (y1 + y2) % p == 0:
            return None
        if A == B:
            lam = (3 * x1 * x1 - 20 * x1 + 9) * pow(2 * y1, -1, p) % p
        else:
            lam = (y2 - y1) * pow(x2 - x1, -1, p) % p
        x3 = (lam * lam + 10 - x1 - x2) % p
        return x3, (lam * (x1 - x3) - y1) % p
    R = None
    while k:
        if k & 1:
            R = add(R, P)
        P = add(P, P)
        k >>= 1
    return R


def a4_point_audit(p: int, a4: int, rng: random.Random, points: int = 2) -> bool:
    """Independent host check of one A4 value: N = 8 A4 + 12 + b with
    b = 4chi(2)+2chi(6)+2chi(3)+2chi(-1)+2chi(-2) must lie in the Hasse
    interval, be divisible by 4 (the rational 2-torsion) and kill random
    points of E: y^2 = x(x-1)(x-9) (theorie/elliptic4_mestre.cpp:42-67)."""
    if p < 1000:
        return True                     # dense count below 1000; nothing to certify
    b = 4 * _legendre(2, p) + 2 * _legendre(6, p) + 2 * _legendre(3, p) + 2 * _legendre(-1, p) + 2 * _legendre(-2, p)
    N = 8 * a4 + 12 + b
    if N % 4 or (N - p - 1) ** 2 > 4 * p:
        return False
    found = 0
    while found < points:
        x = rng.randrange(p)
        rhs = x * (x - 1) * (x - 9) % p
        if rhs == 0 or _legendre(rhs, p) != 1:
            continue
        y = pow(rhs, (p + 1) // 4, p) if p % 4 == 3 else _tonelli(rhs, p)
        if _ec_mul(N, (x, y), p) is not None:
            return False
        found += 1
    return True


def _tonelli(n: int, p: int) -> int:
    q, s = p - 1, 0
    while q % 2 == 0:
        q //= 2
        s += 1
    z = 2
    while _legendre(z, p) != -1:
        z += 1
    m, c, t, r = s, pow(z, q, p), pow(n, q, p), pow(n, (q + 1) // 2, p)
    while t != 1:
        i, t2 = 0, t
        while t2 != 1:
            t2 = t2 * t2 % p
            i += 1
        b = pow(c, 1 << (m - i - 1), p)
        m, c, t, r = i, b * b % p, t * b * b % p, r * b % p
    return r


def audit_block(census, records, bid: int, rng: random.Random, primes: int) -> list:
    """GPU audit: a seeded sample of the block's primes re-run by the dense
    kernel (a different algorithm) must give the same profiles; A4 audit: the
    host point check on the same sample."""
    pick = sorted(rng.sample(range(len(records)), min(primes, len(records))))
    sample = [records[i] for i in pick]
    dense = census.profiles([r.p for r in sample], mode="dense", a4=False)
    same = all([(v.r, v.M, v.L, v.witness) for v in a.profiles] == [(v.r, v.M, v.L, v.witness) for v in b.profiles]
               for a, b in zip(sample, dense))
    a4ok = all(a4_point_audit(r.p, r.a4, rng) for r in sample)
    ps = [r.p for r in sample]
    return [{"kind": "dense_recheck", "items": sum(len(r.profiles) for r in sample),
             "status": "PASS" if same else "FAIL", "detail": {"primes": ps}},
            {"kind": "a4_point_check", "items": len(sample), "status": "PASS" if a4ok else "FAIL",
             "detail": {"primes": ps}}]


# ---- supervisor ----------------------------------------------------------------

def next_block_primes(census, lo: int, hi: int, block_primes: int) -> tuple:
    """(primes, block_hi): the next block from lo -- up to block_primes primes
    of [lo, hi), ending where the following block's first prime starts (or at
    hi), by the device sieve."""
    got = census.sieve([(lo, block_primes + 1)])[0]
    inside = [q for q in got if q < hi]
    if len(inside) > block_primes:
        return inside[:block_primes], inside[block_primes]
    return inside, hi


def run(atlas: Atlas, census, lo: int, hi: int, block_primes: int = BLOCK_PRIMES, mode: str = "auto",
        audit_every: int = 16, audit_primes: int = 4, seed: int = 20261203, max_blocks: int | None = None,
        log=print) -> list:
    """Census [lo, hi) into the atlas, block by block; resumes at the atlas's
    next_lo when it is already past lo.  Any refusal, or an audit that fails,
    stops the run before the block is committed."""
    if atlas.contiguous and lo > atlas.next_lo:
        raise LedgerError(f"atlas continues at {atlas.next_lo}; [{atlas.next_lo}, {lo}) would be a gap")
    cur = max(lo, atlas.next_lo)
    done = []
    while cur < hi and (max_blocks is None or len(done) < max_blocks):
        t0 = time.perf_counter()
        ps, bhi = next_block_primes(census, cur, hi, block_primes)
        if not ps:                       # no prime left in [cur, hi): nothing to record
            break
        recs = census.profiles(ps, mode=mode, a4=True, verify=True)
        bid = atlas.next_block
        audits = []
        if audit_every and bid % audit_every == 0:
            audits = audit_block(census, recs, bid, random.Random(seed * 1000003 + bid), audit_primes)
            bad = [a for a in audits if a["status"] != "PASS"]
            if bad:
                raise LedgerError(f"block {bid} [{cur}, {bhi}): audit failed: {bad}")
        info = atlas.append(cur, bhi, recs, audits=audits)
        info["seconds"] = round(time.perf_counter() - t0, 3)
        log(json.dumps(info))
        done.append(info)
        cur = bhi
    return done


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("run")
    r.add_argument("--root", required=True)
    r.add_argument("--lo", type=int, default=1)
    r.add_argument("--hi", type=int, default=TOP)
    r.add_argument("--block-primes", type=int, default=BLOCK_PRIMES)
    r.add_argument("--mode", default="auto", choices=["auto", "dense", "sparse"])
    r.add_argument("--audit-every", type=int, default=16)
    r.add_argument("--audit-primes", type=int, default=4)
    r.add_argument("--max-blocks", type=int)
    r.add_argument("--device", type=int, default=0)
    v = sub.add_parser("verify")
    v.add_argument("--root", required=True)
    s = sub.add_parser("status")
    s.add_argument("--root", required=True)
    a = ap.parse_args(argv)
    if a.cmd == "run":
        from .census import Census
        with Atlas(a.root) as atlas, Census(device=a.device) as eng:
            if atlas.recovered:
                print(json.dumps({"recovered": atlas.recovered}))
            run(atlas, eng, a.lo, a.hi, a.block_primes, a.mode, a.audit_every, a.audit_primes,
                max_blocks=a.max_blocks)
            print(json.dumps({"status": "done", **atlas.verify(decode=False)}))
    elif a.cmd == "verify":
        with Atlas(a.root) as atlas:
            print(json.dumps({"status": "PASS", **atlas.verify()}, indent=1))
    else:
        with Atlas(a.root) as atlas:
            m = atlas.meta()
            print(json.dumps({k: m[k] for k in ("next_lo", "next_block", "prime_count", "profile_count", "chain")}))


if __name__ == "__main__":
    main()
