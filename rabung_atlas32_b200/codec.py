"""Block record format of the census: VDWSM1 scan frames, VDWA4V1 A4 frames,
the prime / profile / values commitments and the two block chains.

Layouts follow docs/DATA_FORMAT.md:7-77 of the reference and its decoder
scripts/atlas_codec.py:3-60 (header structs, varint rules, mask byte,
record order, hash domains).  The encoder is this project's own: the
reference ships only the decoder.  zlib level 3 reproduces the shipped
sample frames byte for byte.
"""
from __future__ import annotations

import hashlib
import struct
import zlib
from dataclasses import dataclass, field

SCAN_MAGIC = b"VDWSM1\0\0"
SCAN_HEADER = struct.Struct("<8sQQQQII32s")       # atlas_codec.py:4
A4_MAGIC = b"VDWA4V1\0"
A4_HEADER = struct.Struct("<8sQQIIII32s32s32s")   # atlas_codec.py:53
ZLIB_LEVEL = 3
MAX_FRAME = 128 * 1024 ** 2


def expected_mask(p: int) -> int:
    """Bit r-2 set exactly when r | p-1 (atlas_codec.py:6)."""
    return sum(1 << (r - 2) for r in range(2, 10) if (p - 1) % r == 0)


def minimum_k(p: int, r: int, m: int, l: int) -> int:
    """Rabung threshold K (docs/METHODS.md:11-18; atlas_codec.py:8)."""
    return max(m + 1, 2 * l + 2 if ((p - 1) // 2) % r == 0 else l + 2)


def put_uint(out: bytearray, v: int) -> None:
    """Canonical little-endian base-128 varint, at most 64 bits."""
    if v < 0 or v >= 2 ** 64:
        raise ValueError("varint range")
    while True:
        b = v & 127
        v >>= 7
        if v:
            out.append(b | 128)
        else:
            out.append(b)
            return


def get_uint(raw: bytes, i: int) -> tuple[int, int]:
    """Strict varint decoder: rejects truncation, non-canonical and >64-bit
    encodings (atlas_codec.py:10-18)."""
    value = 0
    for n in range(10):
        if i >= len(raw):
            raise ValueError("truncated integer")
        b = raw[i]
        i += 1
        value |= (b & 127) << (7 * n)
        if b < 128:
            if value >= 2 ** 64 or (n and b == 0):
                raise ValueError("noncanonical integer")
            return value, i
    raise ValueError("oversized integer")


@dataclass
class Profile:
    r: int
    M: int
    L: int
    witness: int
    K: int = 0

    def as_dict(self) -> dict:
        return {"r": self.r, "max": self.M, "prefix": self.L, "K": self.K, "witness": self.witness}


@dataclass
class Record:
    p: int
    profiles: list = field(default_factory=list)   # list[Profile], ascending r
    a4: int = 0

    @property
    def mask(self) -> int:
        return expected_mask(self.p)


def scan_payload(lo: int, records: list) -> bytes:
    """Uncompressed scan payload: varint(delta p) (first relative to lo-1),
    mask byte, then varint M, L, witness for each set bit in ascending r."""
    out = bytearray()
    prev = lo - 1
    for rec in records:
        if rec.p <= prev:
            raise ValueError("record ordering")
        put_uint(out, rec.p - prev)
        prev = rec.p
        m = expected_mask(rec.p)
        out.append(m)
        rs = [pr.r for pr in rec.profiles]
        if rs != [r for r in range(2, 10) if m & (1 << (r - 2))]:
            raise ValueError(f"profiles of {rec.p} do not match its mask")
        for pr in rec.profiles:
            if not 1 <= pr.L <= pr.M <= (rec.p - 1) // pr.r:
                raise ValueError("profile bound")
            if not 1 <= pr.witness <= (rec.p - 1) // 2:
                raise ValueError("witness bound")
            put_uint(out, pr.M)
            put_uint(out, pr.L)
            put_uint(out, pr.witness)
    return bytes(out)


def encode_scan_frame(lo: int, hi: int, records: list) -> bytes:
    """VDWSM1 frame (docs/DATA_FORMAT.md:9-33), witness flag 1."""
    for rec in records:
        if not lo <= rec.p < hi:
            raise ValueError("prime outside block interval")
    raw = scan_payload(lo, records)
    comp = zlib.compress(raw, ZLIB_LEVEL)
    head = SCAN_HEADER.pack(SCAN_MAGIC, len(comp), len(raw), lo, hi, len(records), 1,
                            hashlib.sha256(raw).digest())
    return head + comp


def decode_scan_frame(frame: bytes) -> tuple[list, dict]:
    """Strict decoder with the reference's checks (atlas_codec.py:20-44)."""
    if len(frame) < SCAN_HEADER.size:
        raise ValueError("truncated header")
    magic, n, size, lo, hi, count, flags, h = SCAN_HEADER.unpack(frame[:SCAN_HEADER.size])
    if magic != SCAN_MAGIC or flags not in (0, 1) or n != len(frame) - SCAN_HEADER.size:
        raise ValueError("frame header")
    if size > MAX_FRAME or n > MAX_FRAME:
        raise ValueError("oversized frame")
    d = zlib.decompressobj()
    raw = d.decompress(frame[SCAN_HEADER.size:], size + 1)
    if len(raw) != size or not d.eof or d.unused_data or hashlib.sha256(raw).digest() != h:
        raise ValueError("frame hash/length")
    recs, i, p = [], 0, lo - 1
    for _ in range(count):
        delta, i = get_uint(raw, i)
        p += delta
        if delta == 0 or not lo <= p < hi or i >= len(raw):
            raise ValueError("record ordering")
        mask = raw[i]
        i += 1
        if mask != expected_mask(p):
            raise ValueError("decoded mask")
        profs = []
        for r in range(2, 10):
            if mask & (1 << (r - 2)):
                m, i = get_uint(raw, i)
                l, i = get_uint(raw, i)
                if not 1 <= l <= m <= (p - 1) // r:
                    raise ValueError("decoded profile bound")
                w = 0
                if flags:
                    w, i = get_uint(raw, i)
                    if not 1 <= w <= (p - 1) // 2:
                        raise ValueError("decoded witness")
                profs.append(Profile(r, m, l, w, minimum_k(p, r, m, l)))
        recs.append(Record(p, profs))
    if i != len(raw):
        raise ValueError("trailing record bytes")
    return recs, {"lo": lo, "hi": hi, "count": count, "witnesses": bool(flags),
                  "raw_sha256": h.hex(), "raw_bytes": size, "compressed_bytes": n}


def prime_hash(records: list) -> bytes:
    """sha256(b'vdw-primes-u64le' || p as u64 ...) (atlas_io.py:27-31)."""
    h = hashlib.sha256(b"vdw-primes-u64le")
    for rec in records:
        h.update(struct.pack("<Q", rec.p))
    return h.digest()


def science_hash(records: list) -> bytes:
    """Profile commitment: (p, mask) then (M, L, K) per admissible r; the
    witness is excluded (atlas_codec.py:46-51; docs/DATA_FORMAT.md:38-42)."""
    h = hashlib.sha256(b"vdw-p-profile-v1-u64le")
    for rec in records:
        h.update(struct.pack("<QB", rec.p, expected_mask(rec.p)))
        for pr in rec.profiles:
            h.update(struct.pack("<QQQ", pr.M, pr.L, minimum_k(rec.p, pr.r, pr.M, pr.L)))
    return h.digest()


def a4_values_raw(records: list) -> bytes:
    return struct.pack("<" + "I" * len(records), *[rec.a4 for rec in records])


def encode_a4_frame(lo: int, hi: int, records: list) -> bytes:
    """VDWA4V1 frame (docs/DATA_FORMAT.md:44-57)."""
    if len(records) > 4096:
        raise ValueError("A4 frame holds at most 4096 primes")
    raw = a4_values_raw(records)
    comp = zlib.compress(raw, ZLIB_LEVEL)
    head = A4_HEADER.pack(A4_MAGIC, lo, hi, len(records), len(comp), len(raw), 0,
                          prime_hash(records), science_hash(records), hashlib.sha256(raw).digest())
    return head + comp


def decode_a4_frame(frame: bytes) -> tuple[list, dict]:
    """Strict A4 decoder (atlas_codec.py:54-60)."""
    if len(frame) < A4_HEADER.size:
        raise ValueError("A4 short frame")
    magic, lo, hi, n, csize, rsize, flags, ph, sh, digest = A4_HEADER.unpack(frame[:A4_HEADER.size])
    if magic != A4_MAGIC or n > 4096 or rsize != 4 * n or flags or csize != len(frame) - A4_HEADER.size:
        raise ValueError("A4 header")
    d = zlib.decompressobj()
    raw = d.decompress(frame[A4_HEADER.size:], rsize + 1)
    if len(raw) != rsize or not d.eof or d.unused_data or hashlib.sha256(raw).digest() != digest:
        raise ValueError("A4 frame hash")
    return list(struct.unpack("<" + "I" * n, raw)), {
        "lo": lo, "hi": hi, "count": n, "prime_hash": ph.hex(),
        "profile_science_hash": sh.hex(), "values_sha256": digest.hex()}


def chain_step(prev_scan: bytes, prev_a4: bytes, lo: int, hi: int, records: list) -> tuple[bytes, bytes]:
    """Advance the scan and A4 chains by one block (docs/DATA_FORMAT.md:63-70)."""
    ph, sh = prime_hash(records), science_hash(records)
    vh = hashlib.sha256(a4_values_raw(records)).digest()
    tail = struct.pack("<QQ", lo, hi)
    scan = hashlib.sha256(prev_scan + ph + sh + tail).digest()
    a4 = hashlib.sha256(prev_a4 + ph + sh + vh + tail).digest()
    return scan, a4


CHAIN_ZERO = b"\0" * 32
