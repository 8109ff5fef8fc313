"""Record format: the encoder reproduces the reference's shipped sample
frames byte for byte and the decoder rejects damaged frames, as the
reference's tests/test_integrity.py:12-24 requires of its decoder."""
import hashlib
import json

import pytest

from conftest import GOLDEN
from rabung_atlas32_b200 import codec


@pytest.mark.parametrize("blk", ["00000", "49900"])
def test_frames_roundtrip_bytes(golden, blk):
    recs, meta, ameta = golden[blk]
    scan = codec.encode_scan_frame(meta["lo"], meta["hi"], recs)
    a4 = codec.encode_a4_frame(meta["lo"], meta["hi"], recs)
    assert scan == (GOLDEN / f"scan-{blk}.vdw").read_bytes()
    assert a4 == (GOLDEN / f"quadruplets-{blk}.a4").read_bytes()


def test_manifest_hashes(golden):
    man = json.loads((GOLDEN / "manifest.json").read_text())
    for block in man["blocks"]:
        blk = f"{block['block']:05d}"
        recs, meta, ameta = golden[blk]
        assert codec.prime_hash(recs).hex() == block["prime_hash"] == ameta["prime_hash"]
        assert codec.science_hash(recs).hex() == block["science_hash"] == ameta["profile_science_hash"]
        assert hashlib.sha256(codec.a4_values_raw(recs)).hexdigest() == block["values_hash"]
        for f in block["frames"]:
            b = (GOLDEN / f["file"]).read_bytes()
            assert len(b) == f["bytes"] and hashlib.sha256(b).hexdigest() == f["sha256"]


def test_damaged_frames_rejected():
    frame = (GOLDEN / "scan-00000.vdw").read_bytes()
    a4 = (GOLDEN / "quadruplets-00000.a4").read_bytes()
    for bad in (frame[:-1], frame + b"\0", frame[:100] + bytes([frame[100] ^ 1]) + frame[101:]):
        with pytest.raises(Exception):
            codec.decode_scan_frame(bad)
    for bad in (a4[:-1], a4 + b"\0", a4[:150] + bytes([a4[150] ^ 1]) + a4[151:]):
        with pytest.raises(Exception):
            codec.decode_a4_frame(bad)


def test_varint_canonical():
    out = bytearray()
    for v in (0, 1, 127, 128, 300, 2**32, 2**64 - 1):
        out.clear()
        codec.put_uint(out, v)
        assert codec.get_uint(bytes(out), 0) == (v, len(out))
    with pytest.raises(ValueError):
        codec.get_uint(bytes([0x80, 0x00]), 0)      # non-canonical
    with pytest.raises(ValueError):
        codec.get_uint(bytes([0x80]), 0)            # truncated


def test_chain_step_deterministic(golden):
    recs, meta, _ = golden["00000"]
    s1, a1 = codec.chain_step(codec.CHAIN_ZERO, codec.CHAIN_ZERO, meta["lo"], meta["hi"], recs)
    s2, a2 = codec.chain_step(codec.CHAIN_ZERO, codec.CHAIN_ZERO, meta["lo"], meta["hi"], recs)
    assert s1 == s2 and a1 == a2 and s1 != a1 and len(s1) == 32


def test_k_formula():
    # worked example p=101, r=2 -> (M, L, K, w) = (7, 1, 8, 19)
    assert codec.minimum_k(101, 2, 7, 1) == 8
