"""CPU oracle for the power-residue census -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this package, and only as the checker.  The product package
rabung_atlas32_b200 never imports it.

`census_oracle.c` restates the reference's CPU arithmetic (each function
cites the reference file:line it follows); `reference.py` drives the
reference's own CPU programs built from its sources into oracle/_ref by
oracle/Makefile.ref.  Parity of this oracle is pinned against the
reference's shipped sample blocks, holdout profiles and reference-program
outputs in tests/test_oracle.py.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
LIB = BUILD / "liboracle.so"
SRC = HERE / "census_oracle.c"


def build(force: bool = False) -> Path:
    """Compile census_oracle.c into oracle/_build/liboracle.so (rebuilt when
    the SHA-256 of the source, kept in liboracle.so.key, changes)."""
    import hashlib
    key = hashlib.sha256(SRC.read_bytes()).hexdigest()
    kf = BUILD / "liboracle.so.key"
    if LIB.exists() and not force and kf.exists() and kf.read_text().strip() == key:
        return LIB
    BUILD.mkdir(exist_ok=True)
    tmp = BUILD / f"liboracle.{os.getpid()}.so"
    subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-o", str(tmp), str(SRC)], check=True)
    os.replace(tmp, LIB)
    kf.write_text(key + "\n")
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB))
        u64, u32 = ctypes.c_uint64, ctypes.c_uint32
        P = ctypes.POINTER(u64)
        L.orc_is_prime.argtypes = [u64]
        L.orc_is_prime.restype = ctypes.c_int
        L.orc_mask.argtypes = [u64]
        L.orc_mask.restype = u32
        L.orc_profiles_dense.argtypes = [u64, u32, P, P, P]
        L.orc_profiles_dense.restype = ctypes.c_int
        for name in ("orc_a4_dense", "orc_a4", "orc_elliptic_count", "orc_primitive_root"):
            getattr(L, name).argtypes = [u64]
            getattr(L, name).restype = u64
        L.orc_a4_from_count.argtypes = [u64, u64]
        L.orc_a4_from_count.restype = u64
        L.orc_threshold_k.argtypes = [u64, u64, u64, u64]
        L.orc_threshold_k.restype = u64
        L.orc_prefix.argtypes = [u64, u64]
        L.orc_prefix.restype = u64
        L.orc_sieve.argtypes = [u64, u64, P, u64]
        L.orc_sieve.restype = u64
        _lib = L
    return _lib


def is_prime(n: int) -> bool:
    return bool(lib().orc_is_prime(n))


def mask(p: int) -> int:
    return int(lib().orc_mask(p))


def threshold_k(p: int, r: int, M: int, L: int) -> int:
    return int(lib().orc_threshold_k(p, r, M, L))


def profiles(p: int, m: int | None = None) -> list[dict]:
    """Dense profiles of p for every set bit of `m` (default: all admissible r),
    as reference-style dicts {r, max, prefix, K, witness}."""
    if m is None:
        m = mask(p)
    M = (ctypes.c_uint64 * 10)()
    L = (ctypes.c_uint64 * 10)()
    W = (ctypes.c_uint64 * 10)()
    if lib().orc_profiles_dense(p, m, M, L, W) != 0:
        raise MemoryError("oracle walk allocation")
    out = []
    for r in range(2, 10):
        if m & (1 << (r - 2)):
            out.append({"r": r, "max": M[r], "prefix": L[r],
                        "K": threshold_k(p, r, M[r], L[r]), "witness": W[r]})
    return out


def prefix(p: int, r: int) -> int:
    return int(lib().orc_prefix(p, r))


def a4(p: int) -> int:
    if p == 2:
        return 0
    v = int(lib().orc_a4(p))
    if v == 2**64 - 1:
        raise ArithmeticError(f"oracle A4 failed for {p}")
    return v


def a4_dense(p: int) -> int:
    return int(lib().orc_a4_dense(p))


def elliptic_count(p: int) -> int:
    return int(lib().orc_elliptic_count(p))


def sieve(lo: int, hi: int) -> list[int]:
    cap = max(16, int((hi - lo) / 2) + 16)
    buf = (ctypes.c_uint64 * cap)()
    n = lib().orc_sieve(lo, hi, buf, cap)
    return list(buf[:n])
