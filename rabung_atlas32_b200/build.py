"""Build librabung_census.so in-tree with nvcc for sm_100a.

    python -m rabung_atlas32_b200.build        (or build() from Python)

The library is a plain C-ABI shared object (include/rabung_census.h); the
Python package loads it with ctypes.  A build is reused only when the SHA-256
of its sources, flags and compiler path (kept beside the library in
librabung_census.so.key) matches: a library built from other sources, however
new its file time, is rebuilt.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "librabung_census.so"
KEY = PKG / "librabung_census.so.key"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "rabung_census.h"]


def source_key(extra=()) -> str:
    """SHA-256 over every source file's name and bytes, the flags and nvcc."""
    h = hashlib.sha256()
    for p in sources():
        h.update(p.name.encode() + b"\0" + p.read_bytes() + b"\0")
    h.update(" ".join([NVCC, *FLAGS, *extra]).encode())
    return h.hexdigest()


def compile_library(out: Path, extra=(), verbose: bool = False) -> None:
    """nvcc both translation units (32-bit and 33-bit prime words) into one
    shared library at `out`; `extra` adds flags (e.g. -D build macros)."""
    cmd = [NVCC, *FLAGS, *extra, "-I", str(ROOT / "include"), "-o", str(out), str(CSRC / "census.cu"),
           str(CSRC / "census_wide.cu")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed for {out.name}")
    if verbose:
        sys.stderr.write(r.stderr)


def build(force: bool = False, verbose: bool = False) -> Path:
    key = source_key()
    if LIB.exists() and not force and KEY.exists() and KEY.read_text().strip() == key:
        return LIB
    tmp = LIB.with_suffix(f".{os.getpid()}.tmp.so")
    compile_library(tmp, verbose=verbose)
    os.replace(tmp, LIB)
    KEY.write_text(key + "\n")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
