"""Python host API of the B200 census engine.

`Census` wraps one library handle (one CUDA stream).  `profiles()` is the
per-prime computation the reference census worker performs for each line of
its protocol (src/census/worker32.cu:20-41): every admissible r, (M, L,
witness, K), with the same refusal rule (a failed check refuses the whole
request, docs/METHODS.md:35).  `block()` produces the reference's VDWSM1 /
VDWA4V1 frames for an interval (docs/DATA_FORMAT.md).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

from . import _lib, codec

MODES = {"dense": _lib.CZ_DENSE, "sparse": _lib.CZ_SPARSE, "auto": _lib.CZ_AUTO}


class CensusError(RuntimeError):
    """A refused request: no partial result is returned."""


def prime_count(lo: int, hi: int) -> int:
    """Exact number of primes in [lo, hi), hi <= 2^33, computed on the host by
    the library (cz_prime_count; needs no GPU)."""
    return int(_lib.load().cz_prime_count(int(lo), int(hi)))


@dataclass
class Tuning:
    sparse_min_p: int = 1 << 20
    cover_n: int = 3
    q_cap: tuple = (0, 0, 30, 24, 20, 16, 16, 15, 14, 13)
    anchor_bits: int = 4
    screen: int = 1
    sparse_blocks: int = 0
    use_graph: int = 1
    cta_per_profile: int = 1
    epoch_rows: int = 1024
    speculate: int = 1
    spec_margin10: tuple = (0, 0, 30, 20, 15, 15, 10, 0, 5, 10)
    plane_budget_mb: int = 24 * 1024
    dense_steps: int = 256
    anchor_t: tuple = (0, 0, 11, 7, 6, 5, 5, 5, 5, 5)


def _as_u32_array(values):
    arr = (ctypes.c_uint32 * len(values))()
    for i, v in enumerate(values):
        if not 0 <= int(v) < 2 ** 32:
            raise ValueError(f"prime out of the 32-bit domain: {v}")
        arr[i] = int(v)
    return arr


def to_records(primes, out, a4v) -> list:
    """codec.Record list from C records grouped by prime in input order."""
    recs, k = [], 0
    for i, p in enumerate(primes):
        rec = codec.Record(int(p), [], a4v[i] if a4v else 0)
        for _ in range(bin(codec.expected_mask(p)).count("1") if p > 2 else 0):
            v = out[k]
            k += 1
            rec.profiles.append(codec.Profile(v.r, v.M, v.L, v.witness, v.K))
        recs.append(rec)
    return recs


def config(lib, device: int, t: Tuning) -> "_lib.cz_config":
    """The library configuration of a Tuning on `device`."""
    cfg = _lib.cz_config()
    lib.cz_default_config(ctypes.byref(cfg))
    cfg.device = device
    cfg.sparse_min_p = t.sparse_min_p
    cfg.cover_n = t.cover_n
    cfg.anchor_bits = t.anchor_bits
    cfg.screen = t.screen
    cfg.sparse_blocks = t.sparse_blocks
    cfg.use_graph = t.use_graph
    cfg.cta_per_profile = t.cta_per_profile
    cfg.epoch_rows = t.epoch_rows
    cfg.speculate = t.speculate
    cfg.plane_budget_mb = t.plane_budget_mb
    cfg.dense_steps = t.dense_steps
    for r in range(10):
        cfg.q_cap[r] = t.q_cap[r]
        cfg.spec_margin10[r] = t.spec_margin10[r]
        cfg.anchor_t[r] = t.anchor_t[r]
    return cfg


class Census:
    def __init__(self, device: int = 0, tuning: Tuning | None = None, autoload: bool = True):
        """Open a handle on `device`.  Without an explicit tuning, the
        autotuner's saved choices for this GPU (rabung_atlas32_b200/tuned/) are
        used when present."""
        self.lib = _lib.load()
        self.h = None
        self.tuned_from = None
        if tuning is None and autoload:
            self._open(device, Tuning())
            from .autotune import device_key, load_tuned
            key = device_key(self)
            t = load_tuned(key)
            if t is None:
                return
            self.close()
            self.tuned_from = key
            tuning = t
        self._open(device, tuning or Tuning())

    def _open(self, device: int, t: Tuning):
        h = ctypes.c_void_p()
        rc = self.lib.cz_open(ctypes.byref(config(self.lib, device, t)), ctypes.byref(h))
        if rc != 0:
            raise CensusError(f"cz_open failed (rc={rc}): no usable CUDA device or bad tuning")
        self.h = h
        self.tuning = t
        self.last_stats: dict = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.cz_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self) -> str:
        return self.lib.cz_last_error(self.h).decode(errors="replace")

    def count_profiles(self, primes) -> int:
        arr = _as_u32_array(primes)
        return int(self.lib.cz_count_profiles(arr, len(primes)))

    def raw(self, primes, mode: str = "auto", a4: bool = True, verify: bool = True):
        """Run the census; returns (ctypes profile array, A4 list or None, stats dict).

        With verify (the default) every witness run is re-proved on the device
        by direct powers -- monochromatic over its M positions and closed at
        both ends -- and every dense prefix re-checked, as the reference worker
        certifies each record before emitting it (src/census/worker32.cu:37-38,
        B2/src/advance.cpp:7-13); a failure refuses the request."""
        n = len(primes)
        arr = _as_u32_array(primes)
        nprof = int(self.lib.cz_count_profiles(arr, n))
        out = (_lib.cz_profile * max(1, nprof))()
        a4buf = (ctypes.c_uint32 * max(1, n))() if a4 else None
        flags = MODES[mode] | (_lib.CZ_A4 if a4 else 0) | (_lib.CZ_VERIFY if verify else 0)
        st = _lib.cz_stats()
        rc = self.lib.cz_census(self.h, arr, n, flags, out, nprof, a4buf, ctypes.byref(st))
        if rc != 0:
            raise CensusError(f"census refused (rc={rc}): {self._err()}")
        self.last_stats = st.as_dict()
        return out, (list(a4buf[:n]) if a4 else None), self.last_stats

    def profiles(self, primes, mode: str = "auto", a4: bool = True, verify: bool = True):
        """List of codec.Record (profiles ascending r, A4 when requested)."""
        out, a4v, _ = self.raw(primes, mode, a4, verify)
        return to_records(primes, out, a4v)

    def interval(self, lo: int, hi: int, mode: str = "auto", a4: bool = True, verify: bool = True,
                 max_primes: int = 1 << 20):
        """(primes, records) of every prime in [lo, hi): device sieve + census
        in one library call (cz_census_interval), its buffers sized from the
        exact prime count of the interval.  More than max_primes primes in the
        interval is an error."""
        lo, hi = int(lo), int(hi)
        cap = prime_count(lo, hi)
        if cap > max_primes:
            raise CensusError(f"[{lo}, {hi}) holds {cap} primes, above max_primes = {max_primes}")
        out_cap = 8 * max(1, cap)
        flags = MODES[mode] | (_lib.CZ_A4 if a4 else 0) | (_lib.CZ_VERIFY if verify else 0)
        ps = (ctypes.c_uint32 * max(1, cap))()
        npr, nprof = ctypes.c_uint32(), ctypes.c_uint32()
        out = (_lib.cz_profile * out_cap)()
        a4buf = (ctypes.c_uint32 * max(1, cap))() if a4 else None
        st = _lib.cz_stats()
        rc = self.lib.cz_census_interval(self.h, lo, hi, flags, ps, max(1, cap), ctypes.byref(npr), out, out_cap,
                                         ctypes.byref(nprof), a4buf, ctypes.byref(st))
        if rc != 0:
            raise CensusError(f"interval census refused (rc={rc}, primes {npr.value}): {self._err()}")
        self.last_stats = st.as_dict()
        primes = list(ps[:npr.value])
        return primes, to_records(primes, out, list(a4buf[:npr.value]) if a4 else None)

    def replay(self) -> dict:
        """Re-run the device work of the last call on its resident inputs."""
        st = _lib.cz_stats()
        rc = self.lib.cz_replay(self.h, ctypes.byref(st))
        if rc != 0:
            raise CensusError(f"replay refused (rc={rc}): {self._err()}")
        return st.as_dict()

    def microbench(self, kind: int) -> float:
        """Measured peak: kind 0 plane-word tests/s, kind 1 Montgomery products/s."""
        v = ctypes.c_double()
        rc = self.lib.cz_microbench(self.h, kind, ctypes.byref(v))
        if rc != 0:
            raise CensusError(f"microbench failed (rc={rc}): {self._err()}")
        return v.value

    def sieve(self, requests) -> list:
        """Device sieve: for each (lo, count), the first `count` primes >= lo."""
        n = len(requests)
        lo = (ctypes.c_uint32 * max(1, n))(*[int(a) for a, _ in requests])
        cnt = (ctypes.c_uint32 * max(1, n))(*[int(b) for _, b in requests])
        total = sum(int(b) for _, b in requests)
        out = (ctypes.c_uint32 * max(1, total))()
        found = (ctypes.c_uint32 * max(1, n))()
        rc = self.lib.cz_sieve(self.h, lo, cnt, n, out, found)
        if rc != 0:
            raise CensusError(f"sieve refused (rc={rc}): {self._err()}")
        res, off = [], 0
        for i in range(n):
            res.append(list(out[off: off + found[i]]))
            off += int(cnt[i])
        return res

    def plane_bytes(self, primes, mode: str = "auto") -> int:
        arr = _as_u32_array(primes)
        return int(self.lib.cz_plane_bytes(self.h, arr, len(primes), MODES[mode]))

    def mem_info(self) -> tuple:
        f, t = ctypes.c_uint64(), ctypes.c_uint64()
        rc = self.lib.cz_mem_info(self.h, ctypes.byref(f), ctypes.byref(t))
        if rc != 0:
            raise CensusError(f"mem_info failed: {self._err()}")
        return int(f.value), int(t.value)

    def a4(self, primes) -> list:
        n = len(primes)
        arr = _as_u32_array(primes)
        buf = (ctypes.c_uint32 * max(1, n))()
        rc = self.lib.cz_a4(self.h, arr, n, buf)
        if rc != 0:
            raise CensusError(f"A4 refused (rc={rc}): {self._err()}")
        return list(buf[:n])

    def block(self, lo: int, hi: int, primes=None, mode: str = "auto", verify: bool = True):
        """(scan_frame, a4_frame, records) for the primes of [lo, hi), every
        record certified on the device unless verify is False."""
        if primes is None:
            from .sieve import primes_in
            primes = primes_in(lo, hi)
        recs = self.profiles(primes, mode=mode, a4=True, verify=verify)
        return codec.encode_scan_frame(lo, hi, recs), codec.encode_a4_frame(lo, hi, recs), recs


class Census64:
    """The census for primes below 2^33 (the reference's 33-bit domain):
    cz_open64 / cz_census64, the same kernels compiled for 64-bit prime
    words.  Same tuning, modes, A4, certification and refusal rules as
    Census; records carry p as a Python int."""

    def __init__(self, device: int = 0, tuning: Tuning | None = None):
        self.lib = _lib.load()
        self.h = None
        if tuning is None:
            with Census(device=device, autoload=True) as probe:
                tuning = probe.tuning
        h = ctypes.c_void_p()
        rc = self.lib.cz_open64(ctypes.byref(config(self.lib, device, tuning)), ctypes.byref(h))
        if rc != 0:
            raise CensusError(f"cz_open64 failed (rc={rc}): no usable CUDA device or bad tuning")
        self.h = h
        self.tuning = tuning
        self.last_stats: dict = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.cz_close64(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _arr(primes):
        arr = (ctypes.c_uint64 * max(1, len(primes)))()
        for i, v in enumerate(primes):
            if not 0 <= int(v) < 2 ** 33:
                raise ValueError(f"prime out of the 33-bit domain: {v}")
            arr[i] = int(v)
        return arr

    def count_profiles(self, primes) -> int:
        return int(self.lib.cz_count_profiles64(self._arr(primes), len(primes)))

    def raw(self, primes, mode: str = "auto", a4: bool = True, verify: bool = True):
        """(ctypes cz_profile64 array, A4 list or None, stats dict)."""
        n = len(primes)
        arr = self._arr(primes)
        nprof = int(self.lib.cz_count_profiles64(arr, n))
        out = (_lib.cz_profile64 * max(1, nprof))()
        a4buf = (ctypes.c_uint32 * max(1, n))() if a4 else None
        flags = MODES[mode] | (_lib.CZ_A4 if a4 else 0) | (_lib.CZ_VERIFY if verify else 0)
        st = _lib.cz_stats()
        rc = self.lib.cz_census64(self.h, arr, n, flags, out, nprof, a4buf, ctypes.byref(st))
        if rc != 0:
            err = self.lib.cz_last_error64(self.h).decode(errors="replace")
            raise CensusError(f"census refused (rc={rc}): {err}")
        self.last_stats = st.as_dict()
        return out, (list(a4buf[:n]) if a4 else None), self.last_stats

    def profiles(self, primes, mode: str = "auto", a4: bool = True, verify: bool = True):
        """List of codec.Record (profiles ascending r, A4 when requested)."""
        out, a4v, _ = self.raw(primes, mode, a4, verify)
        return to_records(primes, out, a4v)


def main(argv=None):
    """One census of a window of consecutive primes, printing the call's stats:

        python -m rabung_atlas32_b200.census --ending 4294967291 --count 512 --mode sparse
        python -m rabung_atlas32_b200.census --from 16777216 --count 4096 --mode dense --a4
        python -m rabung_atlas32_b200.census --microbench        (measured integer peaks)
    """
    import argparse
    import json
    from . import sieve
    ap = argparse.ArgumentParser(description=main.__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    g = ap.add_mutually_exclusive_group(required=True)
    g.add_argument("--microbench", action="store_true", help="print this GPU's measured integer peaks")
    g.add_argument("--ending", type=int, help="the window ends at this prime")
    g.add_argument("--from", dest="start", type=int, help="the window starts at the first prime >= this")
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--mode", default="auto", choices=list(MODES))
    ap.add_argument("--a4", action="store_true")
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args(argv)
    if a.microbench:
        with Census() as c:
            print(json.dumps({"plane_word_tests_per_s": c.microbench(0), "montgomery_products_per_s": c.microbench(1)}))
        return
    ps = sieve.primes_ending(a.ending, a.count) if a.ending else sieve.primes_from(a.start, a.count)
    with Census() as c:
        for _ in range(a.repeat):
            _, _, st = c.raw(ps, mode=a.mode, a4=a.a4)
            print(json.dumps({k: (round(v, 3) if isinstance(v, float) else v) for k, v in st.items()}))


if __name__ == "__main__":
    main()
