"""Serving loop: census requests for prime intervals arriving over time.

A request asks for the profiles (and A4) of the `count` consecutive primes
starting at `lo`.  `Server` drives the library's native serving runtime
(cz_server_open / cz_submit / cz_next_done / cz_poll, csrc/runtime.cuh):

  * every admitted request stays resident on the GPU (descriptors, state,
    colour planes, records) until its records are final; admission is by free
    colour-plane memory and descriptor space;
  * the anchor filter is one persistent kernel over the unfinished profiles of
    all admitted requests; an arrival makes it yield between work items, the
    arrival is sieved, planned and tabled on the device, and the kernel is
    relaunched over old and new profiles together -- requests join the work in
    flight instead of waiting for a batch to end;
  * a request's records are copied out as soon as its last profile is final.

The reference has no serving path (its supervisor feeds fixed blocks to
worker processes, src/census/worker32.cu:10-45); the records are the same as
the census worker's for the same primes.

`benchmark()` replays a seeded trace (Poisson arrivals at `rate` requests/s,
start log-uniform in [2^12, 2^32), length log-uniform in 1..4096 primes) and
reports p50/p99 latency and profiles/s, next to plain per-request calls.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field

import numpy as np

from .census import Census, CensusError, Tuning, config, to_records


@dataclass
class Request:
    rid: int
    lo: int
    count: int
    arrival: float = 0.0          # seconds from trace start
    primes: list = field(default_factory=list)
    records: list = field(default_factory=list)
    done: float = -1.0            # completion time (seconds from trace start)
    batch: int = -1               # batch that served it


def make_trace(n: int, rate: float, seed: int = 20261203) -> list:
    """Seeded requests: exponential inter-arrival times (Poisson process of
    `rate` requests/s), start 2^U[12, 32), length floor(2^U[0, 12]) primes."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n)
    arr = np.cumsum(gaps) - gaps[0]
    starts = np.exp2(rng.uniform(12, 32, n)).astype(np.int64)
    counts = np.clip(np.floor(np.exp2(rng.uniform(0, 12, n))), 1, 4096).astype(np.int64)
    return [Request(i, int(s), int(c), float(a)) for i, (s, c, a) in enumerate(zip(starts, counts, arr))]


class Server:
    """The library's native serving runtime (cz_server_open / cz_submit /
    cz_next_done / cz_poll); its colour-plane memory is slots x slot_budget_mb."""

    def __init__(self, slots: int = 2, slot_budget_mb: int = 16 * 1024, device: int = 0,
                 tuning: Tuning | None = None):
        import ctypes
        from . import _lib
        self._ct, self._L = ctypes, _lib
        self.lib = _lib.load()
        probe = Census(device=device, tuning=tuning)      # resolves the tuning saved for this device
        try:
            cfg = config(self.lib, device, probe.tuning)
        finally:
            probe.close()
        h = ctypes.c_void_p()
        rc = self.lib.cz_server_open(ctypes.byref(cfg), slots, slot_budget_mb << 20, ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"cz_server_open failed (rc={rc})")
        self.h = h
        self._closed_batches = 0
        self._closed_stats = {}
        self.t0 = 0.0

    @property
    def batches(self) -> int:
        """Filter launches so far (the final count once the server is closed)."""
        if self.h is None:
            return self._closed_batches
        b = self._ct.c_uint64()
        self.lib.cz_server_info(self.h, self._ct.byref(b), None, None)
        return int(b.value)

    def stats(self) -> dict:
        """Scheduler counters (cz_server_stats); the final ones once closed."""
        if self.h is None:
            return dict(self._closed_stats)
        st = self._L.cz_server_counters()
        self.lib.cz_server_stats(self.h, self._ct.byref(st))
        return {k: (round(v, 1) if isinstance(v, float) else int(v)) for k, v in st.as_dict().items()}

    def close(self):
        if self.h is not None:
            self._closed_batches = self.batches
            self._closed_stats = self.stats()
            self.lib.cz_server_close(self.h)
            self.h = None

    def submit(self, lo: int, count: int, flags: int | None = None) -> int:
        ct = self._ct
        rid = ct.c_uint64()
        fl = (self._L.CZ_AUTO | self._L.CZ_A4 | self._L.CZ_VERIFY) if flags is None else flags
        rc = self.lib.cz_submit(self.h, int(lo), int(count), None, fl, ct.byref(rid))
        if rc != 0:
            raise RuntimeError(f"cz_submit failed (rc={rc})")
        return int(rid.value)

    def next_done(self, timeout_ms: int) -> int | None:
        rid = self._ct.c_uint64()
        rc = self.lib.cz_next_done(self.h, int(timeout_ms), self._ct.byref(rid))
        return int(rid.value) if rc == self._L.CZ_OK else None

    def fetch(self, rid: int, count: int) -> tuple:
        """(primes, records) of a completed request (releases it)."""
        ct, L = self._ct, self._L
        ps = (ct.c_uint32 * max(1, count))()
        out = (L.cz_profile * max(1, 8 * count))()
        a4 = (ct.c_uint32 * max(1, count))()
        npr, nprof = ct.c_uint32(), ct.c_uint32()
        rc = self.lib.cz_poll(self.h, rid, -1, ps, count, ct.byref(npr), out, 8 * count, ct.byref(nprof), a4)
        if rc != 0:
            raise CensusError(f"request {rid} refused (rc={rc}): "
                              f"{self.lib.cz_server_last_error(self.h).decode(errors='replace')}")
        primes = list(ps[:npr.value])
        return primes, to_records(primes, out, list(a4[:npr.value]))

    def run(self, requests: list) -> list:
        """Serve a trace in real time: each request is submitted at its arrival
        time; a collector thread takes completions as they happen."""
        by_id, errors = {}, []
        lock = threading.Lock()

        def collect():
            pending = len(requests)
            while pending:
                rid = self.next_done(50)
                if rid is None:
                    continue
                now = time.perf_counter() - self.t0
                with lock:
                    r = by_id[rid]
                try:
                    r.primes, r.records = self.fetch(rid, r.count)
                except Exception as e:              # a refused request fails the run
                    errors.append(e)
                r.done = now
                pending -= 1

        th = threading.Thread(target=collect, daemon=True)
        self.t0 = time.perf_counter()
        th.start()
        for r in sorted(requests, key=lambda x: x.arrival):
            delay = r.arrival - (time.perf_counter() - self.t0)
            if delay > 0:
                time.sleep(delay)
            with lock:
                by_id[self.submit(r.lo, r.count)] = r
        th.join()
        if errors:
            raise errors[0]
        return requests


def serve_plain(requests: list, device: int = 0) -> list:
    """Plain form: one call per request, in arrival order, one stream."""
    eng = Census(device=device)
    t0 = time.perf_counter()
    try:
        for r in sorted(requests, key=lambda x: x.arrival):
            delay = r.arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            (ps,) = eng.sieve([(r.lo, r.count)])
            r.primes = ps
            r.records = eng.profiles(ps, mode="auto", a4=True)
            r.done = time.perf_counter() - t0
    finally:
        eng.close()
    return requests


def summarize(reqs: list) -> dict:
    lat = np.array([r.done - r.arrival for r in reqs])
    prof = sum(len(rec.profiles) for r in reqs for rec in r.records)
    span = max(r.done for r in reqs) - min(r.arrival for r in reqs)
    return {"requests": len(reqs), "profiles": int(prof), "p50_ms": round(1000 * float(np.percentile(lat, 50)), 2),
            "p99_ms": round(1000 * float(np.percentile(lat, 99)), 2),
            "mean_ms": round(1000 * float(lat.mean()), 2), "profiles_per_s": round(prof / span, 1),
            "span_s": round(span, 2)}


def benchmark(requests: int = 10000, rate: float = 40.0, seed: int = 20261203, slots: int = 2,
              plain: bool = True, plain_requests: int | None = None) -> dict:
    """The trace served continuously; then, for comparison, its first
    `plain_requests` requests (all when None) at the same arrival times as
    plain per-request calls, with their records checked equal."""
    trace = make_trace(requests, rate, seed)
    srv = Server(slots=slots)
    try:
        served = srv.run(trace)
    finally:
        srv.close()
    out = {"metric": "serving: p50/p99 latency and profiles/s", "offered_rate_rps": rate, "seed": seed,
           "slots": slots, "filter_launches": srv.batches, "scheduler": srv.stats(),
           "continuous": summarize(served)}
    if plain:
        k = requests if plain_requests is None else min(requests, plain_requests)
        ptrace = make_trace(requests, rate, seed)[:k]
        out["plain_per_request"] = summarize(serve_plain(ptrace))
        out["plain_per_request"]["trace_prefix"] = k
        out["continuous_same_prefix"] = summarize(served[:k])
        same = all([(x.p, [(v.r, v.M, v.L, v.witness) for v in x.profiles], x.a4) for x in a.records] ==
                   [(x.p, [(v.r, v.M, v.L, v.witness) for v in x.profiles], x.a4) for x in b.records]
                   for a, b in zip(served, ptrace))
        out["identical_alone_and_mixed"] = same
    return out
