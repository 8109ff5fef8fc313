"""Serving loop: census requests for prime intervals arriving over time.

A request asks for the profiles (and A4) of the `count` consecutive primes
starting at `lo`.  The server keeps every request's state resident until it
completes and runs continuous batching over `slots` in-flight batches (one
library handle, hence one CUDA stream, per slot):

  * whenever a slot is free, every waiting request that fits is admitted into
    one batch -- admission by device memory: the batch's colour-plane pool must
    fit the slot's budget and the GPU's free memory (cz_mem_info);
  * the batch's intervals are sieved on the device (cz_sieve), merged into one
    census call (one persistent filter launch over all their profiles), and the
    records are split back per request;
  * requests that arrive while batches run wait for the next free slot, so work
    of different batches overlaps on the device.

The reference has no serving path (its supervisor feeds fixed blocks to
worker processes, src/census/worker32.cu:10-45); the records are the same as
the census worker's for the same primes.

`benchmark()` replays a seeded trace (Poisson arrivals at `rate` requests/s,
start log-uniform in [2^12, 2^32), length log-uniform in 1..4096 primes) and
reports p50/p99 latency and profiles/s, next to plain per-request calls.
"""
from __future__ import annotations

import math
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from .census import Census, Tuning


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
    def __init__(self, slots: int = 2, slot_budget_mb: int = 16 * 1024, device: int = 0,
                 reserve_mb: int = 4096, max_batch_requests: int = 4096, tuning: Tuning | None = None):
        self.slots = [Census(device=device, tuning=tuning) for _ in range(slots)]
        self.slot_budget = slot_budget_mb << 20
        self.reserve = reserve_mb << 20
        self.max_batch = max_batch_requests
        self.waiting: list = []
        self.cv = threading.Condition()
        self.closed = False
        self.t0 = 0.0
        self.batches = 0
        self.error: Exception | None = None

    def close(self):
        for s in self.slots:
            s.close()

    # -- admission ------------------------------------------------------------
    def _admit(self, eng: Census) -> list:
        """Take waiting requests (arrival order) while the batch fits memory."""
        free, _ = eng.mem_info()
        cap = min(self.slot_budget, max(0, free - self.reserve))
        batch, used = [], 0
        keep = []
        for r in self.waiting:
            if len(batch) >= self.max_batch:
                keep.append(r)
                continue
            # upper estimate of the request's planes: its count primes near lo's top
            est = eng.plane_bytes([min(2 ** 32 - 5, int(r.lo + r.count * max(1.0, math.log(r.lo + 2)) * 1.3))])
            est *= r.count
            if batch and used + est > cap:
                keep.append(r)
                continue
            batch.append(r)
            used += est
        self.waiting = keep
        return batch

    # -- one slot -------------------------------------------------------------
    def _slot_loop(self, k: int):
        eng = self.slots[k]
        while True:
            with self.cv:
                while not self.waiting and not self.closed:
                    self.cv.wait()
                if not self.waiting and self.closed:
                    return
                batch = self._admit(eng)
                self.batches += 1
                bid = self.batches
            try:
                self._run_batch(eng, batch, bid)
            except Exception as e:          # a refused batch fails the whole run
                self.error = e
                with self.cv:
                    self.closed = True
                    self.cv.notify_all()
                return

    def _run_batch(self, eng: Census, batch: list, bid: int):
        primes_per = eng.sieve([(r.lo, r.count) for r in batch])      # device sieve
        flat = [p for ps in primes_per for p in ps]
        recs = eng.profiles(flat, mode="auto", a4=True) if flat else []
        k = 0
        now = time.perf_counter() - self.t0
        for r, ps in zip(batch, primes_per):
            r.primes = ps
            r.records = recs[k:k + len(ps)]
            k += len(ps)
            r.done = now
            r.batch = bid

    # -- trace replay ---------------------------------------------------------
    def run(self, requests: list) -> list:
        """Serve a trace in real time (arrivals at their timestamps)."""
        threads = [threading.Thread(target=self._slot_loop, args=(k,), daemon=True) for k in range(len(self.slots))]
        self.t0 = time.perf_counter()
        for t in threads:
            t.start()
        for r in sorted(requests, key=lambda x: x.arrival):
            delay = r.arrival - (time.perf_counter() - self.t0)
            if delay > 0:
                time.sleep(delay)
            with self.cv:
                if self.closed:
                    break
                self.waiting.append(r)
                self.cv.notify()
        with self.cv:
            self.closed = True
            self.cv.notify_all()
        for t in threads:
            t.join()
        if self.error:
            raise self.error
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
              plain: bool = True) -> dict:
    trace = make_trace(requests, rate, seed)
    srv = Server(slots=slots)
    try:
        served = srv.run(trace)
    finally:
        srv.close()
    out = {"metric": "serving: p50/p99 latency and profiles/s", "offered_rate_rps": rate, "seed": seed,
           "slots": slots, "batches": srv.batches, "continuous": summarize(served)}
    if plain:
        ptrace = make_trace(requests, rate, seed)
        out["plain_per_request"] = summarize(serve_plain(ptrace))
        same = all([(x.p, [(v.r, v.M, v.L, v.witness) for v in x.profiles], x.a4) for x in a.records] ==
                   [(x.p, [(v.r, v.M, v.L, v.witness) for v in x.profiles], x.a4) for x in b.records]
                   for a, b in zip(served, ptrace))
        out["identical_alone_and_mixed"] = same
    return out
