#!/usr/bin/env python3
"""Benchmark of the B200 power-residue census (one JSON line on rank 0).

Workload (one "step"): the census of the top block -- the 4096 consecutive
primes ending at 4294967291 (4,294,875,371 .. 4,294,967,291), every admissible
order r in 2..9 (13,660 profiles: M, L, witness, K) plus the quadratic A4 of
every prime, through the certified rational-anchor filter.  Metric: profiles/s.

  value     device throughput with the inputs resident in HBM: K replays of
            the captured device work (CUDA graph), timed with CUDA events on
            the library's own stream, L2 flushed between steps; every step
            certifies every record on the device (witness run monochromatic
            and closed at both ends, prefix, by direct powers), as the
            reference worker does before it emits a record;
  e2e       the same certified census through the public C ABI (cz_census)
            from host buffers: planning, pinned host->device copies, kernels
            and the device->host read of every record, timed per step on the
            host;
  roofline  dominant kernel (sparse_kernel): plane-window comparisons per second
            against this GPU's measured integer-ALU peak for the same
            operation (cz_microbench);
  cpu_baseline / --impl reference
            the reference's own CPU sparse engines -- `target p c f 64 1 8192 1`
            for the coupled order pairs {2, 4} and {3, 6}, `advance adaptive
            p r 64 3 1` for every other order -- and its A4 worker
            (`moment_worker`), built from its sources into oracle/_ref, on a
            seeded sample of whole primes of the same workload (every
            admissible order of each, >= 256 profiles), on all host cores;
  c4, c2, c5
            (one GPU, unless --quick) the batched uneven census of 64 blocks
            of 4096 primes against one block per call; the C2 block (4096
            primes from 16,777,259) through the dense scan, with its Montgomery
            roofline, and in auto mode, records compared; and the serving
            stream of 10,000 requests against plain per-request calls -- each
            with its own clock record.

Multi-GPU (torchrun): every rank censuses its own 4096-prime block (rank k
takes the 4096 primes below rank k-1's block): independent blocks, no
collective on the data path (weak scaling); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import random
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "profiles/s (all r|p-1) near 2^32, bit-exact, batched vs plain; serve p50/p99"
TOP = 4294967291
BLOCK = 4096


def uneven_blocks(rank: int = 0, nblocks: int = 64, size: int = BLOCK, seed: int = 20261203) -> list:
    """64 blocks of 4096 consecutive primes, starts log-uniform over [2^16, 2^32)
    from a fixed seed (rank k draws from seed + k)."""
    import numpy as np
    from rabung_atlas32_b200 import sieve
    rng = np.random.default_rng(seed + rank)
    starts = sorted(int(x) for x in np.exp2(rng.uniform(16, 32, nblocks)))
    return [sieve.primes_from(s, size) for s in starts]


def c4_measure(eng, steps: int, warmup: int) -> dict:
    """C4: 64 uneven blocks in one certified call (persistent kernels, waves
    when the plane pool exceeds its budget) against one block per call, same
    GPU, records compared bit for bit."""
    blocks = uneven_blocks(int(os.environ.get("RANK", "0")))
    flat = [p for b in blocks for p in b]
    nprof = eng.count_profiles(flat)
    for _ in range(max(1, warmup)):
        eng.raw(flat, mode="auto", a4=True)
    dev, e2e, waves = [], [], 0
    for _ in range(steps):
        t0 = time.perf_counter()
        out, a4, st = eng.raw(flat, mode="auto", a4=True)
        e2e.append(time.perf_counter() - t0)
        dev.append(st["ms_device"] / 1000.0)
        waves = st["waves"]
    batched = [(o.p, o.r, o.M, o.L, o.witness) for o in out[:nprof]] + [tuple(a4)]
    plain_dev, plain_e2e, plain_rec, plain_a4 = 0.0, 0.0, [], []
    for b in blocks:
        t0 = time.perf_counter()
        o, a, st = eng.raw(b, mode="auto", a4=True)
        plain_e2e += time.perf_counter() - t0
        plain_dev += st["ms_device"] / 1000.0
        plain_rec += [(x.p, x.r, x.M, x.L, x.witness) for x in o[:eng.count_profiles(b)]]
        plain_a4 += a
    same = batched == plain_rec + [tuple(plain_a4)]
    mean_dev = sum(dev) / len(dev)
    return {
        "metric": "profiles/s, batched uneven census (64 blocks x 4096 primes, log-uniform starts in [2^16, 2^32))",
        "value": round(nprof / mean_dev, 1), "unit": "profiles/s", "steps": steps,
        "primes": len(flat), "profiles": nprof, "waves": waves,
        "e2e": round(nprof / (sum(e2e) / len(e2e)), 1),
        "plain_one_block_per_call": {"value": round(nprof / plain_dev, 1), "e2e": round(nprof / plain_e2e, 1)},
        "batched_over_plain": round(plain_dev / mean_dev, 3), "bit_identical": same}


def c2_measure(eng, steps: int, warmup: int) -> dict:
    """C2: the 4096 primes from 16,777,259, certified, with A4 -- through the
    dense scan (every x of each half interval; the independent check) and in
    auto mode (these primes route to the anchor filter); the two record sets
    are compared bit for bit.  The dense scan's algorithmic work is one power
    x^e per x in [1, (p-1)/2], e = (p-1)/m, of bitlen(e) + popcount(e) - 2
    Montgomery products, rated against the measured Montgomery peak."""
    from math import gcd
    from rabung_atlas32_b200 import sieve
    ps = sieve.primes_from(16777259, BLOCK)
    nprof = eng.count_profiles(ps)
    products = 0
    for p in ps:
        m = 1
        for r in range(2, 10):
            if (p - 1) % r == 0:
                m = m * r // gcd(m, r)
        e = (p - 1) // m
        products += ((p - 1) // 2) * (e.bit_length() + bin(e).count("1") - 2)
    out = {"metric": "profiles/s, C2 block (4096 primes from 16,777,259, certified, A4)", "primes": len(ps),
           "profiles": nprof}
    recs = {}
    for mode in ("dense", "auto"):
        for _ in range(max(1, warmup)):
            eng.raw(ps, mode=mode, a4=True)
        dev, kern = [], []
        for _ in range(steps):
            o, a4, st = eng.raw(ps, mode=mode, a4=True)
            dev.append(st["ms_device"])
            kern.append(st["ms_dense"] if mode == "dense" else st["ms_sparse"])
        recs[mode] = [(x.p, x.r, x.M, x.L, x.witness, x.K) for x in o[:nprof]] + [tuple(a4)]
        ms = sum(dev) / len(dev)
        leg = {"value": round(nprof / (ms / 1000.0), 1), "unit": "profiles/s", "ms_device": round(ms, 3),
               "kernel_ms": round(sum(kern) / len(kern), 3)}
        if mode == "dense":
            peak = eng.microbench(1)
            rate = products / (leg["kernel_ms"] / 1000.0)
            leg["roofline"] = {"bound": "int_mul", "kernel": "dense_scan_kernel", "achieved": round(rate / 1e9, 2),
                               "peak": round(peak / 1e9, 2), "unit": "G Montgomery products/s",
                               "frac": round(rate / peak, 4),
                               "algorithmic": f"{products} Montgomery products per call (one power per x)",
                               "peak_source": "measured on this GPU by cz_microbench kind 1"}
        out[mode] = leg
    out["dense_equals_auto"] = recs["dense"] == recs["auto"]
    return out


def uneven_arm(args) -> None:
    from rabung_atlas32_b200.census import Census
    with Census() as eng:
        clk = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
        clk.start()
        res = c4_measure(eng, args.steps, args.warmup)
        res["clocks"] = clk.stop()
    print(json.dumps(res))


def max_over_ranks(values: list, dist=None, device=None) -> list:
    """Element-wise maximum of per-rank timings (every rank gets the result)."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """Sum of a per-rank count (every rank gets the result)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t[0])


def small_arm(args) -> None:
    """C1 (first 256 primes, dense) and C2 (4096 primes from 2^24, dense oracle
    and anchor filter) timings."""
    from rabung_atlas32_b200 import sieve
    from rabung_atlas32_b200.census import Census
    eng = Census()
    res = {}
    for name, ps, mode in (("C1_first_256_dense", sieve.primes_from(2, 256), "dense"),
                           ("C2_2p24_dense", sieve.primes_from(1 << 24, BLOCK), "dense"),
                           ("C2_2p24_sparse", sieve.primes_from(1 << 24, BLOCK), "sparse")):
        for _ in range(args.warmup):
            eng.raw(ps, mode=mode, a4=True)
        ms = []
        for _ in range(args.steps):
            _, _, st = eng.raw(ps, mode=mode, a4=True)
            ms.append(st["ms_device"])
        n = eng.count_profiles(ps)
        res[name] = {"profiles": n, "ms_device": round(sum(ms) / len(ms), 3),
                     "profiles_per_s": round(n / (sum(ms) / len(ms) / 1000.0), 1)}
    print(json.dumps({"metric": "profiles/s, C1 and C2 blocks", "results": res}))


def workload(rank: int) -> list:
    from rabung_atlas32_b200 import sieve
    hi = TOP
    ps = []
    for _ in range(rank + 1):
        ps = sieve.primes_ending(hi, BLOCK)
        hi = ps[0] - 1
    return ps


# ---------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi SM clock / throttle-reason samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = [l.split(",") for l in Path(self.file.name).read_text().splitlines() if l.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1])); smax.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if "Active" in v and "Not" not in v:
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------ reference CPU arm ----
def ref_bin(name: str) -> Path:
    return ROOT / "oracle" / "_ref" / name


def reference_available() -> str | None:
    for n in ("advance", "target", "moment_worker"):
        if not ref_bin(n).exists():
            return f"oracle/_ref/{n} not built (make -f oracle/Makefile.ref)"
    return None


def reference_jobs(primes: list, min_profiles: int = 256, seed: int = 20261203) -> tuple:
    """A seeded sample of whole primes of the workload (every admissible order
    of each) holding at least min_profiles profiles, as reference CPU jobs:
    ("target", p, c, f) for the coupled pairs {2, 4} and {3, 6} (the
    reference's coupled engine), ("advance", p, r, 0) for every other order.
    Returns (jobs, primes, profiles)."""
    rng = random.Random(seed)
    order = list(primes)
    rng.shuffle(order)
    jobs, picked, nprof = [], [], 0
    for p in order:
        if nprof >= min_profiles:
            break
        rs = [r for r in range(2, 10) if (p - 1) % r == 0]
        nprof += len(rs)
        picked.append(p)
        for c, f in ((2, 4), (3, 6)):
            if c in rs and f in rs:
                jobs.append(("target", p, c, f))
                rs = [r for r in rs if r not in (c, f)]
        jobs += [("advance", p, r, 0) for r in rs]
    # longest jobs first, so the pool's tail is short
    jobs.sort(key=lambda j: (j[0] != "target", j[1]))
    return jobs, sorted(picked), nprof


def run_reference_step(jobs: list, primes: list, cores: int) -> tuple:
    """Reference CPU census of a sample, one process per core: the sparse
    engines per job plus moment_worker A4 of the sample's primes; returns
    (seconds, records [p, r, M, L, witness])."""
    def one(job):
        kind, p, r, f = job
        if kind == "target":
            out = subprocess.run([str(ref_bin("target")), str(p), str(r), str(f), "64", "1", "8192", "1"],
                                 capture_output=True, text=True, check=True).stdout
            j = json.loads(out)
            return [(p, r, j["coarse_maximum"], j["coarse_prefix"], j["coarse_witness"]),
                    (p, f, j["fine_maximum"], j["fine_prefix"], j["fine_witness"])]
        out = subprocess.run([str(ref_bin("advance")), "adaptive", str(p), str(r), "64", "3", "1"],
                             capture_output=True, text=True, check=True).stdout
        j = json.loads(out)
        return [(p, r, j["maximum"], j["prefix"], j["witness"])]

    t0 = time.perf_counter()
    with ThreadPoolExecutor(cores) as ex:
        res = [v for part in ex.map(one, jobs) for v in part]
    line = f"0 -1 {len(primes)} " + " ".join(map(str, primes)) + "\nQUIT\n"
    subprocess.run([str(ref_bin("moment_worker"))], input=line.encode(), capture_output=True, check=True)
    return time.perf_counter() - t0, sorted(res)


def reference_sample_text(jobs: list, primes: list, nprof: int) -> str:
    nt = sum(1 for j in jobs if j[0] == "target")
    return (f"{len(primes)} seeded whole primes of the top block, {nprof} profiles per step: {nt} coupled "
            f"pairs by `target p c f 64 1 8192 1`, {len(jobs) - nt} orders by `advance adaptive p r 64 3 1`, "
            f"moment_worker A4 of the {len(primes)} primes")


def reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    why = reference_available()
    if why:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    cores = os.cpu_count() or 1
    primes = workload(0)
    jobs, sp, nprof = reference_jobs(primes)
    wjobs, wsp, _ = reference_jobs(primes, min_profiles=16, seed=1)
    for _ in range(args.warmup):
        run_reference_step(wjobs, wsp, cores)
    secs = []
    for _ in range(args.steps):
        s_, _ = run_reference_step(jobs, sp, cores)
        secs.append(s_)
    total = sum(secs)
    value = nprof * args.steps / total
    sample = reference_sample_text(jobs, sp, nprof)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": "profiles/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * total / args.steps, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "deterministic: the top block's own primes",
        "config": {"workload": "top block: 4096 consecutive primes ending at 4294967291, all admissible r",
                   "primes": BLOCK, "sample_profiles": nprof, "parallelism": "host processes"},
        "cpu_baseline": {"value": round(value, 2), "unit": "profiles/s", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 2), "unit": "profiles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ------------------------------------------------------------- our arm ----
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="top", choices=["top", "uneven", "serve", "small"])
    ap.add_argument("--requests", type=int, default=10000)
    ap.add_argument("--rate", type=float, default=40.0, help="offered load, requests/s (serve)")
    ap.add_argument("--quick", action="store_true", help="top block only: no C4 / C5 sub-objects")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.workload == "uneven":
        uneven_arm(args)
        return
    if args.workload == "small":
        small_arm(args)
        return
    if args.workload == "serve":
        from rabung_atlas32_b200 import serving
        clk = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
        clk.start()
        res = serving.benchmark(requests=args.requests, rate=args.rate, seed=20261203)
        res["clocks"] = clk.stop()
        print(json.dumps(res))
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    from rabung_atlas32_b200.census import Census

    primes = workload(rank)
    eng = Census(device=local)
    nprof = eng.count_profiles(primes)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    # warm-up: full public-API calls, then the graph capture
    for _ in range(args.warmup):
        eng.raw(primes, mode="auto", a4=True)
    kstats = dict(eng.last_stats)                 # per-kernel device times of a plain run
    eng.replay()

    # value: device replays with L2 flushed in between
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    dev_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        st = eng.replay()
        dev_ms.append(st["ms_device"])
    barrier()
    clk = clocks.stop()
    launches_per_step = int(kstats["kernels"])
    total_ms = sum(dev_ms)

    # e2e: the public API from host buffers (planning, pinned H2D, kernels, D2H)
    e2e_ms = []
    h2d = d2h = 0
    barrier()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, _, st = eng.raw(primes, mode="auto", a4=True)
        e2e_ms.append(1000 * (time.perf_counter() - t0))
        h2d, d2h = st["h2d_bytes"], st["d2h_bytes"]
    barrier()
    e2e_total = sum(e2e_ms)
    total_ms, e2e_total = max_over_ranks([total_ms, e2e_total], dist, f"cuda:{local}")
    all_prof = sum_over_ranks(nprof, dist, f"cuda:{local}")   # each rank's block has its own count
    value = all_prof * args.steps / (total_ms / 1000.0)
    e2e_value = all_prof * args.steps / (e2e_total / 1000.0)

    out = None
    if rank == 0:
        # roofline of the dominant kernel: plane-window comparisons per second
        peak_tests = eng.microbench(0)
        peak_mont = eng.microbench(1)
        ms_sparse = kstats["ms_sparse"]
        tests = kstats["tests"]
        achieved = tests / (ms_sparse / 1000.0)
        roof = {"bound": "int_alu", "kernel": "sparse_kernel", "achieved": round(achieved / 1e9, 2),
                "peak": round(peak_tests / 1e9, 2), "unit": "G plane-window tests/s",
                "frac": round(achieved / peak_tests, 4), "traffic": None,
                "algorithmic": f"{tests} tests per launch (stage x plane window comparisons, counted in-kernel)",
                "launch_ms": round(ms_sparse, 3),
                "peak_source": "measured on this GPU by cz_microbench kind 0 (MEASURED_PEAKS.json holds no integer peak)",
                "montgomery_peak_per_s": peak_mont,
                "kernel_ms": {k: round(kstats[k], 3) for k in ("ms_setup", "ms_table", "ms_sparse", "ms_dense",
                                                               "ms_a4", "ms_finalize")},
                "certification": "every record certified on the device in each step (finalize_kernel: witness "
                                 "run and its two ends by direct powers, prefix; its time is ms_finalize)"}
        # traffic measured in this run: the colour-plane bytes the filter staged
        # from global memory into shared memory (cp.async.bulk), counted in-kernel
        roof["traffic"] = int(kstats["staged_bytes"])
        roof["traffic_source"] = ("in-kernel count of plane bytes staged global -> shared by cp.async.bulk, "
                                  "one launch (the screen's and completions' direct plane reads are not included)")
        # for comparison: DRAM bytes of one full-size launch from the committed
        # ncu capture of this workload (dram__bytes_read.sum + dram__bytes_write.sum)
        prof_path = ROOT / "profiles" / "sparse_kernel_dram_top_block.txt"
        if prof_path.exists():
            for line in prof_path.read_text().splitlines():
                if line.startswith("dram_bytes_per_launch:"):
                    try:
                        roof["traffic_ncu_dram"] = int(line.split(":")[1].split()[0])
                        roof["traffic_ncu_source"] = prof_path.name
                    except ValueError:
                        pass
        # plain form: one prime per call (the reference worker's per-prime launches)
        plain_ps = primes[-64:]
        plain_ms, plain_prof = 0.0, 0
        for p in plain_ps:
            _, _, st = eng.raw([p], mode="auto", a4=True)
            plain_ms += st["ms_device"]
            plain_prof += st["n_profiles"]
        out = {
            "metric": METRIC, "value": round(value, 1), "unit": "profiles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "deterministic: the 4096 consecutive primes ending at 4294967291 (rank k: the next 4096 below)",
            "config": {"workload": "top block: 4096 consecutive primes ending at 4294967291, all admissible r, "
                                   "anchor filter + A4", "primes": len(primes), "profiles": nprof,
                       "parallelism": f"replicas x{world} (independent blocks)",
                       "l2": "flushed between timed steps (256 MiB write)"},
            "e2e": {"value": round(e2e_value, 1), "unit": "profiles/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_total / args.steps, 3)},
            "roofline": roof,
            "plain": {"value": round(plain_prof / (plain_ms / 1000.0), 1), "unit": "profiles/s",
                      "form": "one prime per call (device time)", "sample_primes": len(plain_ps),
                      "batched_over_plain": round(value / world / (plain_prof / (plain_ms / 1000.0)), 2)},
            "published_reference": {"value": 3063, "unit": "profiles/s", "hardware": "RTX 5090 (sm_120)",
                                    "window": "1024 primes from 4.237e9 (paper/GPU_METHOD_EN.tex:848)"},
            "clocks": clk, "gpu_launches": launches_per_step * args.steps,
            "stats": {"words": kstats["words"], "completions": kstats["completions"]},
        }
        if world == 1 and not args.no_cpu_baseline:
            why = reference_available()
            if why:
                out["cpu_baseline"] = {"value": None, "unavailable": why}
            else:
                cores = os.cpu_count() or 1
                jobs, sp, nref = reference_jobs(primes)
                secs, _ = run_reference_step(jobs, sp, cores)
                out["cpu_baseline"] = {"value": round(nref / secs, 2), "unit": "profiles/s", "cores": cores,
                                       "kind": "reference", "sample": reference_sample_text(jobs, sp, nref)}
        if world == 1 and not args.quick:
            # C4 and C5 on the same GPU, each with its own clock record
            ck = ClockSampler(local)
            ck.start()
            c4 = c4_measure(eng, steps=2, warmup=1)
            c4["clocks"] = ck.stop()
            out["c4"] = c4
            ck = ClockSampler(local)
            ck.start()
            c2 = c2_measure(eng, steps=2, warmup=1)
            c2["clocks"] = ck.stop()
            out["c2"] = c2
            from rabung_atlas32_b200 import serving
            ck = ClockSampler(local)
            ck.start()
            c5 = serving.benchmark(requests=args.requests, rate=args.rate, seed=20261203,
                                   plain_requests=min(args.requests, 2000))
            c5["clocks"] = ck.stop()
            out["c5"] = c5
        print(json.dumps(out), flush=True)
    if dist:
        barrier()
        dist.destroy_process_group()
    eng.close()


if __name__ == "__main__":
    main()
