#!/usr/bin/env python3
"""Generate the committed golden fixtures from the read-only reference tree.

Run once in a container that has the reference mounted, after
`make -f oracle/Makefile.ref REF=<reference>`:

    python tests/golden/make_golden.py --ref <reference checkout>

Writes into tests/golden/:
  scan-00000.vdw, quadruplets-00000.a4, scan-49900.vdw, quadruplets-49900.a4,
  manifest.json      -- the reference's shipped sample blocks (data/sample/),
                        copied byte for byte: encoder and decoder are checked
                        against these exact bytes.
  holdout32.json.gz  -- reproducibility/gpu_method/throughput/
                        holdout-32-mr_selected.json windows[*].profiles_full,
                        compacted to [p, [[r, M, L, K, w], ...]].
  dense_oracle.json.gz -- the reference GPU dense-oracle records of
                        reproducibility/gpu_method/night/ORACLES_NOUVEAUX.json
                        and throughput/CONTROLES_INDEPENDANTS.json (p < 2^32).
  refcpu_top_block.json.gz -- outputs of the reference's own CPU programs
                        (oracle/_ref) on the 4096 primes ending at 4294967291:
                        moment_worker A4 for all of them and, for EVERY
                        admissible (p, r) of the 1783 primes below block 49900
                        (block 49900's own frame pins the other 2313), the
                        reference's sparse CPU engines: `target p c f 64 1 8192 1`
                        for the coupled pairs {2, 4} and {3, 6}, `advance
                        adaptive p r 64 3 1` for every other order.
  refcpu_2p24.json.gz -- `independent p r 3` (full-walk reference) on a seeded
                        sample of (p, r) pairs from the 4096 primes from 2^24,
                        and moment_worker A4 for all 4096 of them.
  wide33.json.gz     -- the 33-bit domain: reproducibility/gpu_method/throughput/
                        holdout-33-mr_selected.json windows[*].profiles_full
                        (2 x 1024 primes between 2^32 and 2^33), the reference
                        GPU dense-oracle records with 2^32 <= p < 2^33, and A4
                        of every holdout prime by the reference's point counter
                        (src/census/theorie/elliptic4_mestre.cpp, `elliptic4`).

`--parts wide` regenerates only wide33.json.gz.
"""
from __future__ import annotations

import argparse
import gzip
import json
import random
import shutil
import struct
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
import oracle  # noqa: E402  (checker, used here only to list primes)


def dump(name, obj):
    """gzip'd compact JSON, byte-reproducible (no timestamp in the header)."""
    raw = json.dumps(obj, separators=(",", ":")).encode()
    (HERE / name).write_bytes(gzip.compress(raw, mtime=0))


def consecutive_primes_from(start, n):
    out, x = [], start
    while len(out) < n:
        if oracle.is_prime(x):
            out.append(x)
        x += 1
    return out


def consecutive_primes_ending(top, n):
    out, x = [], top
    while len(out) < n:
        if oracle.is_prime(x):
            out.append(x)
        x -= 1
    return out[::-1]


def moment_worker(ref_bin, primes):
    vals = []
    for i in range(0, len(primes), 4096):
        chunk = primes[i:i + 4096]
        line = f"0 -1 {len(chunk)} " + " ".join(map(str, chunk)) + "\nQUIT\n"
        out = subprocess.run([str(ref_bin / "moment_worker")], input=line.encode(),
                             capture_output=True, check=True).stdout
        j = out.index(b"A4BATCH1")
        hdr = out[j:j + 8 + 8 + 4 + 4 + 8 + 8 + 4 + 4 + 8 + 8]
        n = struct.unpack_from("<I", hdr, 16)[0]
        body = out[j + len(hdr): j + len(hdr) + 4 * n]
        vals += list(struct.unpack("<" + "I" * n, body))
    return vals


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="checkout of the reference repository")
    ap.add_argument("--samples", type=int, default=48, help="(p, r) pairs of the 2^24 block for `independent`")
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--parts", default="all", choices=["all", "wide"])
    a = ap.parse_args()
    ref = Path(a.ref)
    ref_bin = REPO / "oracle" / "_ref"
    gm = ref / "reproducibility" / "gpu_method"

    # 33-bit domain
    hold = json.loads((gm / "throughput" / "holdout-33-mr_selected.json").read_text())
    wins = []
    for w in hold["windows"]:
        rows = [[row["p"], [[v["r"], v["max"], v["prefix"], v["K"], v["witness"]] for v in row["profiles"]]]
                for row in w["profiles_full"]]
        wins.append({"lo": w["lo"], "hi": w["hi"], "rows": rows})
    wide = {}
    for rec in json.loads((gm / "night" / "ORACLES_NOUVEAUX.json").read_text()):
        if 2 ** 32 <= rec["p"] < 2 ** 33 and rec.get("status") == "PASS":
            wide[rec["p"]] = rec["profiles"]
    for res in json.loads((gm / "throughput" / "CONTROLES_INDEPENDANTS.json").read_text())["results"]:
        rec = res.get("oracle", {}).get("record", {})
        if 2 ** 32 <= rec.get("p", 0) < 2 ** 33 and rec.get("status") == "PASS":
            wide[rec["p"]] = rec["profiles"]
    hp = sorted({row[0] for w in wins for row in w["rows"]})
    a4w = {}
    for i in range(0, len(hp), 256):
        out = subprocess.run([str(ref_bin / "elliptic4"), *map(str, hp[i:i + 256])], capture_output=True,
                             check=True, text=True).stdout
        for line in out.splitlines():
            j = json.loads(line)
            assert j["status"] == "PASS"
            a4w[str(j["p"])] = j["quadruples"]
    dump("wide33.json.gz", {"holdout": wins, "a4": a4w,
                            "dense_oracle": [[p, [[v["r"], v["max"], v["prefix"], v["K"], v["witness"]] for v in prof]]
                                             for p, prof in sorted(wide.items())]})
    if a.parts == "wide":
        print("wide33.json.gz written to", HERE)
        return

    for f in ["scan-00000.vdw", "quadruplets-00000.a4", "scan-49900.vdw",
              "quadruplets-49900.a4", "manifest.json"]:
        shutil.copyfile(ref / "data" / "sample" / f, HERE / f)

    hold = json.loads((gm / "throughput" / "holdout-32-mr_selected.json").read_text())
    windows = []
    for w in hold["windows"]:
        rows = [[row["p"], [[v["r"], v["max"], v["prefix"], v["K"], v["witness"]] for v in row["profiles"]]]
                for row in w["profiles_full"]]
        windows.append({"lo": w["lo"], "hi": w["hi"], "rows": rows})
    dump("holdout32.json.gz", windows)

    recs = {}
    for rec in json.loads((gm / "night" / "ORACLES_NOUVEAUX.json").read_text()):
        if rec["p"] < 2 ** 32 and rec.get("status") == "PASS":
            recs[rec["p"]] = rec["profiles"]
    for res in json.loads((gm / "throughput" / "CONTROLES_INDEPENDANTS.json").read_text())["results"]:
        rec = res.get("oracle", {}).get("record", {})
        if rec.get("p", 2 ** 40) < 2 ** 32 and rec.get("status") == "PASS":
            recs[rec["p"]] = rec["profiles"]
    dump("dense_oracle.json.gz", [[p, [[v["r"], v["max"], v["prefix"], v["K"], v["witness"]] for v in prof]]
                                  for p, prof in sorted(recs.items())])

    rng = random.Random(20261203)

    # top block: 4096 primes ending at 4294967291
    top = consecutive_primes_ending(4294967291, 4096)
    a4_top = moment_worker(ref_bin, top)
    below = [p for p in top if p < 4294915433]
    jobs = []
    for p in below:
        rs = [r for r in range(2, 10) if (p - 1) % r == 0]
        for c, f in ((2, 4), (3, 6)):
            if c in rs and f in rs:
                jobs.append(("target", p, c, f))
                rs = [r for r in rs if r not in (c, f)]
        jobs += [("advance", p, r, 0) for r in rs]

    def run_job(job):
        kind, p, r, f = job
        if kind == "target":
            out = subprocess.run([str(ref_bin / "target"), str(p), str(r), str(f), "64", "1", "8192", "1"],
                                 capture_output=True, check=True, text=True).stdout
            j = json.loads(out)
            assert j["status"] == "PASS", (p, r, f)
            return [[p, r, j["coarse_maximum"], j["coarse_prefix"], j["coarse_witness"]],
                    [p, f, j["fine_maximum"], j["fine_prefix"], j["fine_witness"]]]
        out = subprocess.run([str(ref_bin / "advance"), "adaptive", str(p), str(r), "64", "3", "1"],
                             capture_output=True, check=True, text=True).stdout
        j = json.loads(out)
        assert j["status"] == "PASS", (p, r)
        return [[p, r, j["maximum"], j["prefix"], j["witness"]]]

    with ThreadPoolExecutor(a.jobs) as ex:
        res = list(ex.map(run_job, jobs))
    adv = sorted(v for part, job in zip(res, jobs) if job[0] == "advance" for v in part)
    tgt = sorted(v for part, job in zip(res, jobs) if job[0] == "target" for v in part)
    dump("refcpu_top_block.json.gz", {"primes": top, "a4": a4_top, "advance": adv, "target": tgt})

    # 2^24 block
    low = consecutive_primes_from(2 ** 24, 4096)
    a4_low = moment_worker(ref_bin, low)
    pairs = []
    while len(pairs) < a.samples:
        p = rng.choice(low)
        rs = [r for r in range(2, 10) if (p - 1) % r == 0]
        pairs.append((p, rng.choice(rs)))

    def run_ind(pr):
        p, r = pr
        out = subprocess.run([str(ref_bin / "independent"), str(p), str(r), "3"],
                             capture_output=True, text=True).stdout
        j = json.loads(out)
        return [p, r, j["M"], j["L"], j["w"]]

    with ThreadPoolExecutor(8) as ex:
        ind = list(ex.map(run_ind, pairs))
    dump("refcpu_2p24.json.gz", {"primes": low, "a4": a4_low, "independent": ind})
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
