"""Autotuner for the census engine; its choices persist per device.

    python -m rabung_atlas32_b200.autotune [--quick]

Searches, by coordinate descent from the defaults, the knobs that set how the
work is cut and scheduled:
  * anchor filter: anchor length policy (anchor_bits, then stages per order
    r, anchor_t), cover window cap and speculation margin per order r, CTAs per profile
    (cta_per_profile: CTAs sharing one profile's work items), rows per
    threshold epoch (epoch_rows),
    cover shape (cover_n: table radius vs rows), on a sample of the block below
    2^32;
  * dense scan: segment length (dense_steps, x per warp task), on primes near
    2^22;
  * routing: the dense/sparse crossover p (sparse_min_p).
Every trial's records must be bit-identical to the defaults' records (a trial
that differs is discarded and reported).  The winner is written to
rabung_atlas32_b200/tuned/<device>.json; Census() loads it for that device.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import re
import time
from pathlib import Path

from . import sieve
from .census import Census, Tuning

TUNED = Path(__file__).resolve().parent / "tuned"


def device_key(eng: Census) -> str:
    import ctypes
    buf = ctypes.create_string_buffer(128)
    sms = ctypes.c_uint32()
    if eng.lib.cz_device_info(eng.h, buf, 128, ctypes.byref(sms)) != 0:
        return "unknown"
    name = re.sub(r"[^A-Za-z0-9]+", "-", buf.value.decode()).strip("-").lower()
    return f"{name}-{sms.value}sm"


def load_tuned(key: str) -> Tuning | None:
    f = TUNED / f"{key}.json"
    if not f.exists():
        return None
    d = json.loads(f.read_text())["tuning"]
    fields = {k: (tuple(v) if isinstance(v, list) else v) for k, v in d.items() if k in Tuning.__dataclass_fields__}
    return Tuning(**fields)


def _measure(t: Tuning, primes, mode: str, reps: int = 2):
    with Census(tuning=t, autoload=False) as c:
        c.raw(primes, mode=mode, a4=False)                    # warm
        best, recs = 1e30, None
        for _ in range(reps):
            out, _, st = c.raw(primes, mode=mode, a4=False)
            ms = st["ms_device"] + st["ms_respec"]
            best = min(best, ms)
            n = c.count_profiles(primes)
            recs = [(o.p, o.r, o.M, o.L, o.witness) for o in out[:n]]
        return best, recs


def anchor_pref(r: int, bits: int) -> int:
    """Stages the filter derives from anchor_bits: least t with r^(t-1) >= 2^(5+bits)."""
    if r < 2:
        raise ValueError(f"order r = {r} has no anchor stages")
    k, pw = 0, 1
    while pw < 1 << (5 + bits):
        pw *= r
        k += 1
    return k + 1


def tune(quick: bool = False, log=print) -> dict:
    base = Tuning()
    top = sieve.primes_ending(4294967291, 512 if quick else 1024)
    ref_ms, ref = _measure(base, top, "sparse")
    log(f"baseline sparse {ref_ms:.1f} ms")
    best = dataclasses.replace(base)
    best_ms = ref_ms
    space = {"anchor_bits": [3, 4, 5], "cta_per_profile": [1, 2, 3, 4], "epoch_rows": [256, 512, 1024, 2048],
             "cover_n": [3, 4]}
    rejected = []
    for _ in range(1 if quick else 2):
        for knob, values in space.items():
            for v in values:
                if getattr(best, knob) == v:
                    continue
                t = dataclasses.replace(best, **{knob: v})
                ms, recs = _measure(t, top, "sparse")
                if recs != ref:
                    rejected.append({knob: v})
                    continue
                log(f"  {knob}={v}: {ms:.1f} ms")
                if ms < best_ms * 0.99:
                    best, best_ms = t, ms
    # anchor stages per order r, one step either side of the current choice
    for r in range(2, 10):
        cur = best.anchor_t[r] or anchor_pref(r, best.anchor_bits)
        for v in (cur - 1, cur + 1):
            if not 2 <= v <= 32:
                continue
            at = list(best.anchor_t)
            at[r] = v
            t = dataclasses.replace(best, anchor_t=tuple(at))
            ms, recs = _measure(t, top, "sparse")
            if recs != ref:
                rejected.append({"anchor_t": r, "t": v})
                continue
            log(f"  anchor_t[{r}]={v}: {ms:.1f} ms")
            if ms < best_ms * 0.995:
                best, best_ms = t, ms
    # cover window cap per order r: q never exceeds it, and the largest cap of
    # a prime's orders sets its table radius
    for r in range(2, 10):
        cur = best.q_cap[r]
        for v in (cur - 4, cur - 2, cur + 2):
            if not 3 <= v <= 255:
                continue
            qc = list(best.q_cap)
            qc[r] = v
            t = dataclasses.replace(best, q_cap=tuple(qc))
            ms, recs = _measure(t, top, "sparse")
            if recs != ref:
                rejected.append({"q_cap": r, "Q": v})
                continue
            log(f"  q_cap[{r}]={v}: {ms:.1f} ms")
            if ms < best_ms * 0.995:
                best, best_ms = t, ms
    # speculation margin per order r (tenths); the measured time includes the
    # re-runs of the primes whose best run stayed below the threshold
    for r in range(2, 10):
        cur = best.spec_margin10[r]
        for v in (cur - 10, cur - 5, cur + 5, cur + 10):
            if not 0 <= v <= 60:
                continue
            sm = list(best.spec_margin10)
            sm[r] = v
            t = dataclasses.replace(best, spec_margin10=tuple(sm))
            ms, recs = _measure(t, top, "sparse")
            if recs != ref:
                rejected.append({"spec_margin10": r, "margin": v})
                continue
            log(f"  spec_margin10[{r}]={v}: {ms:.1f} ms")
            if ms < best_ms * 0.995:
                best, best_ms = t, ms
    # dense segment length near 2^22
    mid = sieve.primes_from(1 << 22, 128 if quick else 256)
    dref_ms, dref = _measure(best, mid, "dense")
    for steps in (64, 128, 512, 1024):
        t = dataclasses.replace(best, dense_steps=steps)
        ms, recs = _measure(t, mid, "dense")
        if recs != dref:
            rejected.append({"dense_steps": steps})
            continue
        log(f"  dense_steps={steps}: {ms:.1f} ms (ref {dref_ms:.1f})")
        if ms < dref_ms * 0.99:
            best, dref_ms = t, ms
    # dense/sparse crossover: least p at which the sparse path is faster
    cross = None
    for e in (14, 16, 18, 20, 22):
        ps = sieve.primes_from(1 << e, 256)
        d_ms, d_rec = _measure(best, ps, "dense", reps=1)
        try:
            s_ms, s_rec = _measure(dataclasses.replace(best, sparse_min_p=2), ps, "sparse", reps=1)
        except Exception as exc:                     # sparse path not certified this low
            log(f"  p=2^{e}: sparse unavailable ({exc})")
            continue
        if s_rec != d_rec:
            rejected.append({"crossover": e})
            continue
        log(f"  p=2^{e}: dense {d_ms:.1f} ms, sparse {s_ms:.1f} ms")
        if s_ms < d_ms and cross is None:
            cross = 1 << e
    if cross:
        best = dataclasses.replace(best, sparse_min_p=cross)
    return {"tuning": dataclasses.asdict(best), "measured": {"sparse_ms_sample": best_ms,
            "sparse_ms_default": ref_ms, "sample_primes": len(top)}, "rejected": rejected}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--no-save", action="store_true")
    a = ap.parse_args(argv)
    with Census(autoload=False) as c:
        key = device_key(c)
    t0 = time.time()
    res = tune(quick=a.quick)
    res["device"] = key
    res["seconds"] = round(time.time() - t0, 1)
    print(json.dumps(res))
    if not a.no_save:
        TUNED.mkdir(exist_ok=True)
        (TUNED / f"{key}.json").write_text(json.dumps(res, indent=1) + "\n")


if __name__ == "__main__":
    main()
