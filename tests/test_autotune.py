"""Autotuner search logic on CPU: the GPU measurement is replaced by a
deterministic cost model, so the coordinate descent over the global knobs and
the per-order steps (anchor stages, cover caps, speculation margins) can be
checked without a device -- each step must move toward the model's optimum and
keep to the allowed ranges, and a trial whose records differ from the
defaults' must be rejected, never adopted."""
import dataclasses

from rabung_atlas32_b200 import autotune
from rabung_atlas32_b200.census import Tuning

RECORDS = [(101, 2, 7, 1, 19)]


def fake_measure(t: Tuning, primes, mode: str, reps: int = 2):
    eff = [0, 0] + [t.anchor_t[r] or autotune.anchor_pref(r, t.anchor_bits) for r in range(2, 10)]
    if mode == "dense":
        return 100.0 + abs(t.dense_steps - 512) / 64.0, RECORDS
    ms = 1000.0
    ms += 30.0 * abs(eff[2] - 13)              # optimum two stages above the default
    ms += 20.0 * abs(t.q_cap[2] - 22)           # optimum below the default cap
    ms += 15.0 * abs(t.spec_margin10[7] - 10)   # optimum above the default margin
    ms += 10.0 * abs(t.cta_per_profile - 2)
    recs = RECORDS
    if eff[3] == 8:                             # a planted record change: must be rejected
        recs = [(101, 2, 8, 1, 19)]
        ms -= 500.0
    if t.sparse_min_p == 2 and mode == "sparse":
        ms = 50.0                               # sparse faster than dense at every crossover probe
    return ms, recs


def test_per_order_steps_descend_and_reject_changed_records(monkeypatch):
    monkeypatch.setattr(autotune, "_measure", fake_measure)
    res = autotune.tune(quick=True, log=lambda s: None)
    t = Tuning(**{k: (tuple(v) if isinstance(v, list) else v) for k, v in res["tuning"].items()})
    base = Tuning()
    eff2 = t.anchor_t[2] or autotune.anchor_pref(2, t.anchor_bits)
    assert eff2 == (base.anchor_t[2] or autotune.anchor_pref(2, base.anchor_bits)) + 1   # one step toward 13
    assert t.q_cap[2] == base.q_cap[2] - 4                                                 # largest step down
    assert t.spec_margin10[7] == base.spec_margin10[7] + 10
    assert (t.anchor_t[3] or autotune.anchor_pref(3, t.anchor_bits)) != 8                   # never adopted
    assert {"anchor_t": 3, "t": 8} in res["rejected"]
    assert all(2 <= v <= 32 for v in t.anchor_t if v) and all(3 <= v <= 255 for v in t.q_cap[2:])
    assert all(0 <= v <= 60 for v in t.spec_margin10)
    assert t.dense_steps == 512 and t.sparse_min_p == 1 << 14
    assert res["measured"]["sparse_ms_sample"] < res["measured"]["sparse_ms_default"]


def test_no_change_when_defaults_are_optimal(monkeypatch):
    base = Tuning()

    def flat(t, primes, mode, reps=2):
        d = dataclasses.asdict(t)
        ms = 100.0 + sum(1.0 for k, v in d.items() if v != dataclasses.asdict(base)[k] and k != "sparse_min_p")
        return ms, RECORDS
    monkeypatch.setattr(autotune, "_measure", flat)
    res = autotune.tune(quick=True, log=lambda s: None)
    got = {k: v for k, v in res["tuning"].items() if k != "sparse_min_p"}
    want = {k: (list(v) if isinstance(v, tuple) else v) for k, v in dataclasses.asdict(base).items()
            if k != "sparse_min_p"}
    assert {k: (list(v) if isinstance(v, tuple) else v) for k, v in got.items()} == want
