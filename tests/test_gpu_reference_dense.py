"""The reference's own GPU dense oracle (src/census/dense_oracle.cu, built
unchanged for sm_100a into oracle/_ref by oracle/Makefile.ref) run beside
this library's dense kernel on the same B200 and the same primes: records
identical, both device times printed (pytest -s shows them)."""
import json
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "dense_oracle"


@pytest.mark.skipif(not BIN.exists(), reason="oracle/_ref/dense_oracle not built")
@pytest.mark.parametrize("p", [16777259, 4237000003, 4294964521])
def test_reference_dense_oracle_same_box(p):
    from rabung_atlas32_b200.census import Census
    out = subprocess.run([str(BIN), "--prime", str(p)], capture_output=True, text=True, check=True).stdout
    ref = json.loads(out)
    assert ref["status"] == "PASS"
    with Census() as c:
        c.raw([p], mode="dense", a4=False)                 # warm
        recs, _, st = c.raw([p], mode="dense", a4=False, verify=True)
        n = c.count_profiles([p])
        mine = [(v.r, v.M, v.L, v.K, v.witness) for v in recs[:n]]
    assert mine == [(v["r"], v["max"], v["prefix"], v["K"], v["witness"]) for v in ref["profiles"]]
    print(json.dumps({"p": p, "reference_dense_oracle_gpu_ms": round(ref["gpu_ms"], 3),
                      "dense_scan_and_merge_ms": round(st["ms_dense"], 3)}))
