"""The line-protocol census worker speaks the reference's protocol
(src/census/worker32.cu:10-45) and reproduces block 49900's records."""
import json
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_worker_protocol_block49900(golden):
    recs, _, _ = golden["49900"]
    ps = [r.p for r in recs[:256]]
    lines = f"0 {' '.join(map(str, ps[:128]))}\n1 {' '.join(map(str, ps[128:]))}\nQUIT\n"
    out = subprocess.run([sys.executable, "-m", "rabung_atlas32_b200.worker"], input=lines, text=True,
                         capture_output=True, cwd=ROOT, timeout=300)
    assert out.returncode == 0, out.stderr
    msgs = [json.loads(l) for l in out.stdout.splitlines()]
    assert msgs[0] == {"type": "ready", "domain_bits": 32} and msgs[-1] == {"type": "bye"}
    meas = [m for m in msgs if m["type"] == "measurement"]
    done = [m for m in msgs if m["type"] == "batch_done"]
    assert [d["id"] for d in done] == [0, 1] and [d["count"] for d in done] == [128, 128]
    for m, r in zip(meas, recs[:256]):
        assert m["p"] == r.p and m["status"] == "PASS"
        assert [(v["r"], v["max"], v["prefix"], v["witness"]) for v in m["profiles"]] == \
               [(v.r, v.M, v.L, v.witness) for v in r.profiles]


def test_worker_refuses_out_of_sequence_batch():
    out = subprocess.run([sys.executable, "-m", "rabung_atlas32_b200.worker"], input="1 4294967291\n",
                         text=True, capture_output=True, cwd=ROOT, timeout=120)
    assert out.returncode == 2 and "VDW_CAMPAIGN_FAILURE" in out.stderr
