import gzip
import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long CPU-only case")


def load_gz(name):
    with gzip.open(GOLDEN / name, "rt") as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden():
    from rabung_atlas32_b200 import codec
    out = {}
    for blk in ("00000", "49900"):
        recs, meta = codec.decode_scan_frame((GOLDEN / f"scan-{blk}.vdw").read_bytes())
        vals, ameta = codec.decode_a4_frame((GOLDEN / f"quadruplets-{blk}.a4").read_bytes())
        for rec, a in zip(recs, vals):
            rec.a4 = a
        out[blk] = (recs, meta, ameta)
    return out
