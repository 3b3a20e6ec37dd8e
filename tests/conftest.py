import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def golden():
    return {
        "kat": json.loads((GOLDEN / "poseidon2_kat.json").read_text()),
        "two_adic": json.loads((GOLDEN / "two_adic.json").read_text()),
        "vectors": json.loads((GOLDEN / "oracle_vectors.json").read_text()),
    }


@pytest.fixture(scope="session")
def orc():
    from oracle import cpu

    cpu.load()
    return cpu


@pytest.fixture(scope="session")
def gpu():
    """Session-wide device context.  No fallback: a missing device or library is an error."""
    from pico_b200 import GpuContext

    ctx = GpuContext(0)
    yield ctx
    ctx.close()
