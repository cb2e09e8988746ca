import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def to_bytes(s: str) -> bytes:
    """Fixture strings: UTF-8 text (the reference's Rust &str inputs)."""
    return s.encode("utf-8")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "reference_kat.json"), encoding="utf-8") as f:
        return json.load(f)


@pytest.fixture(scope="session")
def parser():
    from oneline_b200 import GpuParser

    p = GpuParser(0)
    yield p
    p.close()
