"""pytest configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a CUDA device and the built libgary_b200.so; they fail
(never skip) when either is missing, because the CUDA library is the only
implementation of the path.  Everything else runs on the CPU.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "tests" / "golden"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")


@pytest.fixture(scope="session")
def golden():
    return json.loads((ROOT / "tests" / "golden" / "golden.json").read_text())


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")
