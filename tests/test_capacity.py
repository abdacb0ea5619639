"""Capacity rules of the 4-cycle and 4-clique kernels (gary_b200/csrc/
pattern_rules.cuh), checked on the host by tests/cpp/capacity_test.cu: every
4-clique out-degree the API admits and adversarial 4-cycle neighbourhoods
(equal-degree stars around each class boundary) keep every shared table at
most half full, every counter within its width and every row buffer large
enough.  The plans classify vertices with the same functions."""
from __future__ import annotations

import subprocess
from pathlib import Path

CPP = Path(__file__).resolve().parent / "cpp"


def test_capacity_rules_hold():
    subprocess.run(["make", "-s", "-C", str(CPP), "_bin/capacity_test"], check=True)
    r = subprocess.run([str(CPP / "_bin" / "capacity_test")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failed" in r.stdout
