"""bench.py's host-side contract helpers, on the CPU: the stored ncu counters
apply only to the kernel sources they were captured on, every stored record
names a workload the bench prints, and the pattern lines' roofline is built
from those counters over the line's own time.  No GPU needed.

The first test holds the committed counters to the committed kernels: after a
kernel change, capture them again (the commands are in each record's profile)
before committing."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402

PROFILES = ROOT / "profiles" / "roofline_traffic.json"


def _sources_of(workload: str):
    return bench.PATTERN_SOURCES if ("cycle" in workload or "clique" in workload) else bench.KERNEL_SOURCES


def test_every_stored_record_is_fresh_and_complete():
    recs = json.loads(PROFILES.read_text())
    assert recs, "no stored counters"
    for workload, rec in recs.items():
        for key in ("dram_bytes", "warp_inst", "kernel_src", "profile"):
            assert key in rec, (workload, key)
        assert (ROOT / rec["profile"]).exists(), rec["profile"]
        got = bench.measured_counters(workload, _sources_of(workload))
        assert got is not None and got["stale"] is False, f"{workload}: counters captured on other sources"


def test_stored_workloads_are_the_ones_the_bench_prints():
    recs = json.loads(PROFILES.read_text())
    tri = {f"triangle count, RMAT scale {s} edge factor {e}, seed 1" for s, e in ((24, 32), (22, 16))}
    pat = {f"{p} count, RMAT scale {s} edge factor {e}, seed 1"
           for p in ("4-cycle", "4-clique") for s, e in ((24, 32), (22, 16))}
    assert set(recs) == tri | pat


def test_a_source_change_marks_counters_stale(tmp_path, monkeypatch):
    recs = json.loads(PROFILES.read_text())
    workload = "triangle count, RMAT scale 24 edge factor 32, seed 1"
    rec = dict(recs[workload])
    rec["kernel_src"] = "0" * 16  # as if captured on other sources
    f = tmp_path / "profiles" / "roofline_traffic.json"
    f.parent.mkdir()
    f.write_text(json.dumps({workload: rec}))
    csrc = tmp_path / "gary_b200" / "csrc"
    csrc.mkdir(parents=True)
    for name in set(bench.KERNEL_SOURCES) | set(bench.PATTERN_SOURCES):
        (csrc / name).write_bytes((ROOT / "gary_b200" / "csrc" / name).read_bytes())
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.measured_counters(workload)["stale"] is True
    rec["kernel_src"] = bench.kernel_source_hash()
    f.write_text(json.dumps({workload: rec}))
    assert bench.measured_counters(workload)["stale"] is False
    (csrc / "tc.cu").write_bytes((csrc / "tc.cu").read_bytes() + b"\n")
    assert bench.measured_counters(workload)["stale"] is True
    assert bench.measured_counters("no such workload") is None


def test_pattern_roofline_from_counters(monkeypatch):
    monkeypatch.setattr(bench, "sm_count", lambda: 148)
    workload = "4-clique count, RMAT scale 24 edge factor 32, seed 1"
    rec = json.loads(PROFILES.read_text())[workload]
    ms = 3000.0
    r = bench.pattern_roofline(workload, ms)
    hbm, _ = bench.peak_hbm()
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["stale"] is False
    assert r["traffic"] == rec["dram_bytes"]
    assert r["achieved"] == pytest.approx(rec["dram_bytes"] / (ms / 1e3) / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / hbm)
    assert r["issue"]["frac"] == pytest.approx(rec["warp_inst"] / (ms / 1e3) / (148 * 4 * 1965e6))
    assert len(r["kernels"]) == 4  # the 4-clique call's four kernels
    assert bench.pattern_roofline("no such workload", ms) is None


def test_balance_of():
    assert bench.balance_of({"makespan_ms": 10.0, "mean_cta_finish_ms": 8.0})["schedule_bound"] == 1.25
    assert bench.balance_of({})["schedule_bound"] is None
