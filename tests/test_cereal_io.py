"""Graph binaries in the reference's layout (GraphCSR / GraphCOO through
cereal's binary archive, include/Graph.h:132-148, 269-285, 300-316).

No file written by the reference ships with it, so the fixtures here are
packed byte by byte from the layout rules (struct.pack, independent of the
library's writer): version, format tag, m, nnz, then every array as a new
shared pointer id 0x8000000k, a uint64 count and the elements.  Host only:
no GPU needed."""
from __future__ import annotations

import struct

import numpy as np
import pytest

import gary_b200 as gb
from oracle import oracle as O


def _vec(k: int, arr: np.ndarray, fmt: str) -> bytes:
    return struct.pack("<IQ", 0x80000000 | k, len(arr)) + np.asarray(arr).astype(fmt).tobytes()


def _csr_bytes(ptr, idx, version=1, fmt_tag=0, deg=None, ids=(1, 2, 3)) -> bytes:
    ptr = np.asarray(ptr, np.int64)
    idx = np.asarray(idx, np.int32)
    m = len(ptr) - 1
    deg = np.diff(ptr).astype(np.int32) if deg is None else np.asarray(deg, np.int32)
    out = struct.pack("<IIiq", version, fmt_tag, m, int(ptr[-1]))
    out += _vec(ids[0], ptr, "<i8") + _vec(ids[1], idx, "<i4") + _vec(ids[2], deg, "<i4")
    return out


def _graph(seed=2):
    s, d = gb.gen_er(300, 2000, seed)
    ptr, idx = O.sym_csr(s, d, 300)
    return O.orient(ptr, idx, by_degree=False)  # the reference's csr_dag: id-oriented


def test_read_packed_csr(tmp_path):
    ptr, idx = _graph()
    f = tmp_path / "csr_dag.bin"
    f.write_bytes(_csr_bytes(ptr, idx))
    assert gb.bin_info(f) == (gb.GARY_BIN_CSR, 300, len(idx))
    p2, i2 = gb.read_bin_csr(f)
    assert np.array_equal(p2, ptr) and np.array_equal(i2, idx)


def test_write_matches_layout_and_roundtrips(tmp_path):
    ptr, idx = _graph(5)
    f = tmp_path / "out.bin"
    gb.write_bin_csr(f, ptr, idx)
    assert f.read_bytes() == _csr_bytes(ptr, idx)
    p2, i2 = gb.read_bin_csr(f)
    assert np.array_equal(p2, ptr) and np.array_equal(i2, idx)


def test_read_packed_coo(tmp_path):
    rng = np.random.default_rng(1)
    row = rng.integers(0, 50, 400).astype(np.int32)
    col = rng.integers(0, 50, 400).astype(np.int32)
    data = struct.pack("<IIiq", 1, 1, 50, 400) + _vec(1, row, "<i4") + _vec(2, col, "<i4")
    f = tmp_path / "coo.bin"
    f.write_bytes(data)
    assert gb.bin_info(f) == (gb.GARY_BIN_COO, 50, 400)
    n, s, d = gb.read_bin_coo(f)
    assert n == 50 and np.array_equal(s, row) and np.array_equal(d, col)
    with pytest.raises(gb.GaryError):
        gb.read_bin_csr(f)


def test_committed_fixture():
    """The committed fixture (tests/golden/make_cereal_fixture.py, written from
    cereal's binary rules with the standard library only) reads back as the
    graph it was made from, and writing that graph gives the same bytes."""
    import json
    from pathlib import Path

    g = Path(__file__).parent / "golden"
    want = json.loads((g / "cereal_csr_dag.json").read_text())
    f = g / "cereal_csr_dag.bin"
    assert gb.bin_info(f) == (gb.GARY_BIN_CSR, want["n"], len(want["indices"]))
    p, i = gb.read_bin_csr(f)
    assert p.tolist() == want["indptr"] and i.tolist() == want["indices"]
    assert _csr_bytes(p, i) == f.read_bytes()


def test_empty_graph(tmp_path):
    f = tmp_path / "empty.bin"
    f.write_bytes(_csr_bytes(np.zeros(4, np.int64), np.zeros(0, np.int32)))
    p, i = gb.read_bin_csr(f)
    assert p.tolist() == [0, 0, 0, 0] and len(i) == 0


@pytest.mark.parametrize("case", ["version", "format", "truncated", "pointer_id", "counts", "missing"])
def test_malformed_files_are_rejected(tmp_path, case):
    ptr, idx = _graph(7)
    good = _csr_bytes(ptr, idx)
    data = {
        "version": _csr_bytes(ptr, idx, version=2),
        "format": _csr_bytes(ptr, idx, fmt_tag=7),
        "truncated": good[: len(good) - 9],
        "pointer_id": _csr_bytes(ptr, idx, ids=(1, 1, 3)),
        "counts": _csr_bytes(ptr, idx, deg=np.zeros(5, np.int32)),
        "missing": None,
    }[case]
    f = tmp_path / "bad.bin"
    if data is not None:
        f.write_bytes(data)
    with pytest.raises(gb.GaryError) as e:
        gb.read_bin_csr(f)
    assert e.value.status in (-1, -4)
