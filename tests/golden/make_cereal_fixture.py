"""Write tests/golden/cereal_csr_dag.bin and cereal_csr_dag.json: a small
id-oriented DAG (the reference's csr_dag) in the binary layout that the
reference's GraphCSR::save produces through cereal's BinaryOutputArchive
(include/Graph.h:132-148, 269-285).

The bytes follow cereal's published binary rules, restated here with the
standard library only (no gary_b200, no oracle), so the fixture does not
depend on the reader it checks:
- arithmetic members as their little-endian bytes, in declaration order of
  the archive call: the format version (uint32), the layout tag (uint32,
  0 = CSR), the vertex count m (int32) and the entry count nnz (int64);
- each std::shared_ptr<std::vector<T>> as cereal's pointer-tracking id
  (uint32, 0x80000000 | k for the k-th pointer the archive first meets, k from
  1), then the vector as its size (uint64) and its elements' bytes: the
  offsets (int64, m + 1), the column ids (int32, nnz), the out-degrees
  (int32, m).

The graph: vertices 0..39 on a ring with chords i -> i + 5 and i -> i + 11
(mod 40) plus the 4-clique {0, 1, 2, 3}; every edge kept once with the larger
id first, as convert.cpp writes csr_dag (row u lists its neighbours v < u,
ascending).  Run: python tests/golden/make_cereal_fixture.py
"""
from __future__ import annotations

import json
import struct
from pathlib import Path

HERE = Path(__file__).resolve().parent


def edges(n: int = 40) -> list[tuple[int, int]]:
    e = set()
    for i in range(n):
        for step in (1, 5, 11):
            a, b = i, (i + step) % n
            e.add((max(a, b), min(a, b)))
    for a in range(4):
        for b in range(a):
            e.add((a, b))
    return sorted(e)


def csr_dag(n: int = 40):
    rows = [[] for _ in range(n)]
    for u, v in edges(n):
        rows[u].append(v)
    ptr = [0]
    idx = []
    for r in rows:
        idx.extend(sorted(r))
        ptr.append(len(idx))
    return ptr, idx


def vec(k: int, values: list[int], fmt: str) -> bytes:
    return struct.pack("<IQ", 0x80000000 | k, len(values)) + struct.pack(f"<{len(values)}{fmt}", *values)


def main() -> None:
    n = 40
    ptr, idx = csr_dag(n)
    deg = [ptr[i + 1] - ptr[i] for i in range(n)]
    data = struct.pack("<IIiq", 1, 0, n, len(idx)) + vec(1, ptr, "q") + vec(2, idx, "i") + vec(3, deg, "i")
    (HERE / "cereal_csr_dag.bin").write_bytes(data)
    (HERE / "cereal_csr_dag.json").write_text(json.dumps({"n": n, "indptr": ptr, "indices": idx}) + "\n")


if __name__ == "__main__":
    main()
