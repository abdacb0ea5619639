"""Generate tests/golden/golden.json from the REFERENCE's own code.

    python tests/golden/make_golden.py      # needs oracle/_ref (built from the
                                            # reference tree by `make -C oracle ref`)

The reference ships no known-answer vectors, so the fixtures are outputs of
the reference itself, compiled in place by oracle/Makefile:
  - triangle counts: src/Graph.cpp's pipeline (symmetrize -> toCSR_ -> toCOO ->
    orientation -> toCSR_, as convert.cpp:19-78) and cpuTriCount
    (test/TriQueryTest.cu:17-37, accumulators widened to uint64);
  - search results: binary_search, build_cache and binary_search_2phase of
    include/ops/Search.cuh run on the host, as test/SearchTest.cu:235-257 does.
Inputs come from the seeded generators of gary_b200 (ER, RMAT) and from
tests/golden/vectors.py; each graph case stores an edge-list digest so the
tests can prove they regenerate the same input.
"""
from __future__ import annotations

import itertools
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))

import gary_b200 as gb  # noqa: E402  (generators only)
from oracle import oracle as O  # noqa: E402
from vectors import edge_checksum, pack_bits, search_case  # noqa: E402


def explicit_graphs():
    g = {}
    g["K5"] = (5, list(itertools.combinations(range(5), 2)))
    g["K8"] = (8, list(itertools.combinations(range(8), 2)))
    g["star16"] = (17, [(0, i) for i in range(1, 17)])
    g["cycle4"] = (4, [(0, 1), (1, 2), (2, 3), (3, 0)])
    g["triangle"] = (3, [(0, 1), (1, 2), (0, 2)])
    g["single_edge"] = (2, [(0, 1)])
    g["no_edges"] = (6, [])
    g["two_triangles_shared_edge"] = (4, [(0, 1), (1, 2), (0, 2), (1, 3), (2, 3)])
    g["wheel10"] = (11, [(0, i) for i in range(1, 11)] + [(i, i % 10 + 1) for i in range(1, 11)])
    # a 40-clique planted in a sparse ER background
    n = 2000
    s, d = gb.gen_er(n, 6000, 99)
    planted = list(itertools.combinations(range(100, 140), 2))
    edges = list(zip(s.tolist(), d.tolist())) + planted
    g["planted_clique40"] = (n, edges)
    return g


def ref_tri(n, src, dst):
    """Reference pipeline on an undirected, deduplicated, loop-free edge list."""
    r = O.RefCSR.dag_from_edges(n, np.asarray(src, np.int32), np.asarray(dst, np.int32))
    ptr, idx = r.arrays()
    t = r.tri_count()
    r.free()
    return t, int(ptr[-1])


def graph_case(name, n, src, dst, extra):
    ptr, idx = O.sym_csr(src, dst, n)  # dedup + loops dropped (the reference does not dedup)
    us, ud = O.unique_pairs(ptr, idx)
    t, dag_nnz = ref_tri(n, us, ud)
    return {
        "name": name,
        "n": n,
        "edges_in": int(len(src)),
        "edge_digest": edge_checksum(src, dst),
        "sym_nnz": int(len(idx)),
        "dag_nnz": dag_nnz,
        "ref_triangles": t,
        **extra,
    }


def main():
    out = {"source": "reference (hirayaku/Gary) compiled in place; see make_golden.py", "graphs": [], "search": []}
    for name, (n, edges) in explicit_graphs().items():
        e = np.array(edges, np.uint32).reshape(-1, 2)
        case = graph_case(name, n, e[:, 0], e[:, 1], {"gen": "explicit"})
        case["edges"] = [list(map(int, x)) for x in edges] if name != "planted_clique40" else None
        if name == "planted_clique40":
            case["gen"] = "er+clique"
            case["gen_args"] = {"n": n, "m": 6000, "seed": 99, "clique": [100, 140]}
        out["graphs"].append(case)
    for seed in (1, 2, 3):
        n, m = 16384, 131072
        s, d = gb.gen_er(n, m, seed)
        out["graphs"].append(graph_case(f"er_{n}_{m}_s{seed}", n, s, d,
                                        {"gen": "er", "gen_args": {"n": n, "m": m, "seed": seed}}))
    for seed in (5, 6):
        n, m = 3000, 60000
        s, d = gb.gen_er(n, m, seed)
        out["graphs"].append(graph_case(f"er_{n}_{m}_s{seed}", n, s, d,
                                        {"gen": "er", "gen_args": {"n": n, "m": m, "seed": seed}}))
    for scale, ef, seed in ((8, 16, 1), (10, 16, 2), (12, 16, 3), (14, 16, 4), (16, 16, 5), (12, 32, 7)):
        s, d = gb.gen_rmat(scale, seed, ef << scale)
        out["graphs"].append(graph_case(f"rmat{scale}_ef{ef}_s{seed}", 1 << scale, s, d,
                                        {"gen": "rmat", "gen_args": {"scale": scale, "ef": ef, "seed": seed}}))
    # search vectors (include/ops/Search.cuh via the reference's host templates)
    for seed, nl, nk, lo, hi, sk in ((0, 4096, 2048, 1 << 29, 1 << 30, True),
                                      (1, 4096, 2048, 1 << 29, 1 << 30, False),
                                      (2, 100, 500, 0, 200, True),
                                      (3, 31, 64, 0, 64, False),
                                      (4, 1, 8, 0, 4, True),
                                      (5, 70000, 4096, 1 << 26, 1 << 30, True),
                                      (6, 4096, 4096, 0, 8192, True),
                                      (7, 100000, 8192, 0, 150000, False)):
        lst, keys = search_case(seed, nl, nk, lo, hi, sk)
        f1, f2 = O.ref_search(lst, keys)
        out["search"].append({
            "seed": seed, "n_list": nl, "n_keys": nk, "lo": lo, "hi": hi, "sort_keys": sk,
            "found": pack_bits(f1), "found_2phase": pack_bits(f2),
            "cache32": O.ref_build_cache32(lst).tolist(),
        })
    path = Path(__file__).with_name("golden.json")
    path.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {path}: {len(out['graphs'])} graphs, {len(out['search'])} search cases")


if __name__ == "__main__":
    main()
