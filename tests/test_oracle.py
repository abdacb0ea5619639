"""The CPU oracle against the reference's golden vectors and closed-form
known answers (no GPU).  Pins the checker before anything is checked with it."""
from __future__ import annotations

import itertools
from math import comb

import numpy as np
import pytest

from graphs import edges_of
from oracle import oracle as O
from vectors import search_case, unpack_bits, splitmix

GRAPH_IDS = lambda g: g["name"]  # noqa: E731


def _cases(golden):
    return golden["graphs"]


def test_golden_graphs_triangles(golden):
    """orc_tri_count == the reference pipeline + cpuTriCount on every fixture,
    for both the reference's id orientation and the degree orientation."""
    for case in _cases(golden):
        n, src, dst = edges_of(case)
        ptr, idx = O.sym_csr(src, dst, n)
        assert len(idx) == case["sym_nnz"], case["name"]
        iptr, iidx = O.orient(ptr, idx, by_degree=False)
        assert int(iptr[-1]) == case["dag_nnz"], case["name"]
        dptr, didx = O.orient(ptr, idx, by_degree=True)
        assert int(dptr[-1]) == case["dag_nnz"], case["name"]
        assert O.tri_count(iptr, iidx) == case["ref_triangles"], case["name"]
        assert O.tri_count(dptr, didx) == case["ref_triangles"], case["name"]


def test_golden_search(golden):
    """binary_search / build_cache / binary_search_2phase restatements equal the
    reference's own host templates (include/ops/Search.cuh)."""
    for c in golden["search"]:
        lst, keys = search_case(c["seed"], c["n_list"], c["n_keys"], c["lo"], c["hi"], c["sort_keys"])
        lst32 = lst.astype(np.uint32)
        f1 = unpack_bits(c["found"], c["n_keys"])
        f2 = unpack_bits(c["found_2phase"], c["n_keys"])
        assert np.array_equal(O.binary_search(lst32, keys), f1)
        assert np.array_equal(O.binary_search_2phase(lst32, keys), f2)
        assert O.build_cache(lst32).tolist() == [x & 0xFFFFFFFF for x in c["cache32"]]
        # membership ground truth
        truth = np.isin(keys, lst).astype(np.uint8)
        assert np.array_equal(f1, truth)


@pytest.mark.parametrize("n", [4, 5, 7, 12])
def test_complete_graph_kats(n):
    e = np.array(list(itertools.combinations(range(n), 2)), np.uint32)
    ptr, idx = O.sym_csr(e[:, 0], e[:, 1], n)
    dptr, didx = O.orient(ptr, idx)
    assert O.tri_count(dptr, didx) == comb(n, 3)
    assert O.k4_count(dptr, didx) == comb(n, 4)
    assert O.c4_count(ptr, idx) == 3 * comb(n, 4)


def test_small_kats():
    def counts(n, edges):
        e = np.array(edges, np.uint32).reshape(-1, 2)
        ptr, idx = O.sym_csr(e[:, 0], e[:, 1], n)
        dptr, didx = O.orient(ptr, idx)
        return O.tri_count(dptr, didx), O.c4_count(ptr, idx), O.k4_count(dptr, didx)

    assert counts(17, [(0, i) for i in range(1, 17)]) == (0, 0, 0)          # star
    assert counts(4, [(0, 1), (1, 2), (2, 3), (3, 0)]) == (0, 1, 0)         # C4
    wheel = [(0, i) for i in range(1, 11)] + [(i, i % 10 + 1) for i in range(1, 11)]
    assert counts(11, wheel) == (10, 10, 0)
    assert counts(6, []) == (0, 0, 0)
    assert counts(2, [(0, 1)]) == (0, 0, 0)
    # duplicates and loops in the input do not change anything
    assert counts(3, [(0, 1), (1, 0), (1, 2), (2, 2), (0, 2), (0, 2)]) == (1, 0, 0)
    # K_{2,3}: C(3,2) 4-cycles
    assert counts(5, [(0, 2), (0, 3), (0, 4), (1, 2), (1, 3), (1, 4)]) == (0, 3, 0)


@pytest.mark.parametrize("leaves", [1000, 65535, 70000])
def test_two_hub_bipartite_c4(leaves):
    """K_{2,n} holds C(n,2) 4-cycles and nothing else; the GPU tests use the
    same graphs at the window kernel's counter-width limits."""
    n = leaves + 2
    a = np.arange(2, n, dtype=np.uint32)
    src = np.concatenate([np.zeros(leaves, np.uint32), np.ones(leaves, np.uint32)])
    dst = np.concatenate([a, a])
    ptr, idx = O.sym_csr(src, dst, n)
    dptr, didx = O.orient(ptr, idx)
    assert O.c4_count(ptr, idx) == comb(leaves, 2)
    assert O.tri_count(dptr, didx) == 0 and O.k4_count(dptr, didx) == 0


def test_c4_trace_identity(golden):
    """tr(A^4) = 8 C4 + 2 sum d(d-1) + 2m on real fixtures: two independent
    computations of the 4-cycle count agree."""
    for case in _cases(golden):
        if case["sym_nnz"] > 500_000:
            continue
        n, src, dst = edges_of(case)
        ptr, idx = O.sym_csr(src, dst, n)
        d = np.diff(ptr.astype(np.int64))
        hom = O.c4_hom(ptr, idx)
        c4 = O.c4_count(ptr, idx)
        assert hom == 8 * c4 + 2 * int((d * (d - 1)).sum()) + int(d.sum()), case["name"]


def test_planted_clique_k4(golden):
    case = next(c for c in golden["graphs"] if c["name"] == "planted_clique40")
    n, src, dst = edges_of(case)
    ptr, idx = O.sym_csr(src, dst, n)
    dptr, didx = O.orient(ptr, idx)
    k4 = O.k4_count(dptr, didx)
    assert k4 >= comb(40, 4)
    # the clique alone, counted in isolation
    cl = np.array(list(itertools.combinations(range(40), 2)), np.uint32)
    p2, i2 = O.sym_csr(cl[:, 0], cl[:, 1], 40)
    q2, j2 = O.orient(p2, i2)
    assert O.k4_count(q2, j2) == comb(40, 4)


def test_tc_bytes_formula(golden):
    case = next(c for c in golden["graphs"] if c["name"] == "rmat12_ef16_s3")
    n, src, dst = edges_of(case)
    ptr, idx = O.sym_csr(src, dst, n)
    dptr, didx = O.orient(ptr, idx)
    wedges, alg = O.tc_bytes(dptr, didx)
    dp = np.diff(dptr.astype(np.int64))
    rows = np.repeat(np.arange(n), dp)
    assert wedges == int(dp[didx].sum())
    assert alg == int((4 * (dp[rows] + dp[didx]) + 24).sum())


def test_intersection_oracle():
    a = np.array([1, 3, 5, 7, 9, 11], np.uint32)
    b = np.array([0, 3, 4, 7, 8, 11, 12], np.uint32)
    assert O.intersect(a, b) == 3
    assert O.intersect(a, b, materialise=True).tolist() == [3, 7, 11]
    assert O.intersect(a[:0], b) == 0


def _rmat_numpy(scale, seed, first, count):
    """Independent numpy restatement of the RMAT generator's specification."""
    key = splitmix(np.array([seed ^ 0x5851F42D4C957F2D], np.uint64))[0]
    i = np.arange(first, first + count, dtype=np.uint64)
    A, B, Cc = (57 << 32) // 100, (76 << 32) // 100, (95 << 32) // 100
    src = np.zeros(count, np.uint64)
    dst = np.zeros(count, np.uint64)
    with np.errstate(over="ignore"):
        for l in range(0, scale, 2):
            r = splitmix(key + (i * np.uint64(16) + np.uint64(l >> 1)) * np.uint64(0x9E3779B97F4A7C15))
            for h in range(2):
                if l + h >= scale:
                    break
                x = (r >> np.uint64(32)) if h else (r & np.uint64(0xFFFFFFFF))
                sb = (x >= B).astype(np.uint64)
                db = (((x >= A) & (x < B)) | (x >= Cc)).astype(np.uint64)
                src = (src << np.uint64(1)) | sb
                dst = (dst << np.uint64(1)) | db
    return src.astype(np.uint32), dst.astype(np.uint32)


def test_rmat_generator_matches_spec():
    import gary_b200 as gb

    for scale, seed, first, count in ((10, 3, 0, 5000), (21, 9, 123456789, 4000), (1, 1, 0, 100)):
        s, d = gb.gen_rmat(scale, seed, count, first)
        s2, d2 = _rmat_numpy(scale, seed, first, count)
        assert np.array_equal(s, s2) and np.array_equal(d, d2)
    # quadrant frequencies follow (0.57, 0.19, 0.19, 0.05) at scale 1
    s, d = gb.gen_rmat(1, 5, 200000)
    q = np.bincount(s.astype(np.int64) * 2 + d, minlength=4) / 200000
    assert np.allclose(q, [0.57, 0.19, 0.19, 0.05], atol=0.01)


def test_er_generator():
    import gary_b200 as gb

    s, d = gb.gen_er(1000, 20000, 4)
    assert (s < d).all() and (d < 1000).all()
    keys = s.astype(np.int64) * 1000 + d
    assert len(np.unique(keys)) == 20000
    s2, d2 = gb.gen_er(1000, 20000, 4)
    assert np.array_equal(s, s2) and np.array_equal(d, d2)


@pytest.mark.parametrize("scale,seed,first,count", [(12, 3, 0, 1 << 16), (24, 1, 12_345_678, 100_000),
                                                    (31, 9, 0, 1000), (1, 2, 0, 50), (17, 4, 7, 3)])
def test_rmat_restatement_matches_library(scale, seed, first, count):
    """The oracle's RMAT restatement (used by bench.py's reference arm, which
    must not load the product library) is the library's generator, edge for
    edge (gary_gen_rmat runs on the host)."""
    import gary_b200 as gb

    a_src, a_dst = gb.gen_rmat(scale, seed, count, first)
    b_src, b_dst = O.gen_rmat(scale, seed, count, first)
    assert np.array_equal(a_src, b_src) and np.array_equal(a_dst, b_dst)


def test_unique_edges_match_symmetric_csr():
    """orc_unique_edges (each undirected edge once, loops dropped) is the
    edge set of the oracle's symmetric CSR, in the same (u, v) order."""
    for scale, ef, seed in ((10, 16, 1), (14, 8, 4)):
        n = 1 << scale
        s, d = O.gen_rmat(scale, seed, ef << scale)
        s = np.concatenate([s, d[:100], np.arange(50, dtype=np.uint32)])  # reversed duplicates, loops
        d = np.concatenate([d, s[:100], np.arange(50, dtype=np.uint32)])
        us, vs = O.unique_edges(n, s, d)
        pu, pv = O.unique_pairs(*O.sym_csr(s, d, n))
        assert np.array_equal(us, pu) and np.array_equal(vs, pv)
        assert np.all(us < vs)


def _brute_counts(n: int, edges: set) -> tuple[int, int, int]:
    """Triangles, 4-cycles and 4-cliques of a small graph by looking at every
    3- and 4-vertex subset: a 4-set carries one of its three 4-cycles for each
    cyclic order whose four edges exist, and is a 4-clique when all six do."""
    e = lambda a, b: (min(a, b), max(a, b)) in edges  # noqa: E731
    tri = sum(e(a, b) and e(b, c) and e(a, c) for a, b, c in itertools.combinations(range(n), 3))
    c4 = k4 = 0
    for a, b, c, d in itertools.combinations(range(n), 4):
        c4 += (e(a, b) and e(b, c) and e(c, d) and e(d, a)) + (e(a, b) and e(b, d) and e(d, c) and e(c, a)) \
            + (e(a, c) and e(c, b) and e(b, d) and e(d, a))
        k4 += all(e(x, y) for x, y in itertools.combinations((a, b, c, d), 2))
    return tri, c4, k4


@pytest.mark.parametrize("seed", range(12))
def test_pattern_oracle_against_brute_force(seed):
    """The oracle's triangle, 4-cycle and 4-clique counts equal a brute-force
    enumeration on random small graphs of every density (the reference has no
    4-vertex pattern implementation to pin them to)."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(8, 19))
    p = [0.15, 0.35, 0.6, 0.9][seed % 4]
    edges = {(a, b) for a, b in itertools.combinations(range(n), 2) if rng.random() < p}
    if not edges:
        edges = {(0, 1)}
    src = np.array([a for a, _ in edges], np.uint32)
    dst = np.array([b for _, b in edges], np.uint32)
    ptr, idx = O.sym_csr(src, dst, n)
    dptr, didx = O.orient(ptr, idx)
    got = (O.tri_count(dptr, didx), O.c4_count(ptr, idx), O.k4_count(dptr, didx))
    assert got == _brute_counts(n, edges)
