"""4-cycle and 4-clique counts on the GPU against the CPU oracle and
closed-form known answers (the reference has no implementation of these
patterns: rectCountHom is declared only, include/kernels/GraphQueryHom.cuh:48)."""
from __future__ import annotations

import itertools
from math import comb

import numpy as np
import pytest

import gary_b200 as gb
from gary_b200 import _lib
from graphs import edges_of
from oracle import oracle as O

pytestmark = pytest.mark.gpu
K3, C4, K4 = _lib.GARY_PATTERN_TRIANGLE, _lib.GARY_PATTERN_4CYCLE, _lib.GARY_PATTERN_4CLIQUE


def _graph(n, edges):
    e = np.array(edges, np.uint32).reshape(-1, 2)
    ptr, idx = O.sym_csr(e[:, 0], e[:, 1], n)
    return ptr, idx


def _counts(ptr, idx, n):
    with gb.Graph.upload(ptr, idx, n) as g:
        return g.count(K3), g.count(C4), g.count(K4)


# 1100 and 1500: d+ up to 1499, past the 1024 whose bit rows fit shared memory (rows in HBM)
@pytest.mark.parametrize("n", [4, 5, 8, 13, 40, 600, 1100, 1500])
def test_complete_graphs(cuda, n):
    ptr, idx = _graph(n, list(itertools.combinations(range(n), 2)))
    assert _counts(ptr, idx, n) == (comb(n, 3), 3 * comb(n, 4), comb(n, 4))


def test_small_kats(cuda):
    assert _counts(*_graph(17, [(0, i) for i in range(1, 17)]), 17) == (0, 0, 0)
    assert _counts(*_graph(4, [(0, 1), (1, 2), (2, 3), (3, 0)]), 4) == (0, 1, 0)
    wheel = [(0, i) for i in range(1, 11)] + [(i, i % 10 + 1) for i in range(1, 11)]
    assert _counts(*_graph(11, wheel), 11) == (10, 10, 0)
    assert _counts(*_graph(5, [(0, 2), (0, 3), (0, 4), (1, 2), (1, 3), (1, 4)]), 5) == (0, 3, 0)
    assert _counts(*_graph(6, []), 6) == (0, 0, 0)
    # complete bipartite K_{30,40}: C(30,2) C(40,2) 4-cycles, no triangles
    kb = [(a, 30 + b) for a in range(30) for b in range(40)]
    assert _counts(*_graph(70, kb), 70) == (0, comb(30, 2) * comb(40, 2), 0)


def test_golden_graphs_vs_oracle(golden, cuda):
    for case in golden["graphs"]:
        if case["sym_nnz"] > 2_000_000:
            continue
        n, src, dst = edges_of(case)
        ptr, idx = O.sym_csr(src, dst, n)
        dptr, didx = O.orient(ptr, idx)
        want = (case["ref_triangles"], O.c4_count(ptr, idx), O.k4_count(dptr, didx))
        assert _counts(ptr, idx, n) == want, case["name"]


@pytest.mark.parametrize("scale,ef,seed", [(16, 16, 3), (18, 8, 4)])
def test_rmat_vs_oracle(cuda, scale, ef, seed):
    n = 1 << scale
    src, dst = gb.gen_rmat(scale, seed, ef << scale)
    ptr, idx = gb.csr_from_edges(src, dst, n)
    dptr, didx = O.orient(ptr, idx)
    with gb.Graph.upload(ptr, idx, n) as g:
        assert g.count(C4) == O.c4_count(ptr, idx)
        assert g.count(K4) == O.k4_count(dptr, didx)
        # counting again reuses the cached plans and gives the same numbers
        assert g.count(C4) == O.c4_count(ptr, idx)


def test_c4_trace_identity_on_gpu(cuda):
    """hom(C4) = tr(A^4) = 8 C4 + 2 sum d(d-1) + 2m, with C4 from the GPU."""
    src, dst = gb.gen_rmat(12, 9, 16 << 12)
    ptr, idx = gb.csr_from_edges(src, dst, 1 << 12)
    d = np.diff(ptr.astype(np.int64))
    with gb.Graph.upload(ptr, idx, 1 << 12) as g:
        c4 = g.count(C4)
    assert O.c4_hom(ptr, idx) == 8 * c4 + 2 * int((d * (d - 1)).sum()) + int(d.sum())


@pytest.mark.parametrize("leaves", [65535, 65536, 70000])
def test_c4_counter_width_limits(cuda, leaves):
    """K_{2,n}: two hubs joined to n leaves hold C(n,2) 4-cycles.  The top hub
    has n lower neighbours and one wedge end (the other hub) reached n times,
    so its window counter climbs to n.  Up to 65535 lower neighbours the
    window kernel packs 16-bit counters (n = 65535 drives one to its maximum);
    from 65536 it counts 32-bit counters over half windows."""
    n = leaves + 2
    a = np.arange(2, n, dtype=np.uint32)
    src = np.concatenate([np.zeros(leaves, np.uint32), np.ones(leaves, np.uint32)])
    dst = np.concatenate([a, a])
    ptr, idx = O.sym_csr(src, dst, n)
    with gb.Graph.upload(ptr, idx, n) as g:
        assert g.count(C4) == comb(leaves, 2)
        assert g.count(K3) == 0


def test_c4_many_heavy_hubs(cuda):
    """Several hubs over a shared leaf set, with leaves also joined in a ring:
    every pair of hubs closes C(leaves, 2) 4-cycles through two leaves, plus
    the cycles that use ring edges; the oracle settles the total.  Hubs are
    heavy vertices whose windows span the whole leaf range."""
    hubs, leaves = 6, 3000
    n = hubs + leaves
    lv = np.arange(hubs, n, dtype=np.uint32)
    src = np.concatenate([np.full(leaves, h, np.uint32) for h in range(hubs)] + [lv])
    dst = np.concatenate([lv for _ in range(hubs)] + [np.roll(lv, 1)])
    ptr, idx = O.sym_csr(src, dst, n)
    with gb.Graph.upload(ptr, idx, n) as g:
        assert g.count(C4) == O.c4_count(ptr, idx)
