"""Batched counting of many graphs: workload generation on the CPU; on the GPU
the one-launch per-graph counts against separately uploaded graphs and the
CPU oracle, and CUDA-graph replay."""
from __future__ import annotations

import math

import numpy as np
import pytest

from gary_b200 import batch as B
from oracle import oracle as O


def test_specs_deterministic_and_log_uniform():
    a = B.make_specs(4096, seed=1)
    b = B.make_specs(4096, seed=1)
    assert [(s.kind, s.n, s.m, s.seed) for s in a] == [(s.kind, s.n, s.m, s.seed) for s in b]
    ns = np.array([s.n for s in a])
    assert ns.min() >= 1000 and ns.max() <= 200000
    # log-uniform: the median of log n sits in the middle of the range
    assert abs(np.median(np.log(ns)) - 0.5 * (math.log(1e3) + math.log(2e5))) < 0.15
    assert {s.kind for s in a[::2]} == {"ba"} and {s.kind for s in a[1::2]} == {"rmat"}
    assert {s.m for s in a[::2]} <= set(range(2, 17)) and len({s.m for s in a[::2]}) == 15


def test_ba_generator():
    spec = B.GraphSpec(0, "ba", 5000, 7, 42)
    s, d = B.generate(spec)
    assert len(s) == 7 * 8 // 2 + (5000 - 8) * 7
    keys = np.minimum(s, d).astype(np.int64) * 5000 + np.maximum(s, d)
    assert len(np.unique(keys)) == len(keys) and not np.any(s == d)
    ptr, idx = O.sym_csr(s, d, 5000)
    deg = np.diff(ptr.astype(np.int64))
    assert deg.min() >= 7 and deg.max() > 10 * 7   # preferential attachment grows hubs
    s2, d2 = B.generate(spec)
    assert np.array_equal(s, s2) and np.array_equal(d, d2)


def test_rmat_member_rejection():
    spec = B.GraphSpec(1, "rmat", 3000, 0, 7)
    s, d = B.generate(spec)
    assert len(s) > 0 and s.max() < 3000 and d.max() < 3000


@pytest.mark.gpu
def test_batched_counts_match_per_graph_and_oracle(cuda):
    import torch

    specs = B.make_specs(64, seed=5, n_lo=300, n_hi=3000)
    batch = B.Batch.build(specs)
    counts, total = batch.count()
    assert total == int(counts.sum())
    graphs = B.per_graph_graphs(specs)
    for spec, g, c in zip(specs, graphs, counts):
        assert g.count() == int(c), spec
        g.free()
    for spec, c in list(zip(specs, counts))[:12]:
        s, d = B.generate(spec)
        ptr, idx = O.sym_csr(s, d, spec.n)
        dp, di = O.orient(ptr, idx)
        assert O.tri_count(dp, di) == int(c), spec
    # CUDA-graph replay gives the same numbers, twice
    stream = torch.cuda.Stream()
    exe = batch.capture(stream)
    for _ in range(2):
        exe.counts.fill_(0)
        exe.launch(stream)
        stream.synchronize()
        assert np.array_equal(exe.counts.cpu().numpy().view(np.uint64), counts)
        assert int(exe.total.item()) == total
    exe.free()
    batch.free()


@pytest.mark.gpu
def test_full_4096_graph_batch(cuda):
    """The batched workload at its full size: 4096 graphs, n log-uniform in
    [1e3, 2e5], half Barabasi-Albert (m in 2..16), half RMAT ef8, counted in
    one launch.  Every graph's count equals its own upload counted alone, and
    a spread of graphs (the smallest, the largest, every 256th) equals the CPU
    oracle."""
    import ctypes as C
    from concurrent.futures import ThreadPoolExecutor

    import torch

    import gary_b200 as gb
    from gary_b200 import _lib

    specs = B.make_specs(4096, seed=1)
    batch = B.Batch.build(specs)
    try:
        counts, total = batch.count()
        st = batch.graph.status()
        assert st == 0
    finally:
        batch.free()
    torch.cuda.empty_cache()
    assert total == int(counts.sum())
    ns = np.array([s.n for s in specs])
    sample = sorted({int(ns.argmin()), int(ns.argmax()), *range(0, 4096, 256), *range(1, 4096, 256)})
    with ThreadPoolExecutor(16) as ex:
        for lo in range(0, 4096, 512):
            edges = list(ex.map(B.generate, specs[lo:lo + 512]))
            for k, (s, d) in enumerate(edges):
                spec = specs[lo + k]
                with gb.csr_from_edges_device(s, d, spec.n) as csr:
                    p, i = csr.device_ptrs()
                    _, nnz = csr.shape()
                    h = C.c_void_p()
                    _lib.check(_lib.load().gary_graph_upload(p, i, spec.n, nnz, _lib.GARY_INPUT_DEVICE, None,
                                                             C.byref(h)), "upload")
                with gb.Graph(h.value) as g:
                    assert g.count() == int(counts[spec.index]), spec
                if spec.index in sample:
                    ptr, idx = O.sym_csr(s, d, spec.n)
                    dp, di = O.orient(ptr, idx)
                    assert O.tri_count(dp, di) == int(counts[spec.index]), spec
