"""Every way a triangle CTA tile can hold N+(v), run and counted.

A CTA tile holds N+(v) in the cheapest shared-memory set that fits: a bitmap
of its id span, 4-slot hash buckets, the sorted list staged whole by a bulk
copy (cp.async.bulk with an mbarrier), or evenly spaced samples for the
two-phase search with its second phase in HBM (the reference's
binary_search_2phase, include/ops/Search.cuh:93-138; its staging precedent is
intersectSmall's cg::memcpy_async, include/ops/Intersection.cuh:142-164).  On
the bench graphs only the first two occur: the last two need d+(v) > 8192
with an id span beyond 2^19.  The test-only tuning keys "warp_cap" and
"cta_set_words" send small RMAT graphs down every path, and the per-path tile
counts in gary_count_last_stats prove each one ran.  The graph that reaches
them is an Erdos-Renyi graph of 2^17 vertices and average degree 96: ranks by
degree put most out-neighbour lists across more than 32 K ids (too wide for
a warp bitmap), with out-degrees from a few to over 100, so with warp_cap 8
and 64 shared words per CTA set the CTA tiles split between buckets
(d+ <= 32), staged lists (<= 64) and samples (beyond).  RMAT graphs of this
size have no such vertices: their wide lists are short.  Counts are
bit-exact against the CPU oracle.

The bounded waits: "stage_wait_polls" = 0 makes the first wait for every
staging copy give up at once.  The launch must then report GARY_ERR_TIMEOUT
on every count path (gary_count, and gary_count_status after an
asynchronous count), while the drain wait, which keeps its full limit, lets
the copy land, so the count itself is still exact.  No GPU is faulted or
hung: the expired wait is a poll limit of zero, not a copy that never lands.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import gary_b200 as gb
from gary_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PATHS = ("bitmap", "buckets", "staged", "sampled")


def _tune(**kv):
    L = _lib.load()
    for k, v in kv.items():
        _lib.check(L.gary_tune(k.encode(), v), f"gary_tune({k})")


def _reset():
    _lib.check(_lib.load().gary_tune(b"reset", 0), "gary_tune(reset)")


def _rmat(scale, ef, seed):
    n = 1 << scale
    src, dst = gb.gen_rmat(scale, seed, ef << scale)
    ptr, idx = gb.csr_from_edges(src, dst, n)
    optr, oidx = O.orient(ptr, idx)
    return n, ptr, idx, O.tri_count(optr, oidx)


def _er_wide():
    n = 1 << 17
    src, dst = gb.gen_er(n, n * 48, 7)
    ptr, idx = O.sym_csr(src, dst, n)
    optr, oidx = O.orient(ptr, idx)
    return n, ptr, idx, O.tri_count(optr, oidx)


def _count_with(g, **kv):
    """Count after rebuilding the plan under the given knobs; (count, stats)."""
    _lib.check(_lib.load().gary_graph_drop_plans(g.handle), "drop plans")
    _reset()
    _tune(**kv)
    c = g.count()
    return c, g.last_stats()


def test_every_cta_set_path_runs_and_counts_exactly(cuda):
    n, ptr, idx, want = _er_wide()
    try:
        with gb.Graph.upload(ptr, idx, n) as g:
            plain = g.count()
            assert plain == want
            # many CTA vertices, full shared buffer: all of them fit a bitmap
            c, st = _count_with(g, warp_cap=8)
            assert c == want and st["error"] == 0
            assert st["cta_tiles"] > 0 and st["cta_path_tiles"]["bitmap"] == st["cta_tiles"], st
            # 64 shared words: d+ <= 32 buckets, <= 64 staged whole, beyond sampled
            c, st = _count_with(g, warp_cap=8, cta_set_words=64)
            assert c == want and st["error"] == 0
            p = st["cta_path_tiles"]
            assert p["buckets"] > 0 and p["staged"] > 0 and p["sampled"] > 0, st
            assert sum(p.values()) == st["cta_tiles"]
            # a mid-sized buffer mixes the paths
            c, st = _count_with(g, warp_cap=16, cta_set_words=256)
            assert c == want and st["error"] == 0
            assert sum(st["cta_path_tiles"].values()) == st["cta_tiles"]
    finally:
        _reset()


@pytest.mark.parametrize("scale,ef,seed", [(16, 16, 5), (18, 16, 11)])
def test_small_cta_sets_keep_rmat_counts(cuda, scale, ef, seed):
    """The same knobs on RMAT graphs (whatever paths their CTA tiles take)."""
    n, ptr, idx, want = _rmat(scale, ef, seed)
    try:
        with gb.Graph.upload(ptr, idx, n) as g:
            for kv in ({"warp_cap": 8}, {"warp_cap": 8, "cta_set_words": 64}, {"warp_cap": 16, "cta_set_words": 256}):
                c, st = _count_with(g, **kv)
                assert c == want and st["error"] == 0, kv
                assert sum(st["cta_path_tiles"].values()) == st["cta_tiles"], kv
    finally:
        _reset()


def test_expired_staging_wait_is_reported_everywhere(cuda):
    import torch

    n, ptr, idx, want = _er_wide()
    L = _lib.load()
    try:
        with gb.Graph.upload(ptr, idx, n) as g:
            _lib.check(L.gary_graph_drop_plans(g.handle), "drop plans")
            _tune(warp_cap=8, cta_set_words=64, stage_wait_polls=0)
            # blocking count: the status, not a silent number
            v = C.c_uint64(0)
            assert L.gary_count(g.handle, 3, 0, None, C.byref(v)) == _lib.GARY_ERR_TIMEOUT
            assert b"bounded device wait" in L.gary_last_error()
            st = g.last_stats()
            assert st["cta_path_tiles"]["staged"] > 0
            assert st["error"] == 1, st  # the first wait gave up; every drain wait succeeded
            # asynchronous count and shard paths: gary_count_status reports it
            dout = torch.zeros(1, dtype=torch.int64, device="cuda")
            g.count_async(dout)
            assert g.status() == _lib.GARY_ERR_TIMEOUT
            # the drained copies landed, so the count itself is exact
            assert int(dout.item()) == want
            _lib.check(L.gary_count_shard_async(g.handle, 3, 0, 0, 2, None, dout.data_ptr()), "shard")
            assert g.status() == _lib.GARY_ERR_TIMEOUT
            # full poll limit again: clean
            _lib.check(L.gary_graph_drop_plans(g.handle), "drop plans")
            _reset()
            _tune(warp_cap=8, cta_set_words=64)
            g.count_async(dout)
            assert g.status() == _lib.GARY_OK
            assert int(dout.item()) == want
            assert g.last_stats()["error"] == 0
    finally:
        _reset()


def test_count_status_clean_on_every_pattern(cuda):
    import torch

    n, ptr, idx, want = _rmat(14, 16, 3)
    with gb.Graph.upload(ptr, idx, n) as g:
        dout = torch.zeros(1, dtype=torch.int64, device="cuda")
        for pat in (3, 4, 5):
            g.count_async(dout, pat)
            assert g.status() == _lib.GARY_OK, pat
            assert g.last_stats()["error"] == 0
        g.count_async(dout, 3)
        assert g.status() == _lib.GARY_OK and int(dout.item()) == want


@pytest.mark.skipif(not O.have_ref_gpu(), reason="reference GPU build absent")
def test_rmat22_ef16_matches_reference_kernel_and_oracle(cuda):
    """The RMAT-22 edge-factor-16 workload (seeded, deduplicated, symmetrised,
    degree-oriented): our count equals the reference's triangleCountHom<true,32>
    built for sm_100a (test/TriQueryTest.cu:114-133) and the CPU oracle."""
    import torch

    scale, ef, seed = 22, 16, 1
    n = 1 << scale
    src, dst = gb.gen_rmat_device(scale, seed, ef << scale)
    csr = gb.csr_from_edges_device(src, dst, n)
    del src, dst
    p, i = csr.device_ptrs()
    _, nnz = csr.shape()
    h = C.c_void_p()
    _lib.check(_lib.load().gary_graph_upload(p, i, n, nnz, _lib.GARY_INPUT_DEVICE, None, C.byref(h)), "upload")
    csr.free()
    g = gb.Graph(h.value)
    try:
        ours = g.count()
        assert g.info()["m"] == 64_156_972
        dptr, didx, _ = g.download()
    finally:
        g.free()
    torch.cuda.empty_cache()
    want = O.tri_count(dptr, didx)
    ref = O.RefGpuGraph(dptr.astype(np.int64), didx.astype(np.int32))
    try:
        ref_count, _ = ref.tri_count(0)
    finally:
        ref.free()
    assert ours == want == ref_count == 2_109_520_824


@pytest.mark.skipif(not O.have_ref_gpu(), reason="reference GPU build absent")
def test_rmat24_ef32_full_size_properties(cuda):
    """The bench workload itself (RMAT scale 24, edge factor 32: 511,877,083
    oriented edges), through properties that do not need a CPU count at this
    size: the plain count, the learned schedule's count, the sum of three
    shards and the reference's own triangleCountHom<true,32> (sm_100a build)
    on the same DAG all give 46,507,684,959, and every launch reports a clean
    status."""
    import torch

    from gary_b200.costmodel import CostModel

    scale, ef, seed = 24, 32, 1
    n = 1 << scale
    src, dst = gb.gen_rmat_device(scale, seed, ef << scale)
    csr = gb.csr_from_edges_device(src, dst, n)
    del src, dst
    torch.cuda.empty_cache()
    p, i = csr.device_ptrs()
    _, nnz = csr.shape()
    h = C.c_void_p()
    _lib.check(_lib.load().gary_graph_upload(p, i, n, nnz, _lib.GARY_INPUT_DEVICE, None, C.byref(h)), "upload")
    csr.free()
    torch.cuda.empty_cache()
    want = 46_507_684_959
    g = gb.Graph(h.value)
    try:
        assert g.info()["m"] == 511_877_083
        assert g.count() == want
        CostModel.load().install()
        assert g.count(3, _lib.GARY_SCHED_LEARNED) == want
        out = torch.zeros(1, dtype=torch.int64, device="cuda")
        total = 0
        for sh in range(3):
            _lib.check(_lib.load().gary_count_shard_async(g.handle, 3, 0, sh, 3, None, out.data_ptr()), "shard")
            assert g.status() == _lib.GARY_OK
            total += int(out.item())
        assert total == want
        dptr, didx, _ = g.download()
    finally:
        g.free()
        _lib.load().gary_set_cost_model(None)
    torch.cuda.empty_cache()
    ref = O.RefGpuGraph(dptr.astype(np.int64), didx.astype(np.int32))
    try:
        ref_count, _ = ref.tri_count(0)
    finally:
        ref.free()
    assert ref_count == want
