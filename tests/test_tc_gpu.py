"""Triangle counting on the GPU through the C ABI, against the reference's
golden counts, the CPU oracle and the reference's own kernel built for sm_100a.
Counts are bit-exact uint64."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import gary_b200 as gb
from gary_b200 import _lib
from graphs import edges_of
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _has_lib(name):
    try:
        C.CDLL(name)
        return True
    except OSError:
        return False


def _upload_host(ptr, idx, n, flags=0):
    return gb.Graph.upload(np.ascontiguousarray(ptr, np.uint64), np.ascontiguousarray(idx, np.uint32), n, flags)


def test_golden_triangles(golden, cuda):
    for case in golden["graphs"]:
        n, src, dst = edges_of(case)
        ptr, idx = O.sym_csr(src, dst, n)
        with _upload_host(ptr, idx, n) as g:
            assert g.count() == case["ref_triangles"], case["name"]
            inf = g.info()
            assert inf["m"] == case["dag_nnz"]
            # counting twice gives the same number (scheduler state is reset)
            assert g.count() == case["ref_triangles"], case["name"]


def test_device_csr_builder_matches_oracle(golden, cuda):
    for case in golden["graphs"]:
        n, src, dst = edges_of(case)
        ptr, idx = O.sym_csr(src, dst, n)
        gptr, gidx = gb.csr_from_edges(src, dst, n)
        assert np.array_equal(gptr, ptr), case["name"]
        assert np.array_equal(gidx, idx), case["name"]


def test_orientation_structure(golden, cuda):
    """The uploaded DAG is exactly the oracle's degree orientation: with
    GARY_KEEP_IDS list by list; relabeled, after mapping ranks back."""
    for name in ("er_3000_60000_s5", "rmat14_ef16_s4", "planted_clique40", "K8", "no_edges"):
        case = next(c for c in golden["graphs"] if c["name"] == name)
        n, src, dst = edges_of(case)
        ptr, idx = O.sym_csr(src, dst, n)
        optr, oidx = O.orient(ptr, idx, by_degree=True)
        with _upload_host(ptr, idx, n, _lib.GARY_KEEP_IDS) as g:
            p, i, perm = g.download()
            assert g.info()["relabeled"] == 0
            assert np.array_equal(p, optr) and np.array_equal(i, oidx), name
        with _upload_host(ptr, idx, n) as g:
            p, i, perm = g.download()
            assert sorted(perm.tolist()) == list(range(n))
            deg = np.diff(ptr.astype(np.int64))
            # ranks follow (degree, id)
            assert np.all(np.diff(deg[perm] * (n + 1) + perm.astype(np.int64)) > 0)
            rows = np.repeat(np.arange(n), np.diff(p.astype(np.int64)))
            got = set(zip(perm[rows].tolist(), perm[i].tolist()))
            orows = np.repeat(np.arange(n), np.diff(optr.astype(np.int64)))
            want = set(zip(orows.tolist(), oidx.tolist()))
            assert got == want, name
            # every relabeled list is strictly increasing and points to higher ranks
            assert _rows_strictly_increasing(p, i), name
            assert np.all(i.astype(np.int64) > rows), name


def _rows_strictly_increasing(p, i) -> bool:
    p = p.astype(np.int64)
    i = i.astype(np.int64)
    if len(i) < 2:
        return True
    step = np.diff(i) > 0
    starts = p[1:-1][(p[1:-1] > 0) & (p[1:-1] < len(i))]
    step[starts - 1] = True  # a row boundary lies between i[s-1] and i[s]
    return bool(np.all(step))


def test_rmat_rows_sorted_every_length(cuda):
    """RMAT-18 ef32 has oriented rows of every length class the upload's
    warp row sort distinguishes (up to 32, 64, 128, 256, 512 and 1024 ids):
    each row comes back strictly increasing and the edge set is the oracle's."""
    n = 1 << 18
    src, dst = gb.gen_rmat(18, 9, 32 << 18)
    ptr, idx = gb.csr_from_edges(src, dst, n)
    optr, oidx = O.orient(ptr, idx, by_degree=True)
    lens = np.diff(optr.astype(np.int64))
    for lo, hi in ((2, 32), (33, 64), (65, 128), (129, 256), (257, 512), (513, 1024)):
        assert np.any((lens >= lo) & (lens <= hi)), (lo, hi)
    with _upload_host(ptr, idx, n, _lib.GARY_KEEP_IDS) as g:
        p, i, _ = g.download()
        assert np.array_equal(p, optr) and np.array_equal(i, oidx)
    with _upload_host(ptr, idx, n) as g:
        p, i, perm = g.download()
        assert _rows_strictly_increasing(p, i)
        assert np.array_equal(np.sort(np.diff(p.astype(np.int64))), np.sort(lens))
        assert g.count() == O.tri_count(optr, oidx)


def test_input_modes_agree(golden, cuda):
    """Symmetric input, DAG input (the reference's id-oriented csr_dag), kept
    ids and device-resident input all give the reference count."""
    import torch

    case = next(c for c in golden["graphs"] if c["name"] == "rmat14_ef16_s4")
    n, src, dst = edges_of(case)
    ptr, idx = O.sym_csr(src, dst, n)
    iptr, iidx = O.orient(ptr, idx, by_degree=False)
    want = case["ref_triangles"]
    with _upload_host(iptr, iidx, n, _lib.GARY_INPUT_DAG | _lib.GARY_VALIDATE) as g:
        assert g.count() == want
    with _upload_host(ptr, idx, n, _lib.GARY_KEEP_IDS | _lib.GARY_VALIDATE) as g:
        assert g.count() == want
    dp = torch.from_numpy(ptr.astype(np.int64)).cuda()
    di = torch.from_numpy(idx.astype(np.int32)).cuda()
    with gb.Graph.upload(dp, di, n) as g:
        assert g.count() == want
        out = torch.zeros(1, dtype=torch.int64, device="cuda")
        g.count_async(out)
        torch.cuda.synchronize()
        assert int(out.item()) == want
        # shards sum to the total
        total = 0
        for s in range(5):
            _lib.check(_lib.load().gary_count_shard_async(g.handle, 3, 0, s, 5, None, out.data_ptr()),
                       "shard")
            torch.cuda.synchronize()
            total += int(out.item())
        assert total == want


def test_malformed_input_rejected(cuda):
    def up(ptr, idx, n, flags=_lib.GARY_VALIDATE):
        return _lib.load().gary_graph_upload(np.asarray(ptr, np.uint64).ctypes.data,
                                             np.asarray(idx, np.uint32).ctypes.data, n, len(idx),
                                             flags, None, C.byref(C.c_void_p()))

    good_p, good_i = [0, 2, 4, 6], [1, 2, 0, 2, 0, 1]
    assert up(good_p, good_i, 3) == _lib.GARY_OK
    assert up([0, 2, 4, 6], [2, 1, 0, 2, 0, 1], 3) == _lib.GARY_ERR_INPUT       # unsorted
    assert up([0, 2, 4, 6], [0, 2, 0, 2, 0, 1], 3) == _lib.GARY_ERR_INPUT       # self loop
    assert up([0, 2, 4, 6], [1, 7, 0, 2, 0, 1], 3) == _lib.GARY_ERR_INPUT       # id >= n
    assert up([0, 2, 4, 5], [1, 2, 0, 2, 0], 3) == _lib.GARY_ERR_INPUT          # 1->2 one-way
    assert up([0, 1, 2, 3, 4], [1, 2, 3, 0], 4) == _lib.GARY_ERR_INPUT          # directed 4-cycle
    assert up([0, 1, 2], [1, 0], 2, _lib.GARY_INPUT_DAG) == _lib.GARY_ERR_INPUT  # edge listed twice
    assert b"malformed" in _lib.load().gary_last_error()
    assert up([0, 1, 1], [1, 1], 2, _lib.GARY_INPUT_DAG) == _lib.GARY_ERR_INVALID  # ptr[n] != nnz


def test_empty_and_tiny(cuda):
    for n, edges, want in ((1, [], 0), (5, [], 0), (3, [(0, 1), (1, 2), (0, 2)], 1), (2, [(0, 1)], 0)):
        e = np.array(edges, np.uint32).reshape(-1, 2)
        ptr, idx = O.sym_csr(e[:, 0], e[:, 1], n)
        with _upload_host(ptr, idx, n) as g:
            assert g.count() == want


def test_alg_bytes_match_oracle(golden, cuda):
    case = next(c for c in golden["graphs"] if c["name"] == "rmat16_ef16_s5")
    n, src, dst = edges_of(case)
    ptr, idx = O.sym_csr(src, dst, n)
    with _upload_host(ptr, idx, n) as g:
        p, i, _ = g.download()
        w, b = O.tc_bytes(p, i)
        inf = g.info()
        assert inf["wedges"] == w and inf["alg_bytes"] == b
        assert inf["max_out_degree"] == int(np.diff(p.astype(np.int64)).max())


def test_device_views(golden, cuda):
    import torch

    case = next(c for c in golden["graphs"] if c["name"] == "rmat12_ef16_s3")
    n, src, dst = edges_of(case)
    ptr, idx = O.sym_csr(src, dst, n)
    with _upload_host(ptr, idx, n) as g:
        p, i, _ = g.download()
        csr = g.device_csr()
        coo = g.device_coo()
        assert csr.m == n and csr.nnz == len(i) and coo.nnz == len(i)
        # the views are raw device pointers: read them back through torch
        cudart = C.CDLL("libcudart.so.12") if _has_lib("libcudart.so.12") else C.CDLL(
            "/usr/local/cuda/lib64/libcudart.so")
        cudart.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]

        def dev(ptr_, count, dt):
            out = np.empty(count, dt)
            assert cudart.cudaMemcpy(out.ctypes.data, ptr_, out.nbytes, 2) == 0  # DeviceToHost
            return out
        rows = dev(coo.rowIdx, len(i), np.uint32)
        cols = dev(coo.colIdx, len(i), np.uint32)
        assert np.array_equal(cols, i)
        assert np.array_equal(rows, np.repeat(np.arange(n, dtype=np.uint32), np.diff(p.astype(np.int64))))
        deg = dev(csr.deg, n, np.uint32)
        assert np.array_equal(deg, np.diff(p.astype(np.int64)).astype(np.uint32))
        indptr = dev(csr.indPtr, n + 1, np.uint64)
        assert np.all(indptr % 8 == 0)                      # 32-byte aligned lists
        adj = dev(csr.colIdx, int(indptr[-1]), np.uint32)
        for v in range(0, n, 37):
            assert np.array_equal(adj[indptr[v]:indptr[v] + deg[v]], i[p[v]:p[v + 1]])
            pad = adj[indptr[v] + deg[v]:indptr[v + 1]]
            assert np.all(pad == 0xFFFFFFFF)


@pytest.mark.skipif(not O.have_ref_gpu(), reason="reference GPU build absent")
def test_reference_kernel_parity(golden, cuda):
    """Our count == the reference's triangleCountHom (cache, interleaved and
    chunked; no cache) and triangleCountLegacy built for sm_100a, on the same
    graphs."""
    for name in ("er_16384_131072_s3", "rmat16_ef16_s5", "planted_clique40", "rmat12_ef32_s7"):
        case = next(c for c in golden["graphs"] if c["name"] == name)
        n, src, dst = edges_of(case)
        ptr, idx = O.sym_csr(src, dst, n)
        iptr, iidx = O.orient(ptr, idx, by_degree=False)
        ref = O.RefGpuGraph(iptr, iidx)
        with _upload_host(ptr, idx, n) as g:
            ours = g.count()
        for v in (0, 1, 2, 3):
            c, _ = ref.tri_count(v)
            assert c == ours == case["ref_triangles"], (name, v)
        ref.free()


def test_rmat18_vs_oracle(cuda):
    src, dst = gb.gen_rmat(18, 11, 16 << 18)
    ptr, idx = gb.csr_from_edges(src, dst, 1 << 18)
    optr, oidx = O.orient(ptr, idx)
    want = O.tri_count(optr, oidx)
    with _upload_host(ptr, idx, 1 << 18) as g:
        assert g.count() == want


@pytest.mark.parametrize("cfg", [
    {"warp_tile_cost": 1 << 12, "cta_tile_cost": 1 << 16, "min_blocks": 3},
    {"warp_tile_cost": 1 << 18, "cta_tile_cost": 1 << 23, "min_blocks": 2},
    {"warp_tile_cost": 1 << 15, "cta_tile_cost": 1 << 20, "vertex_overhead": 0, "min_blocks": 2},
    {"warp_cap": 8, "cta_set_words": 64, "warp_tile_cost": 1 << 11},
])
def test_tile_shapes_keep_the_count(cuda, cfg):
    """The scheduler's tile shapes change only how work is cut, never the count."""
    from gary_b200 import autotune

    src, dst = gb.gen_rmat(16, 21, 32 << 16)
    ptr, idx = gb.csr_from_edges(src, dst, 1 << 16)
    optr, oidx = O.orient(ptr, idx)
    want = O.tri_count(optr, oidx)
    try:
        autotune.apply(cfg)
        with _upload_host(ptr, idx, 1 << 16) as g:
            assert g.count() == want
    finally:
        autotune.apply({})


def test_scratch_pool_setting_keeps_results(cuda):
    """Trimming the library's scratch pool at every sync (pool_keep_bytes 0)
    and keeping it mapped give the same graph and count."""
    L = _lib.load()
    src, dst = gb.gen_rmat(14, 2, 16 << 14)
    ptr, idx = gb.csr_from_edges(src, dst, 1 << 14)
    optr, oidx = O.orient(ptr, idx)
    want = O.tri_count(optr, oidx)
    try:
        for keep in (0, (1 << 64) - 1):
            _lib.check(L.gary_tune(b"pool_keep_bytes", keep), "gary_tune")
            with _upload_host(ptr, idx, 1 << 14) as g:
                assert g.count() == want
    finally:
        _lib.check(L.gary_tune(b"pool_keep_bytes", (1 << 64) - 1), "gary_tune")


@pytest.mark.parametrize("k", [33, 1500, 9000])
def test_complete_graph_long_rows(cuda, k):
    """K_k: C(k,3) triangles.  Its oriented rows hold up to k-1 ids, so the
    upload's row sort takes every path: warp ranks (<= 32), warp bitonic
    (<= 1024), CTA bitonic (<= 8192) and the per-row library sort beyond."""
    from math import comb

    ptr = (np.arange(k + 1, dtype=np.uint64) * (k - 1))
    full = np.tile(np.arange(k, dtype=np.uint32), k).reshape(k, k)
    idx = full[~np.eye(k, dtype=bool)].astype(np.uint32)
    with _upload_host(ptr, idx, k, _lib.GARY_VALIDATE) as g:
        assert g.count() == comb(k, 3)
        dp, di, _ = g.download()
        assert np.all(np.diff(dp.astype(np.int64)) == np.arange(k - 1, -1, -1))
        want = np.concatenate([np.arange(u + 1, k, dtype=np.uint32) for u in range(k)])
        assert np.array_equal(di, want)


def test_block_cache_reuse_across_shapes(cuda):
    """Freed graphs hand their device blocks to later uploads (the library's
    block cache): graphs of three sizes, uploaded, freed out of order and
    uploaded again, keep their exact counts."""
    cases = []
    for scale, ef, seed in ((12, 8, 1), (15, 16, 2), (13, 4, 3)):
        n = 1 << scale
        src, dst = gb.gen_rmat(scale, seed, ef << scale)
        ptr, idx = gb.csr_from_edges(src, dst, n)
        optr, oidx = O.orient(ptr, idx)
        cases.append((ptr, idx, n, O.tri_count(optr, oidx)))
    live = [_upload_host(p, i, n) for p, i, n, _ in cases]
    for g, (_, _, _, want) in zip(live, cases):
        assert g.count() == want
    live[1].free()
    live[0].free()
    again = [_upload_host(p, i, n) for p, i, n, _ in reversed(cases)]
    for g, (_, _, _, want) in zip(again, reversed(cases)):
        assert g.count() == want
    live[2].free()
    for g in again:
        g.free()

