"""The allocation-free triangle count, for callers that cannot call cudaMalloc.

Such a caller already holds the oriented graph on the device and passes it,
with a device word for the result; the library's only scratch is a fixed
file-scope device array.  This test calls gary_count_triangles_noalloc through
the C ABI, twice in a row on the same scratch, and checks each result against
gary_count on the same graph (counts are integers: equal exactly).  It sits
in its own file, collected last, and passes alone or after the other tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import gary_b200 as gb
from gary_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _noalloc(indptr, colidx, deg, n, out):
    return _lib.load().gary_count_triangles_noalloc(indptr, colidx, deg, n, None, out)


def test_noalloc_matches_count(cuda):
    import torch

    for scale, ef, seed in ((16, 16, 5), (18, 8, 2)):
        n = 1 << scale
        src, dst = gb.gen_rmat(scale, seed, ef << scale)
        ptr, idx = gb.csr_from_edges(src, dst, n)
        with gb.Graph.upload(ptr, idx, n) as g:
            want = g.count()
            v = g.device_csr()  # degree-ranked, padded lists already on the device
            out = torch.full((1,), -1, dtype=torch.int64, device="cuda")
            for _ in range(2):  # two calls in a row share the same scratch
                assert _noalloc(v.indPtr, v.colIdx, v.deg, n, out.data_ptr()) == _lib.GARY_OK
                torch.cuda.synchronize()
                assert int(out.item()) == want
                out.fill_(-1)


def test_noalloc_on_reference_orientation(golden, cuda):
    """An unpadded CSR oriented by id (the reference's csr_dag layout) that the
    caller placed on the device itself."""
    import torch

    from graphs import edges_of

    case = next(c for c in golden["graphs"] if c["name"] == "rmat14_ef16_s4")
    n, src, dst = edges_of(case)
    sptr, sidx = O.sym_csr(src, dst, n)
    iptr, iidx = O.orient(sptr, sidx, by_degree=False)
    dptr = torch.from_numpy(iptr[:-1].astype(np.int64)).cuda()
    didx = torch.from_numpy(iidx.astype(np.int32)).cuda()
    ddeg = torch.from_numpy(np.diff(iptr.astype(np.int64)).astype(np.int32)).cuda()
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    for _ in range(2):
        assert _noalloc(dptr.data_ptr(), didx.data_ptr(), ddeg.data_ptr(), n, out.data_ptr()) == _lib.GARY_OK
        torch.cuda.synchronize()
        assert int(out.item()) == case["ref_triangles"]


def test_noalloc_long_scattered_list(cuda):
    """A vertex whose list is too long for a warp's shared hash (more than
    512 ids) and spread too wide for its bitmap (ids over more than 32 K
    values): the kernel searches that list in device memory.  An id-oriented
    hub at the top id of a 70,000-vertex graph, with 900 neighbours spread
    over the whole id range and random edges among them."""
    import torch

    n, hub = 70_000, 69_999
    rng = np.random.default_rng(7)
    nb = np.unique(rng.choice(hub, 900, replace=False)).astype(np.uint32)
    assert nb.max() - nb.min() > 32_768
    es, ed = gb.gen_er(n, 200_000, 9)
    pairs = rng.integers(0, len(nb), size=(6_000, 2))
    src = np.concatenate([np.full(len(nb), hub, np.uint32), nb[pairs[:, 0]], es])
    dst = np.concatenate([nb, nb[pairs[:, 1]], ed])
    sptr, sidx = O.sym_csr(src, dst, n)
    iptr, iidx = O.orient(sptr, sidx, by_degree=False)
    assert int(iptr[hub + 1] - iptr[hub]) > 512
    want = O.tri_count(iptr, iidx)
    assert want > 0
    dptr = torch.from_numpy(iptr[:-1].astype(np.int64)).cuda()
    didx = torch.from_numpy(iidx.astype(np.int32)).cuda()
    ddeg = torch.from_numpy(np.diff(iptr.astype(np.int64)).astype(np.int32)).cuda()
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    for _ in range(2):
        out.fill_(-1)
        assert _noalloc(dptr.data_ptr(), didx.data_ptr(), ddeg.data_ptr(), n, out.data_ptr()) == _lib.GARY_OK
        torch.cuda.synchronize()
        assert int(out.item()) == want
    with gb.Graph.upload(sptr, sidx, n) as g:
        assert g.count() == want


def test_noalloc_rejects_oversize(cuda):
    v = C.c_uint64()
    st = _noalloc(None, None, None, 33_550_337, C.addressof(v))
    assert st == _lib.GARY_ERR_INVALID
    assert b"no-allocation limit" in _lib.load().gary_last_error()
