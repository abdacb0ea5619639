"""Byte planes (the reference's segmentKernel, include/kernels/SegmentArray.cuh;
its tests test/CUDATest.cu:60-130 split 0xAABBCCDD words into four byte
planes at sizes 128, 256 and 127): against numpy's byte view, and the join
as its inverse."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import gary_b200 as gb
from gary_b200 import _lib

CONFIGS = [(4, 1), (4, 2), (8, 1), (8, 2), (8, 4)]


def _numpy_planes(words: np.ndarray, pb: int) -> list[np.ndarray]:
    wb = words.dtype.itemsize
    b = words.view(np.uint8).reshape(len(words), wb)
    return [b[:, j * pb:(j + 1) * pb].copy().view({1: np.uint8, 2: np.uint16, 4: np.uint32}[pb]).ravel()
            for j in range(wb // pb)]


def test_argument_checks_without_device():
    L = _lib.load()
    planes = (C.c_void_p * 4)(0x1000, 0x2000, 0x3000, 0x4000)
    assert L.gary_planes_split(C.c_void_p(0x1001), 16, 4, 1, planes, None) == _lib.GARY_ERR_INVALID
    assert L.gary_planes_split(C.c_void_p(0x1000), 16, 4, 4, planes, None) == _lib.GARY_ERR_INVALID
    assert L.gary_planes_split(C.c_void_p(0x1000), 16, 2, 1, planes, None) == _lib.GARY_ERR_INVALID
    bad = (C.c_void_p * 4)(0x1000, 0x2008, 0x3000, 0x4000)
    assert L.gary_planes_join(bad, 16, 4, 1, C.c_void_p(0x1000), None) == _lib.GARY_ERR_INVALID
    assert L.gary_planes_split(None, 0, 4, 1, None, None) == _lib.GARY_OK


@pytest.mark.gpu
@pytest.mark.parametrize("size", [128, 256, 127])
def test_reference_cases(cuda, size):
    import torch

    words = torch.full((size,), 0xAABBCCDD - (1 << 32), dtype=torch.int32, device="cuda")
    planes = gb.planes_split(words, 1)
    expected = 0xAABBCCDD
    for j in range(4):
        assert torch.all(planes[j] == (expected & 0xFF)).item()
        expected >>= 8


@pytest.mark.gpu
@pytest.mark.parametrize("wb,pb", CONFIGS)
@pytest.mark.parametrize("n", [0, 1, 15, 16, 17, 1000, 1 << 20, (1 << 22) + 7])
def test_split_join_match_numpy(cuda, wb, pb, n):
    import torch

    rng = np.random.default_rng(n * 31 + wb * 7 + pb)
    host = rng.integers(0, 1 << 62, n, dtype=np.int64).astype(np.uint64 if wb == 8 else np.uint32)
    dt = torch.int64 if wb == 8 else torch.int32
    words = torch.from_numpy(host.view(np.int64 if wb == 8 else np.int32)).to("cuda", dt)
    planes = gb.planes_split(words, pb)
    assert len(planes) == wb // pb
    for got, want in zip(planes, _numpy_planes(host, pb)):
        assert np.array_equal(got.cpu().numpy().view(want.dtype), want)
    if n:
        back = gb.planes_join(planes, wb)
        assert torch.equal(back, words)
