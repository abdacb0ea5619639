"""gary_b200 -- B200-native subgraph counting (triangles, 4-cycles, 4-cliques).

Python host mirror of the reference's DeviceGraphCtx / graph_query call
surface, over the C ABI in include/gary_b200.h (libgary_b200.so).  All
compute runs in the CUDA library; this module only moves pointers.

    import numpy as np, gary_b200 as gb
    src, dst = gb.gen_er(16384, 131072, seed=1)
    ptr, idx = gb.csr_from_edges(src, dst, 16384)       # symmetric CSR (host)
    with gb.Graph.upload(ptr, idx, 16384) as g:          # DeviceGraphCtx::loadFromHost
        t = g.count(gb.GARY_PATTERN_TRIANGLE)            # triangleCountHom
"""
from __future__ import annotations

import ctypes as C
from typing import Any

import numpy as np

from ._lib import *  # noqa: F401,F403  (constants, GaryError)
from ._lib import (
    CountStats,
    DeviceCOO,
    DeviceCSR,
    GaryError,
    GraphInfo,
    check,
    load,
)

__all__ = [
    "Graph",
    "DeviceCsr",
    "csr_from_edges",
    "gen_er",
    "gen_rmat",
    "gen_rmat_device",
    "GaryError",
    "load",
]


def _is_torch(x: Any) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x: Any, dtype) -> tuple[int, bool]:
    """(address, on_device) of a numpy array or torch tensor of `dtype`."""
    if x is None:
        return 0, False
    if _is_torch(x):
        import torch

        want = {np.uint32: (torch.uint32, torch.int32), np.uint64: (torch.uint64, torch.int64)}[dtype]
        if x.dtype not in want:
            raise TypeError(f"expected a tensor of {dtype.__name__}, got {x.dtype}")
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return x.data_ptr(), x.is_cuda
    if not isinstance(x, np.ndarray) or x.dtype != dtype or not x.flags.c_contiguous:
        raise TypeError(f"expected a contiguous numpy array of {np.dtype(dtype).name}")
    return x.ctypes.data, False


def _stream(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


class Graph:
    """Device graph handle; the counterpart of DeviceGraphCtx
    (include/DeviceGraph.cuh:75-133)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    # -- lifetime -----------------------------------------------------------
    @classmethod
    def upload(cls, ptr, idx, n: int, flags: int = 0, stream=None) -> "Graph":
        """DeviceGraphCtx::loadFromHost + degree orientation on the device."""
        p, pdev = _ptr(ptr, np.uint64)
        i, idev = _ptr(idx, np.uint32)
        if pdev != idev:
            raise ValueError("ptr and idx must both be on the host or both on the device")
        nnz = int(idx.numel() if _is_torch(idx) else idx.size)
        if pdev:
            flags |= GARY_INPUT_DEVICE  # noqa: F405
        out = C.c_void_p()
        check(load().gary_graph_upload(p, i or None, n, nnz, flags, _stream(stream), C.byref(out)),
              "gary_graph_upload")
        return cls(out.value)

    def free(self) -> None:
        if self._h:
            check(load().gary_graph_free(self._h), "gary_graph_free")
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    def __del__(self):
        try:
            if self._h:
                load().gary_graph_free(self._h)
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- queries --------------------------------------------------------------
    def info(self) -> dict:
        inf = GraphInfo()
        check(load().gary_graph_get_info(self._h, C.byref(inf)), "gary_graph_get_info")
        return {k: getattr(inf, k) for k, _ in GraphInfo._fields_}

    def device_csr(self) -> DeviceCSR:
        v = DeviceCSR()
        check(load().gary_graph_device_csr(self._h, C.byref(v)), "gary_graph_device_csr")
        return v

    def device_coo(self) -> DeviceCOO:
        v = DeviceCOO()
        check(load().gary_graph_device_coo(self._h, C.byref(v)), "gary_graph_device_coo")
        return v

    def download(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Oriented CSR (unpadded) on the host and the rank -> caller id map."""
        inf = self.info()
        ptr = np.zeros(inf["n"] + 1, np.uint64)
        idx = np.zeros(max(inf["m"], 1), np.uint32)
        perm = np.zeros(inf["n"], np.uint32)
        check(load().gary_graph_download(self._h, ptr.ctypes.data, idx.ctypes.data, perm.ctypes.data),
              "gary_graph_download")
        return ptr, idx[: inf["m"]], perm

    # -- counting -------------------------------------------------------------
    def count(self, pattern: int = 3, sched: int = 0, stream=None) -> int:
        """uint64 count of `pattern` (graph_query::triangleCountHom for K3)."""
        out = C.c_uint64()
        check(load().gary_count(self._h, pattern, sched, _stream(stream), C.byref(out)), "gary_count")
        return int(out.value)

    def count_async(self, out_dev, pattern: int = 3, sched: int = 0, stream=None) -> None:
        """Asynchronous count into a device uint64 word (torch tensor)."""
        p, dev = _ptr(out_dev, np.uint64)
        if not dev:
            raise ValueError("count_async needs a device tensor")
        check(load().gary_count_async(self._h, pattern, sched, _stream(stream), p), "gary_count_async")

    def status(self, stream=None) -> int:
        """Status of the last counting launch (gary_count_status): waits for
        `stream` and returns GARY_OK, GARY_ERR_TIMEOUT or GARY_ERR_INTERNAL."""
        return load().gary_count_status(self._h, _stream(stream))

    def check_status(self, stream=None) -> None:
        """Raise GaryError when the last counting launch reported a failure."""
        check(self.status(stream), "gary_count_status")

    def last_stats(self) -> dict:
        """Kernel time, tiles, CTA tiles per set path (bitmap, buckets, staged,
        sampled), the error word and the triangle plan's probe count of the
        last count (after its stream is synchronised)."""
        st = CountStats()
        check(load().gary_count_last_stats(self._h, C.byref(st)), "gary_count_last_stats")
        return {"kernel_ms": st.kernel_ms, "tiles": st.tiles, "cta_tiles": st.cta_tiles,
                "cta_path_tiles": dict(zip(("bitmap", "buckets", "staged", "sampled"), st.cta_path_tiles)),
                "error": st.error, "work": st.work, "makespan_ms": st.makespan_ms,
                "mean_cta_finish_ms": st.mean_cta_finish_ms}


class DeviceCsr:
    """Device-resident symmetric CSR built by gary_csr_from_edges."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    def shape(self) -> tuple[int, int]:
        n = C.c_uint32()
        nnz = C.c_uint64()
        check(load().gary_csr_info(self._h, C.byref(n), C.byref(nnz)), "gary_csr_info")
        return n.value, nnz.value

    def device_ptrs(self) -> tuple[int, int]:
        p = C.c_void_p()
        i = C.c_void_p()
        check(load().gary_csr_device_ptrs(self._h, C.byref(p), C.byref(i)), "gary_csr_device_ptrs")
        return p.value or 0, i.value or 0

    def download(self, ptr: np.ndarray | None = None, idx: np.ndarray | None = None):
        n, nnz = self.shape()
        ptr = np.empty(n + 1, np.uint64) if ptr is None else ptr
        idx = np.empty(max(nnz, 1), np.uint32) if idx is None else idx
        check(load().gary_csr_download(self._h, ptr.ctypes.data, idx.ctypes.data), "gary_csr_download")
        return ptr, idx[:nnz]

    def free(self) -> None:
        if self._h:
            check(load().gary_csr_free(self._h), "gary_csr_free")
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    def __del__(self):
        try:
            if self._h:
                load().gary_csr_free(self._h)
        except Exception:
            pass


def csr_from_edges_device(src, dst, n: int, stream=None) -> DeviceCsr:
    s, sdev = _ptr(src, np.uint32)
    d, ddev = _ptr(dst, np.uint32)
    m = int(src.numel() if _is_torch(src) else src.size)
    flags = GARY_INPUT_DEVICE if sdev else 0  # noqa: F405
    out = C.c_void_p()
    check(load().gary_csr_from_edges(s or None, d or None, m, n, flags, _stream(stream), C.byref(out)),
          "gary_csr_from_edges")
    return DeviceCsr(out.value)


def csr_from_edges(src, dst, n: int, stream=None) -> tuple[np.ndarray, np.ndarray]:
    """Symmetric sorted CSR (dedup, no loops) built on the device, returned on the host."""
    with csr_from_edges_device(src, dst, n, stream) as c:
        return c.download()


def gen_er(n: int, m: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    src = np.empty(m, np.uint32)
    dst = np.empty(m, np.uint32)
    check(load().gary_gen_er(n, m, seed, src.ctypes.data, dst.ctypes.data), "gary_gen_er")
    return src, dst


def gen_rmat(scale: int, seed: int, count: int, first: int = 0) -> tuple[np.ndarray, np.ndarray]:
    src = np.empty(count, np.uint32)
    dst = np.empty(count, np.uint32)
    check(load().gary_gen_rmat(scale, seed, first, count, src.ctypes.data, dst.ctypes.data),
          "gary_gen_rmat")
    return src, dst


def gen_rmat_device(scale: int, seed: int, count: int, first: int = 0, stream=None):
    import torch

    src = torch.empty(count, dtype=torch.int32, device="cuda")
    dst = torch.empty(count, dtype=torch.int32, device="cuda")
    check(load().gary_gen_rmat_device(scale, seed, first, count, src.data_ptr(), dst.data_ptr(),
                                      _stream(stream)), "gary_gen_rmat_device")
    return src, dst


# ---- the reference's graph binaries (cereal binary archive layout) --------
GARY_BIN_CSR = 0
GARY_BIN_COO = 1


def bin_info(path) -> tuple[int, int, int]:
    """(format, n, nnz) of a graph binary written by the reference's
    saveToBinary (format GARY_BIN_CSR or GARY_BIN_COO)."""
    fmt, n, nnz = C.c_uint32(), C.c_uint32(), C.c_uint64()
    check(load().gary_bin_info(str(path).encode(), C.byref(fmt), C.byref(n), C.byref(nnz)), "gary_bin_info")
    return fmt.value, n.value, nnz.value


def read_bin_csr(path) -> tuple[np.ndarray, np.ndarray]:
    """(ptr uint64[n+1], idx uint32[nnz]) of a CSR graph binary, e.g. the
    reference's csr_dag.bin (loadFromBinary<GraphCSR>)."""
    fmt, n, nnz = bin_info(path)
    if fmt != GARY_BIN_CSR:
        raise GaryError(-4, f"{path} holds a COO graph, not a CSR")
    ptr = np.empty(n + 1, np.uint64)
    idx = np.empty(max(nnz, 1), np.uint32)
    check(load().gary_bin_read_csr(str(path).encode(), ptr.ctypes.data, idx.ctypes.data), "gary_bin_read_csr")
    return ptr, idx[:nnz]


def read_bin_coo(path) -> tuple[int, np.ndarray, np.ndarray]:
    """(n, src, dst) of a COO graph binary (loadFromBinary<GraphCOO>)."""
    fmt, n, nnz = bin_info(path)
    if fmt != GARY_BIN_COO:
        raise GaryError(-4, f"{path} holds a CSR graph, not a COO")
    src = np.empty(max(nnz, 1), np.uint32)
    dst = np.empty(max(nnz, 1), np.uint32)
    check(load().gary_bin_read_coo(str(path).encode(), src.ctypes.data, dst.ctypes.data), "gary_bin_read_coo")
    return n, src[:nnz], dst[:nnz]


def write_bin_csr(path, ptr, idx) -> None:
    """Write a CSR graph binary in the reference's layout (saveToBinary)."""
    ptr = np.ascontiguousarray(ptr, np.uint64)
    idx = np.ascontiguousarray(idx, np.uint32)
    n = len(ptr) - 1
    check(load().gary_bin_write_csr(str(path).encode(), ptr.ctypes.data, idx.ctypes.data if len(idx) else None,
                                    n, int(ptr[-1])), "gary_bin_write_csr")


__all__ += ["bin_info", "read_bin_csr", "read_bin_coo", "write_bin_csr", "GARY_BIN_CSR", "GARY_BIN_COO"]


# ---- byte planes ------------------------------------------------------------
def planes_split(words, plane_bytes: int, stream=None) -> list:
    """Split a CUDA tensor of 4- or 8-byte words (int32/uint32/int64) into
    word_bytes / plane_bytes CUDA tensors of plane_bytes-wide entries (plane j
    = byte group j of every word, least significant first)."""
    import torch

    wb = words.element_size()
    k = wb // plane_bytes
    dt = {1: torch.uint8, 2: torch.int16, 4: torch.int32}[plane_bytes]
    planes = [torch.empty(words.numel(), dtype=dt, device=words.device) for _ in range(k)]
    arr = (C.c_void_p * k)(*[p.data_ptr() for p in planes])
    check(load().gary_planes_split(words.data_ptr(), words.numel(), wb, plane_bytes, arr, _stream(stream)),
          "gary_planes_split")
    return planes


def planes_join(planes: list, word_bytes: int, stream=None):
    """Inverse of planes_split: a CUDA tensor of word_bytes-wide words."""
    import torch

    n = planes[0].numel()
    pb = planes[0].element_size()
    words = torch.empty(n, dtype=torch.int32 if word_bytes == 4 else torch.int64, device=planes[0].device)
    arr = (C.c_void_p * len(planes))(*[p.data_ptr() for p in planes])
    check(load().gary_planes_join(arr, n, word_bytes, pb, words.data_ptr(), _stream(stream)), "gary_planes_join")
    return words


__all__ += ["planes_split", "planes_join"]
