"""ctypes front end of the CPU oracle and of the reference builds -- TEST
INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs may import this module, and only as the checker or as the timed
reference.  The product (gary_b200) never imports it.

    oracle/_build/liboracle.so     C restatement (oracle.c)
    oracle/_ref/libgary_ref_cpu.so the reference's own host code, compiled in place
    oracle/_ref/libgary_ref_gpu.so the reference's own kernels for sm_100a
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_CPU_SO = HERE / "_ref" / "libgary_ref_cpu.so"
REF_GPU_SO = HERE / "_ref" / "libgary_ref_gpu.so"

_P, _U32, _U64, _I32, _I64, _INT = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_int64, C.c_int

_ORC = {
    "orc_sym_csr": (_I64, [_U32, _I64, _P, _P, _P, _P]),
    "orc_orient": (None, [_U32, _P, _P, _INT, _P, _P]),
    "orc_tri_count": (_U64, [_U32, _P, _P, _INT]),
    "orc_k4_count": (_U64, [_U32, _P, _P, _INT]),
    "orc_c4_count": (_U64, [_U32, _P, _P, _INT]),
    "orc_c4_hom": (_U64, [_U32, _P, _P]),
    "orc_tc_bytes": (None, [_U32, _P, _P, C.POINTER(_U64), C.POINTER(_U64)]),
    "orc_intersect": (_I64, [_P, _I64, _P, _I64, _P]),
    "orc_intersect_batch": (_U64, [_I64, _P, _P, _P, _P, _P, _P, _P, _INT]),
    "orc_binary_search": (_INT, [_P, _I64, _U32]),
    "orc_build_cache": (None, [_P, _I64, _INT, _P]),
    "orc_binary_search_2phase": (_INT, [_P, _I64, _P, _INT, _U32]),
    "orc_mlp_forward": (None, [_P, _P, _I64, _P]),
    "orc_gen_rmat": (None, [_INT, _U64, _U64, _U64, _P, _P]),
    "orc_unique_edges": (_I64, [_U32, _I64, _P, _P, _P, _P, _INT]),
    "orc_mlp_grad": (None, [_P, _P, _P, _P, _I64, C.c_double, _P, C.POINTER(C.c_double)]),
}

_REF_CPU = {
    "ref_last_error": (C.c_char_p, []),
    "ref_dag_from_edges": (_P, [_I32, _I64, _P, _P]),
    "ref_sym_from_edges": (_P, [_I32, _I64, _P, _P]),
    "ref_csr_from_arrays": (_P, [_I32, _I64, _P, _P]),
    "ref_csr_num_v": (_I32, [_P]),
    "ref_csr_num_e": (_I64, [_P]),
    "ref_csr_copy": (None, [_P, _P, _P]),
    "ref_csr_free": (None, [_P]),
    "ref_cpu_tri_count": (_U64, [_P, _I64, _I64, _I64, _I32]),
    "ref_omp_max_threads": (_I32, []),
    "ref_binary_search": (None, [_P, _I64, _P, _I64, _P]),
    "ref_binary_search_pos": (None, [_P, _I64, _P, _I64, _P, _P]),
    "ref_build_cache32": (None, [_P, _I64, _P]),
    "ref_binary_search_2phase": (None, [_P, _I64, _P, _I64, _P]),
}

_REF_GPU = {
    "ref_gpu_last_error": (C.c_char_p, []),
    "ref_gpu_graph_create": (_P, [_I32, _I64, _P, _P]),
    "ref_gpu_graph_free": (None, [_P]),
    "ref_gpu_tri_count": (_INT, [_P, _I32, C.POINTER(_U64), C.POINTER(C.c_float)]),
}

_cache: dict[str, C.CDLL] = {}


def _load(path: Path, sigs: dict) -> C.CDLL:
    key = str(path)
    if key not in _cache:
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (run `make -C oracle`)")
        lib = C.CDLL(key)
        for name, (res, args) in sigs.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _cache[key] = lib
    return _cache[key]


def orc() -> C.CDLL:
    return _load(ORACLE_SO, _ORC)


def ref_cpu() -> C.CDLL:
    return _load(REF_CPU_SO, _REF_CPU)


def ref_gpu() -> C.CDLL:
    return _load(REF_GPU_SO, _REF_GPU)


def have_ref_cpu() -> bool:
    return REF_CPU_SO.exists()


def have_ref_gpu() -> bool:
    return REF_GPU_SO.exists()


def _a(x, dt):
    return np.ascontiguousarray(x, dtype=dt)


# ---- restatement ---------------------------------------------------------
def sym_csr(src, dst, n: int):
    src, dst = _a(src, np.uint32), _a(dst, np.uint32)
    ptr = np.zeros(n + 1, np.uint64)
    idx = np.zeros(max(2 * len(src), 1), np.uint32)
    k = orc().orc_sym_csr(n, len(src), src.ctypes.data, dst.ctypes.data, ptr.ctypes.data, idx.ctypes.data)
    return ptr, idx[:k].copy()


def orient(ptr, idx, by_degree: bool = True):
    ptr, idx = _a(ptr, np.uint64), _a(idx, np.uint32)
    n = len(ptr) - 1
    optr = np.zeros(n + 1, np.uint64)
    oidx = np.zeros(max(len(idx) // 2, 1), np.uint32)
    orc().orc_orient(n, ptr.ctypes.data, idx.ctypes.data, int(by_degree), optr.ctypes.data, oidx.ctypes.data)
    return optr, oidx[: int(optr[-1])].copy()


def tri_count(ptr, idx, threads: int = 0) -> int:
    ptr, idx = _a(ptr, np.uint64), _a(idx, np.uint32)
    return int(orc().orc_tri_count(len(ptr) - 1, ptr.ctypes.data, idx.ctypes.data, threads))


def k4_count(ptr, idx, threads: int = 0) -> int:
    ptr, idx = _a(ptr, np.uint64), _a(idx, np.uint32)
    return int(orc().orc_k4_count(len(ptr) - 1, ptr.ctypes.data, idx.ctypes.data, threads))


def c4_count(sym_ptr, sym_idx, threads: int = 0) -> int:
    ptr, idx = _a(sym_ptr, np.uint64), _a(sym_idx, np.uint32)
    return int(orc().orc_c4_count(len(ptr) - 1, ptr.ctypes.data, idx.ctypes.data, threads))


def c4_hom(sym_ptr, sym_idx) -> int:
    ptr, idx = _a(sym_ptr, np.uint64), _a(sym_idx, np.uint32)
    return int(orc().orc_c4_hom(len(ptr) - 1, ptr.ctypes.data, idx.ctypes.data))


def tc_bytes(ptr, idx) -> tuple[int, int]:
    ptr, idx = _a(ptr, np.uint64), _a(idx, np.uint32)
    w, b = C.c_uint64(), C.c_uint64()
    orc().orc_tc_bytes(len(ptr) - 1, ptr.ctypes.data, idx.ctypes.data, C.byref(w), C.byref(b))
    return int(w.value), int(b.value)


def intersect(a, b, materialise: bool = False):
    a, b = _a(a, np.uint32), _a(b, np.uint32)
    out = np.zeros(max(min(len(a), len(b)), 1), np.uint32) if materialise else None
    k = orc().orc_intersect(a.ctypes.data, len(a), b.ctypes.data, len(b), out.ctypes.data if materialise else None)
    return out[:k].copy() if materialise else int(k)


def intersect_batch(a_off, la, a, b_off, lb, b, threads: int = 0):
    """(per-pair counts, total) by merge over a pair batch, OpenMP over pairs."""
    a_off, b_off = _a(a_off, np.int64), _a(b_off, np.int64)
    la, lb = _a(la, np.int32), _a(lb, np.int32)
    a, b = _a(a, np.uint32), _a(b, np.uint32)
    counts = np.zeros(len(la), np.int64)
    t = orc().orc_intersect_batch(len(la), a_off.ctypes.data, la.ctypes.data, a.ctypes.data,
                                  b_off.ctypes.data, lb.ctypes.data, b.ctypes.data, counts.ctypes.data,
                                  threads)
    return counts, int(t)


def binary_search(lst, keys) -> np.ndarray:
    lst = _a(lst, np.uint32)
    return np.array([orc().orc_binary_search(lst.ctypes.data, len(lst), int(k)) for k in keys], np.uint8)


def build_cache(lst, N: int = 32) -> np.ndarray:
    lst = _a(lst, np.uint32)
    c = np.zeros(N, np.uint32)
    orc().orc_build_cache(lst.ctypes.data, len(lst), N, c.ctypes.data)
    return c


def binary_search_2phase(lst, keys, N: int = 32) -> np.ndarray:
    lst = _a(lst, np.uint32)
    c = build_cache(lst, N)
    return np.array(
        [orc().orc_binary_search_2phase(lst.ctypes.data, len(lst), c.ctypes.data, N, int(k)) for k in keys],
        np.uint8,
    )


def gen_rmat(scale: int, seed: int, count: int, first: int = 0):
    """The seeded RMAT workload's edges, restated (no product library)."""
    src = np.empty(count, np.uint32)
    dst = np.empty(count, np.uint32)
    orc().orc_gen_rmat(scale, seed, first, count, src.ctypes.data, dst.ctypes.data)
    return src, dst


def unique_edges(n: int, src, dst, threads: int = 0):
    """Each undirected edge once, (u < v), loops dropped, sorted by (u, v)."""
    src, dst = _a(src, np.uint32), _a(dst, np.uint32)
    us = np.empty(max(len(src), 1), np.uint32)
    vs = np.empty(max(len(src), 1), np.uint32)
    k = orc().orc_unique_edges(n, len(src), src.ctypes.data, dst.ctypes.data, us.ctypes.data, vs.ctypes.data,
                               threads)
    return us[:k], vs[:k]


def unique_pairs(sym_ptr, sym_idx) -> tuple[np.ndarray, np.ndarray]:
    """Each undirected edge once (u < v) from a symmetric CSR."""
    ptr = np.asarray(sym_ptr, np.int64)
    idx = np.asarray(sym_idx, np.uint32)
    rows = np.repeat(np.arange(len(ptr) - 1, dtype=np.uint32), np.diff(ptr))
    keep = rows < idx
    return rows[keep].copy(), idx[keep].copy()


# ---- the reference's own code ---------------------------------------------
class RefCSR:
    """The reference's GraphCSR built by its own pipeline (src/Graph.cpp)."""

    def __init__(self, handle):
        if not handle:
            raise RuntimeError(ref_cpu().ref_last_error().decode())
        self.h = C.c_void_p(handle)

    @classmethod
    def dag_from_edges(cls, n: int, src, dst) -> "RefCSR":
        src, dst = _a(src, np.int32), _a(dst, np.int32)
        return cls(ref_cpu().ref_dag_from_edges(n, len(src), src.ctypes.data, dst.ctypes.data))

    @classmethod
    def from_arrays(cls, ptr, idx) -> "RefCSR":
        ptr, idx = _a(ptr, np.int64), _a(idx, np.int32)
        return cls(ref_cpu().ref_csr_from_arrays(len(ptr) - 1, len(idx), ptr.ctypes.data, idx.ctypes.data))

    def arrays(self):
        L = ref_cpu()
        n, m = L.ref_csr_num_v(self.h), L.ref_csr_num_e(self.h)
        ptr = np.zeros(n + 1, np.int64)
        idx = np.zeros(max(m, 1), np.int32)
        L.ref_csr_copy(self.h, ptr.ctypes.data, idx.ctypes.data)
        return ptr, idx[:m]

    def tri_count(self, v_begin: int = 0, v_end: int | None = None, stride: int = 1, threads: int = 0) -> int:
        L = ref_cpu()
        if v_end is None:
            v_end = L.ref_csr_num_v(self.h)
        return int(L.ref_cpu_tri_count(self.h, v_begin, v_end, stride, threads))

    def free(self):
        if self.h:
            ref_cpu().ref_csr_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def ref_search(lst, keys):
    """(found, found_2phase) from the reference's host search templates."""
    lst, keys = _a(lst, np.int32), _a(keys, np.int32)
    f1 = np.zeros(len(keys), np.uint8)
    f2 = np.zeros(len(keys), np.uint8)
    ref_cpu().ref_binary_search(lst.ctypes.data, len(lst), keys.ctypes.data, len(keys), f1.ctypes.data)
    ref_cpu().ref_binary_search_2phase(lst.ctypes.data, len(lst), keys.ctypes.data, len(keys), f2.ctypes.data)
    return f1, f2


def ref_build_cache32(lst) -> np.ndarray:
    lst = _a(lst, np.int32)
    c = np.zeros(32, np.int32)
    ref_cpu().ref_build_cache32(lst.ctypes.data, len(lst), c.ctypes.data)
    return c


class RefGpuGraph:
    """The reference's DeviceGraphCtx + triangleCountHom on the GPU."""

    HOM_CACHE, HOM_CACHE_CHUNKED, HOM_NOCACHE, LEGACY = 0, 1, 2, 3

    def __init__(self, ptr, idx):
        ptr, idx = _a(ptr, np.int64), _a(idx, np.int32)
        h = ref_gpu().ref_gpu_graph_create(len(ptr) - 1, len(idx), ptr.ctypes.data, idx.ctypes.data)
        if not h:
            raise RuntimeError(ref_gpu().ref_gpu_last_error().decode())
        self.h = C.c_void_p(h)

    def tri_count(self, variant: int = 0) -> tuple[int, float]:
        c = C.c_uint64()
        ms = C.c_float()
        st = ref_gpu().ref_gpu_tri_count(self.h, variant, C.byref(c), C.byref(ms))
        if st != 0:
            raise RuntimeError(ref_gpu().ref_gpu_last_error().decode())
        return int(c.value), float(ms.value)

    def free(self):
        if self.h:
            ref_gpu().ref_gpu_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def mlp_forward(params, x) -> np.ndarray:
    params, x = _a(params, np.float32), _a(x, np.float32)
    y = np.zeros((len(x), 4), np.float64)
    orc().orc_mlp_forward(params.ctypes.data, x.ctypes.data, len(x), y.ctypes.data)
    return y


def mlp_grad(params, x, t, mask, norm: float):
    params, x, t, mask = _a(params, np.float32), _a(x, np.float32), _a(t, np.float32), _a(mask, np.uint8)
    g = np.zeros(len(params), np.float64)
    loss = C.c_double()
    orc().orc_mlp_grad(params.ctypes.data, x.ctypes.data, t.ctypes.data, mask.ctypes.data, len(x), norm,
                       g.ctypes.data, C.byref(loss))
    return g, loss.value
