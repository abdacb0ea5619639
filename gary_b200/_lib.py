"""ctypes binding of libgary_b200.so (declarations mirror include/gary_b200.h).

The library is the product: there is no Python or CPU fallback.  Loading fails
loudly when the shared object is missing; build it with
``python -m gary_b200.build`` (``__graft_entry__.build()`` does it too).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(os.environ.get("GARY_B200_LIB", Path(__file__).resolve().parent / "libgary_b200.so"))

GARY_OK = 0
GARY_ERR_INVALID = -1
GARY_ERR_CUDA = -2
GARY_ERR_OOM = -3
GARY_ERR_INPUT = -4
GARY_ERR_TIMEOUT = -5
GARY_ERR_UNSUPPORTED = -6
GARY_ERR_INTERNAL = -7

GARY_INPUT_SYMMETRIC = 0x0
GARY_INPUT_DAG = 0x1
GARY_INPUT_DEVICE = 0x2
GARY_KEEP_IDS = 0x4
GARY_VALIDATE = 0x8

GARY_PATTERN_TRIANGLE = 3
GARY_PATTERN_4CYCLE = 4
GARY_PATTERN_4CLIQUE = 5

GARY_SCHED_PLAIN = 0
GARY_SCHED_LEARNED = 1

GARY_ISECT_AUTO = 0
GARY_ISECT_MERGE = 1
GARY_ISECT_SEARCH = 2
GARY_ISECT_BITMAP = 3


class GraphInfo(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("max_degree", C.c_uint32),
        ("max_out_degree", C.c_uint32),
        ("relabeled", C.c_uint32),
        ("m", C.c_uint64),
        ("adj_words", C.c_uint64),
        ("wedges", C.c_uint64),
        ("out_deg_sq", C.c_uint64),
        ("alg_bytes", C.c_uint64),
        ("device_bytes", C.c_uint64),
    ]


class DeviceCSR(C.Structure):
    _fields_ = [
        ("m", C.c_uint32),
        ("nnz", C.c_uint64),
        ("indPtr", C.c_void_p),
        ("colIdx", C.c_void_p),
        ("deg", C.c_void_p),
    ]


class DeviceCOO(C.Structure):
    _fields_ = [
        ("m", C.c_uint32),
        ("nnz", C.c_uint64),
        ("rowIdx", C.c_void_p),
        ("colIdx", C.c_void_p),
        ("deg", C.c_void_p),
    ]


class CountStats(C.Structure):
    _fields_ = [
        ("kernel_ms", C.c_float),
        ("tiles", C.c_uint32),
        ("cta_tiles", C.c_uint32),
        ("cta_path_tiles", C.c_uint32 * 4),  # bitmap, buckets, staged whole, sampled
        ("error", C.c_uint32),
        ("work", C.c_uint64),
        ("makespan_ms", C.c_float),
        ("mean_cta_finish_ms", C.c_float),
    ]


_P = C.c_void_p
_U32 = C.c_uint32
_U64 = C.c_uint64
_I32 = C.c_int32
_INT = C.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "gary_last_error": (C.c_char_p, []),
    "gary_abi_version": (_INT, []),
    "gary_graph_upload": (_INT, [_P, _P, _U32, _U64, _U32, _P, C.POINTER(_P)]),
    "gary_graph_free": (_INT, [_P]),
    "gary_graph_get_info": (_INT, [_P, C.POINTER(GraphInfo)]),
    "gary_graph_device_csr": (_INT, [_P, C.POINTER(DeviceCSR)]),
    "gary_graph_device_coo": (_INT, [_P, C.POINTER(DeviceCOO)]),
    "gary_graph_download": (_INT, [_P, _P, _P, _P]),
    "gary_count": (_INT, [_P, _INT, _INT, _P, C.POINTER(_U64)]),
    "gary_count_async": (_INT, [_P, _INT, _INT, _P, _P]),
    "gary_count_shard_async": (_INT, [_P, _INT, _INT, _U32, _U32, _P, _P]),
    "gary_count_last_stats": (_INT, [_P, C.POINTER(CountStats)]),
    "gary_count_status": (_INT, [_P, _P]),
    "gary_count_triangles_noalloc": (_INT, [_P, _P, _P, _U32, _P, _P]),
    "gary_tune": (_INT, [C.c_char_p, _U64]),
    "gary_batch_upload": (_INT, [_P, _U32, _P, _P, _U32, _U64, _U32, _P, C.POINTER(_P)]),
    "gary_batch_count_async": (_INT, [_P, _INT, _P, _P, _P]),
    "gary_batch_capture": (_INT, [_P, _INT, _P, _P, _P, C.POINTER(_P)]),
    "gary_exec_launch": (_INT, [_P, _P]),
    "gary_exec_free": (_INT, [_P]),
    "gary_gen_ba": (_INT, [_U32, _U32, _U64, _P, _P, C.POINTER(_U64)]),
    "gary_mlp_param_count": (_INT, []),
    "gary_mlp_init": (_INT, [_U64, _P]),
    "gary_mlp_forward": (_INT, [_P, _P, _U64, _INT, _P, _P]),
    "gary_mlp_grad": (_INT, [_P, _P, _P, _P, _U64, C.c_float, _P, _P, _P]),
    "gary_mlp_adam": (_INT, [_P, _P, _P, _P, _U32, C.c_float, _P]),
    "gary_mlp_save": (_INT, [C.c_char_p, _P]),
    "gary_mlp_load": (_INT, [C.c_char_p, _P]),
    "gary_set_cost_model": (_INT, [_P]),
    "gary_tc_features": (_INT, [_P, _P, _P, _P]),
    "gary_tc_profile": (_INT, [_P, _INT, _P, _P, _P]),
    "gary_intersect_batch": (_INT, [_U64, _P, _P, _P, _P, _P, _P, _INT, _P, _P, _P, _P, _P, _P]),
    "gary_intersect_num_batch": (_INT, [_U64, _P, _P, _P, _P, _P, _P, _INT, _P, _P, _P, _P, _P, _P, _P]),
    "gary_search_batch": (_INT, [_P, _U64, _P, _U64, _U32, _P, _P, _P]),
    "gary_zipf_table": (_INT, [_U32, C.c_double, _P]),
    "gary_gen_pair_host": (_INT, [_U64, _U64, _U32, _P, C.c_double, _U64, _P, _P, _P, _P]),
    "gary_gen_pairs_lengths": (_INT, [_U64, _U64, _U64, _U32, _P, _P, _P, _P, _P, _P]),
    "gary_gen_pairs_values": (_INT, [_U64, _U64, _U64, _U32, _P, C.c_double, _U64, _P, _P, _P, _P, _P, _P, _P]),
    "gary_graph_drop_plans": (_INT, [_P]),
    "gary_csr_from_edges": (_INT, [_P, _P, _U64, _U32, _U32, _P, C.POINTER(_P)]),
    "gary_csr_info": (_INT, [_P, C.POINTER(_U32), C.POINTER(_U64)]),
    "gary_csr_device_ptrs": (_INT, [_P, C.POINTER(_P), C.POINTER(_P)]),
    "gary_csr_download": (_INT, [_P, _P, _P]),
    "gary_csr_free": (_INT, [_P]),
    "gary_planes_split": (_INT, [_P, _U64, _INT, _INT, _P, _P]),
    "gary_planes_join": (_INT, [_P, _U64, _INT, _INT, _P, _P]),
    "gary_bin_info": (_INT, [C.c_char_p, _P, _P, _P]),
    "gary_bin_read_csr": (_INT, [C.c_char_p, _P, _P]),
    "gary_bin_read_coo": (_INT, [C.c_char_p, _P, _P]),
    "gary_bin_write_csr": (_INT, [C.c_char_p, _P, _P, _U32, _U64]),
    "gary_gen_er": (_INT, [_U32, _U64, _U64, _P, _P]),
    "gary_gen_rmat": (_INT, [_INT, _U64, _U64, _U64, _P, _P]),
    "gary_gen_rmat_device": (_INT, [_INT, _U64, _U64, _U64, _P, _P, _P]),
}

_lib = None


def load() -> C.CDLL:
    """Load (once) and return the library, with every signature declared."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: the CUDA library is the only implementation of this "
            "path (no CPU fallback). Build it with `python -m gary_b200.build`."
        )
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class GaryError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = load().gary_last_error()
        self.status = status
        super().__init__(f"{where} failed with status {status}: {msg.decode() if msg else ''}")


def check(status: int, where: str) -> None:
    if status != GARY_OK:
        raise GaryError(status, where)
