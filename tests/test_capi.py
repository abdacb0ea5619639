"""The C ABI without a GPU: the library loads, exports every declared symbol,
and rejects bad arguments before touching the device."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

import gary_b200 as gb
from gary_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(gary_[a-z0-9_]+)\s*\(", text))
    return names


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares each one
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_abi_version():
    assert _lib.load().gary_abi_version() == 2


def test_argument_errors_without_device():
    lib = _lib.load()
    out = C.c_void_p()
    # NULL out
    assert lib.gary_graph_upload(None, None, 4, 0, 0, None, None) == _lib.GARY_ERR_INVALID
    assert b"out" in lib.gary_last_error()
    # n = 0
    ptr = np.zeros(1, np.uint64)
    assert lib.gary_graph_upload(ptr.ctypes.data, None, 0, 0, 0, None, C.byref(out)) == _lib.GARY_ERR_INVALID
    # host ptr inconsistent with nnz
    ptr = np.array([0, 1, 2], np.uint64)
    idx = np.array([1, 0], np.uint32)
    assert lib.gary_graph_upload(ptr.ctypes.data, idx.ctypes.data, 2, 3, 0, None, C.byref(out)) == _lib.GARY_ERR_INVALID
    # counting on NULL graph
    v = C.c_uint64()
    assert lib.gary_count(None, 3, 0, None, C.byref(v)) == _lib.GARY_ERR_INVALID
    assert lib.gary_count_async(None, 3, 0, None, None) == _lib.GARY_ERR_INVALID
    # generators
    s = np.zeros(4, np.uint32)
    assert lib.gary_gen_er(3, 4, 0, s.ctypes.data, s.ctypes.data) == _lib.GARY_ERR_INVALID
    assert lib.gary_gen_rmat(0, 0, 0, 4, s.ctypes.data, s.ctypes.data) == _lib.GARY_ERR_INVALID
    assert lib.gary_gen_rmat(32, 0, 0, 4, s.ctypes.data, s.ctypes.data) == _lib.GARY_ERR_INVALID
    # free(NULL) is a no-op
    assert lib.gary_graph_free(None) == _lib.GARY_OK
    assert lib.gary_csr_free(None) == _lib.GARY_OK


def test_python_errors_raise():
    try:
        gb.gen_er(3, 4, 0)
    except gb.GaryError as e:
        assert e.status == _lib.GARY_ERR_INVALID
        assert "m exceeds" in str(e)
    else:
        raise AssertionError("expected GaryError")


def test_header_compiles_as_c():
    """include/gary_b200.h is plain C (no CUDA or C++ types in signatures)."""
    import subprocess
    import tempfile

    with tempfile.TemporaryDirectory() as d:
        src = Path(d) / "t.c"
        src.write_text('#include "gary_b200.h"\nint main(void){return gary_abi_version() != 2;}\n')
        r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", f"-I{ROOT / 'include'}", "-c", str(src),
                            "-o", str(Path(d) / "t.o")], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_tuning_keys_checked():
    """gary_tune validates every key's range on the host (no device needed)."""
    L = _lib.load()
    try:
        for key, bad in (("warp_cap", 4), ("warp_cap", 1024), ("cta_set_words", 100), ("cta_set_words", 32),
                         ("cta_set_words", 32768), ("stage_wait_polls", (1 << 24) + 1), ("min_blocks", 1),
                         ("no_such_key", 1)):
            assert L.gary_tune(key.encode(), bad) == _lib.GARY_ERR_INVALID, (key, bad)
        for key, good in (("warp_cap", 8), ("cta_set_words", 64), ("cta_set_words", 0),
                          ("stage_wait_polls", 0), ("min_blocks", 3)):
            assert L.gary_tune(key.encode(), good) == _lib.GARY_OK, (key, good)
    finally:
        assert L.gary_tune(b"reset", 0) == _lib.GARY_OK


def test_count_status_needs_a_launch():
    L = _lib.load()
    assert L.gary_count_status(None, None) == _lib.GARY_ERR_INVALID
