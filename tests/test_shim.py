"""The C++ shim layer (include/gary/): the host side of its search functions
against the reference's own search results (CPU), and a program written the
way the reference's tests use DeviceGraphCtx / graph_query::triangleCountHom /
the ops intersections, run on the GPU and checked against the oracle."""
from __future__ import annotations

import ctypes as C
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from vectors import search_case, unpack_bits

ROOT = Path(__file__).resolve().parents[1]
CPP = ROOT / "tests" / "cpp"
BIN = CPP / "_bin"


def _make(target: str) -> Path:
    out = BIN / target
    if not out.exists():
        subprocess.run(["make", "-s", "-C", str(CPP), f"_bin/{target}"], check=True)
    return out


@pytest.fixture(scope="module")
def search_lib():
    lib = C.CDLL(str(_make("libsearch_host.so")))
    P = C.c_void_p
    lib.shim_binary_search.argtypes = [P, C.c_uint64, P, C.c_uint64, P]
    lib.shim_binary_search_pos.argtypes = [P, C.c_uint64, P, C.c_uint64, P, P]
    lib.shim_search_2phase.argtypes = [P, C.c_uint64, P, C.c_uint64, P, P]
    return lib


def _ptr(a):
    return a.ctypes.data


def test_shim_search_matches_reference_golden(golden, search_lib):
    """binary_search, build_cache and binary_search_2phase of the shim give the
    reference's recorded results (include/ops/Search.cuh run on the host)."""
    for c in golden["search"]:
        lst, keys = search_case(c["seed"], c["n_list"], c["n_keys"], c["lo"], c["hi"], c["sort_keys"])
        lst = np.ascontiguousarray(lst.astype(np.uint32))
        keys = np.ascontiguousarray(keys.astype(np.uint32))
        n = len(keys)
        f1 = np.zeros(n, np.uint8)
        f2 = np.zeros(n, np.uint8)
        cache = np.zeros(32, np.uint32)
        search_lib.shim_binary_search(_ptr(lst), len(lst), _ptr(keys), n, _ptr(f1))
        search_lib.shim_search_2phase(_ptr(lst), len(lst), _ptr(keys), n, _ptr(cache), _ptr(f2))
        assert np.array_equal(f1, unpack_bits(c["found"], n))
        assert np.array_equal(f2, unpack_bits(c["found_2phase"], n))
        assert cache.tolist() == [x & 0xFFFFFFFF for x in c["cache32"]]


@pytest.mark.parametrize("n", [0, 1, 2, 31, 32, 33, 1000, 70001])
def test_shim_search_pos_and_edges(search_lib, n):
    """pos semantics of binary_search(span, key, pos) (Search.cuh:63-81): the
    key's index, else the index of the last element < key, -1 when none; and
    2-phase membership on short, exact-multiple and long lists."""
    r = np.random.default_rng(n)
    lst = np.unique(r.integers(0, 4 * n + 10, size=n)).astype(np.uint32)
    keys = r.integers(0, 4 * n + 12, size=4000).astype(np.uint32)
    found = np.zeros(len(keys), np.uint8)
    pos = np.zeros(len(keys), np.int32)
    search_lib.shim_binary_search_pos(_ptr(lst), len(lst), _ptr(keys), len(keys), _ptr(found), _ptr(pos))
    ins = np.searchsorted(lst, keys, side="left")
    hit = (ins < len(lst)) & (lst[np.minimum(ins, max(len(lst) - 1, 0))] == keys) if len(lst) else np.zeros(len(keys), bool)
    assert np.array_equal(found.astype(bool), hit)
    assert np.array_equal(pos, np.where(hit, ins, ins - 1))
    f2 = np.zeros(len(keys), np.uint8)
    cache = np.zeros(32, np.uint32)
    search_lib.shim_search_2phase(_ptr(lst), len(lst), _ptr(keys), len(keys), _ptr(cache), _ptr(f2))
    assert np.array_equal(f2.astype(bool), hit)
    if len(lst):
        assert np.array_equal(cache, lst[(np.arange(32, dtype=np.uint64) * len(lst) // 32).astype(np.int64)])


@pytest.mark.gpu
@pytest.mark.parametrize("scale,ef,seed", [(12, 8, 1), (14, 16, 5)])
def test_shim_program_on_gpu(cuda, scale, ef, seed):
    """The shim program: reference-style kernels, the library's own counts and
    the ops intersections all agree with the oracle on the same graph."""
    import gary_b200 as gb

    exe = _make("shim_test")
    r = subprocess.run([str(exe), str(scale), str(ef), str(seed)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    src, dst = gb.gen_rmat(scale, seed, ef << scale)
    ptr, idx = gb.csr_from_edges(src, dst, 1 << scale)
    dptr, didx = O.orient(ptr, idx)
    assert res["cpu"] == res["fast"] == O.tri_count(dptr, didx)
    assert res["hom_cache"] == res["hom_nocache"] == res["hom_chunked"] == res["cpu"]
    assert res["legacy_u32"] == res["cpu"] & 0xFFFFFFFF
    assert res["c4"] == O.c4_count(ptr, idx)
    assert res["k4"] == O.k4_count(dptr, didx)
    assert res["pair_mismatches"] == 0 and res["search_mismatches"] == 0 and res["views_ok"]
