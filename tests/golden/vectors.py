"""Deterministic input builders shared by make_golden.py and the tests.

Only numpy integer arithmetic (wrapping uint64), so the inputs are the same on
every machine and numpy version.
"""
from __future__ import annotations

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix(x: np.ndarray) -> np.ndarray:
    """splitmix64 finalizer, vectorised (uint64 wraps)."""
    z = np.asarray(x, np.uint64).copy()
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def stream(seed: int, count: int, salt: int = 0) -> np.ndarray:
    """`count` pseudo-random uint64 values keyed by (seed, salt)."""
    base = splitmix(np.array([seed ^ (salt << 32) ^ 0x1234567], np.uint64))[0]
    with np.errstate(over="ignore"):
        return splitmix(base + np.arange(count, dtype=np.uint64) * GOLDEN)


def uniform_ints(seed: int, count: int, lo: int, hi: int, salt: int = 0) -> np.ndarray:
    """Integers in [lo, hi) (multiply-shift, no modulo bias beyond 2^-32)."""
    r = stream(seed, count, salt) >> np.uint64(32)
    span = np.uint64(hi - lo)
    with np.errstate(over="ignore"):
        return (np.uint64(lo) + ((r * span) >> np.uint64(32))).astype(np.int64)


def edge_checksum(src: np.ndarray, dst: np.ndarray) -> str:
    """Order-sensitive 64-bit digest of an edge list, as hex."""
    s = np.asarray(src, np.uint64)
    d = np.asarray(dst, np.uint64)
    with np.errstate(over="ignore"):
        k = (s << np.uint64(32)) | d
        h = splitmix(k + np.arange(len(k), dtype=np.uint64) * GOLDEN)
        return f"{int(np.bitwise_xor.reduce(h)) if len(h) else 0:016x}:{int(h.sum(dtype=np.uint64)) if len(h) else 0:016x}"


def search_case(seed: int, n_list: int, n_keys: int, lo: int, hi: int, sort_keys: bool):
    """A sorted list (duplicates possible) and keys, like test/SearchTest.cu:196-210."""
    lst = np.sort(uniform_ints(seed, n_list, lo, hi, salt=1)).astype(np.int32)
    keys = uniform_ints(seed, n_keys, lo, hi, salt=2).astype(np.int32)
    if sort_keys:
        keys = np.sort(keys)
    return lst, keys


def pack_bits(b: np.ndarray) -> str:
    return np.packbits(np.asarray(b, np.uint8)).tobytes().hex()


def unpack_bits(s: str, n: int) -> np.ndarray:
    return np.unpackbits(np.frombuffer(bytes.fromhex(s), np.uint8))[:n]
