"""Host mirror of the batched set operations (include/ops in the reference).

    cdf = zipf_table(65536, 1.2)
    batch = PairBatch.generate(seed=1, first=0, npairs=1 << 20, cdf=cdf, overlap=0.25)
    counts, total = intersect(batch, GARY_ISECT_MERGE)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import (
    GARY_ISECT_AUTO,
    GARY_ISECT_BITMAP,
    GARY_ISECT_MERGE,
    GARY_ISECT_SEARCH,
    check,
    load,
)

VARIANTS = {"auto": GARY_ISECT_AUTO, "merge": GARY_ISECT_MERGE, "search": GARY_ISECT_SEARCH,
            "bitmap": GARY_ISECT_BITMAP}
RANGE = 1 << 26


def _s(stream) -> int:
    if stream is None:
        return 0
    return stream if isinstance(stream, int) else stream.cuda_stream


def zipf_table(nmax: int = 65536, s: float = 1.2) -> np.ndarray:
    cdf = np.zeros(nmax, np.uint64)
    check(load().gary_zipf_table(nmax, s, cdf.ctypes.data), "gary_zipf_table")
    return cdf


def gen_pair_host(seed: int, pair: int, cdf: np.ndarray, overlap: float = 0.0, rng: int = RANGE):
    """One pair regenerated on the host (the checker's view of the workload)."""
    la, lb = C.c_uint32(), C.c_uint32()
    L = load()
    check(L.gary_gen_pair_host(seed, pair, len(cdf), cdf.ctypes.data, overlap, rng, None,
                               C.byref(la), None, C.byref(lb)), "gary_gen_pair_host")
    a = np.zeros(max(la.value, 1), np.uint32)
    b = np.zeros(max(lb.value, 1), np.uint32)
    check(L.gary_gen_pair_host(seed, pair, len(cdf), cdf.ctypes.data, overlap, rng, a.ctypes.data,
                               C.byref(la), b.ctypes.data, C.byref(lb)), "gary_gen_pair_host")
    return a[: la.value], b[: lb.value]


@dataclass
class PairBatch:
    """Pairs of sorted lists on the device (torch tensors), lists 16-byte padded."""
    npairs: int
    la: "object"
    lb: "object"
    a_off: "object"
    b_off: "object"
    a: "object"
    b: "object"

    @classmethod
    def generate(cls, seed: int, first: int, npairs: int, cdf: np.ndarray, overlap: float = 0.0,
                 rng: int = RANGE, stream=None) -> "PairBatch":
        import torch

        L = load()
        dev = "cuda"
        dcdf = torch.from_numpy(cdf.view(np.int64)).to(dev)
        la = torch.empty(npairs, dtype=torch.int32, device=dev)
        lb = torch.empty(npairs, dtype=torch.int32, device=dev)
        qa = torch.empty(npairs, dtype=torch.int64, device=dev)
        qb = torch.empty(npairs, dtype=torch.int64, device=dev)
        check(L.gary_gen_pairs_lengths(seed, first, npairs, len(cdf), dcdf.data_ptr(), la.data_ptr(),
                                       lb.data_ptr(), qa.data_ptr(), qb.data_ptr(), _s(stream)),
              "gary_gen_pairs_lengths")
        a_off = torch.zeros(npairs + 1, dtype=torch.int64, device=dev)
        b_off = torch.zeros(npairs + 1, dtype=torch.int64, device=dev)
        torch.cumsum(qa * 4, 0, out=a_off[1:])
        torch.cumsum(qb * 4, 0, out=b_off[1:])
        na, nb = int(a_off[-1].item()), int(b_off[-1].item())
        a = torch.empty(max(na, 4), dtype=torch.int32, device=dev)
        b = torch.empty(max(nb, 4), dtype=torch.int32, device=dev)
        check(L.gary_gen_pairs_values(seed, first, npairs, len(cdf), dcdf.data_ptr(), overlap, rng,
                                      la.data_ptr(), lb.data_ptr(), a_off.data_ptr(), b_off.data_ptr(),
                                      a.data_ptr(), b.data_ptr(), _s(stream)), "gary_gen_pairs_values")
        return cls(npairs, la, lb, a_off, b_off, a, b)

    def input_bytes(self) -> int:
        """Algorithmic bytes of a count pass: 4 (|A| + |B|) per pair."""
        return 4 * (int(self.la.sum().item()) + int(self.lb.sum().item()))


def output_buffers(batch: PairBatch):
    """(out, out_off) for a materialising pass: pair i may write min(|A_i|, |B_i|)
    ids from out_off[i]."""
    import torch

    cap = torch.minimum(batch.la, batch.lb).to(torch.int64)
    out_off = torch.zeros(batch.npairs + 1, dtype=torch.int64, device=cap.device)
    torch.cumsum(cap, 0, out=out_off[1:])
    out = torch.empty(max(int(out_off[-1].item()), 1), dtype=torch.int32, device=cap.device)
    return out, out_off


def intersect(batch: PairBatch, variant: int = GARY_ISECT_AUTO, materialise: bool = False,
              stream=None, counts=None, queue=None, total=None, outputs=None):
    """Per-pair counts (int64 tensor) and total; with materialise also the
    sorted intersections (out, out_off).  Buffers given by the caller
    (counts, queue, total, outputs = output_buffers(batch)) are reused, so the
    call then launches the kernel and nothing else."""
    import torch

    dev = "cuda"
    counts = torch.empty(batch.npairs, dtype=torch.int64, device=dev) if counts is None else counts
    total = torch.zeros(1, dtype=torch.int64, device=dev) if total is None else total
    queue = torch.zeros(1, dtype=torch.int64, device=dev) if queue is None else queue
    out = out_off = None
    if materialise:
        out, out_off = output_buffers(batch) if outputs is None else outputs
    check(load().gary_intersect_batch(
        batch.npairs, batch.a_off.data_ptr(), batch.la.data_ptr(), batch.a.data_ptr(),
        batch.b_off.data_ptr(), batch.lb.data_ptr(), batch.b.data_ptr(), variant, counts.data_ptr(),
        out_off.data_ptr() if materialise else None, out.data_ptr() if materialise else None,
        total.data_ptr(), queue.data_ptr(), _s(stream)), "gary_intersect_batch")
    if materialise:
        return counts, total, out, out_off
    return counts, total


def intersect_num(batch: PairBatch, bound=None, ex_off=None, ex=None, variant: int = GARY_ISECT_AUTO,
                  stream=None):
    """Per-pair |{x in A & B : x < bound[i], x not excluded}| (int64 tensor)
    and total: the bounded / ancestor-filtered counts of pattern matching.
    bound: per-pair uint32 tensor or None; ex_off (npairs + 1, int64) / ex
    (uint32 ids): per-pair excluded ids, or None."""
    import torch

    dev = "cuda"
    counts = torch.empty(batch.npairs, dtype=torch.int64, device=dev)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    queue = torch.zeros(1, dtype=torch.int64, device=dev)
    check(load().gary_intersect_num_batch(
        batch.npairs, batch.a_off.data_ptr(), batch.la.data_ptr(), batch.a.data_ptr(),
        batch.b_off.data_ptr(), batch.lb.data_ptr(), batch.b.data_ptr(), variant,
        bound.data_ptr() if bound is not None else None, ex_off.data_ptr() if ex_off is not None else None,
        ex.data_ptr() if ex is not None else None, counts.data_ptr(), total.data_ptr(), queue.data_ptr(),
        _s(stream)), "gary_intersect_num_batch")
    return counts, total


def search(lst, keys, cache_entries: int = 0, stream=None):
    """(found uint8 tensor, count) for keys in the sorted list (device tensors)."""
    import torch

    found = torch.empty(keys.numel(), dtype=torch.uint8, device="cuda")
    count = torch.zeros(1, dtype=torch.int64, device="cuda")
    check(load().gary_search_batch(lst.data_ptr(), lst.numel(), keys.data_ptr(), keys.numel(),
                                   cache_entries, found.data_ptr(), count.data_ptr(), _s(stream)),
          "gary_search_batch")
    return found, count
