"""Batched triangle counting: thousands of graphs of uneven sizes in one
persistent, CUDA-graph-captured launch.

Workload (seeded): graph i has n_i = round(exp(U(ln n_lo, ln n_hi))) vertices;
even i: Barabasi-Albert with m_i uniform in 2..16; odd i: RMAT (.57,.19,.19,.05)
at scale ceil(log2 n_i) with 8 n_i samples, keeping samples whose endpoints
are both < n_i.  Graphs are deduplicated, loop-free and symmetrised.

    batch = Batch.build(make_specs(4096, seed=1))
    counts = batch.count()                       # one launch, per-graph counts
    exe = batch.capture(stream); exe.launch(stream)
"""
from __future__ import annotations

import ctypes as C
import math
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from . import DeviceCsr, Graph, csr_from_edges_device, gen_rmat
from ._lib import GARY_INPUT_DEVICE, GARY_SCHED_PLAIN, check, load


def _mix(z: int) -> int:
    m = (1 << 64) - 1
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9 & m
    z = (z ^ (z >> 27)) * 0x94D049BB133111EB & m
    return z ^ (z >> 31)


@dataclass
class GraphSpec:
    index: int
    kind: str  # "ba" or "rmat"
    n: int
    m: int     # BA attachment count (0 for RMAT)
    seed: int


def make_specs(count: int = 4096, seed: int = 1, n_lo: float = 1e3, n_hi: float = 2e5) -> list[GraphSpec]:
    specs = []
    for i in range(count):
        r = _mix((seed << 20) ^ (i * 0x9E3779B97F4A7C15 & ((1 << 64) - 1)))
        u = (r >> 11) / float(1 << 53)
        n = int(round(math.exp(math.log(n_lo) + u * (math.log(n_hi) - math.log(n_lo)))))
        gseed = _mix(r ^ 0x1234)
        if i % 2 == 0:
            specs.append(GraphSpec(i, "ba", n, 2 + (r >> 3) % 15, gseed))
        else:
            specs.append(GraphSpec(i, "rmat", n, 0, gseed))
    return specs


def generate(spec: GraphSpec) -> tuple[np.ndarray, np.ndarray]:
    """Edge list of one graph (host, as generated: may hold duplicates)."""
    if spec.kind == "ba":
        cap = spec.m * (spec.m + 1) // 2 + (spec.n - spec.m - 1) * spec.m
        src = np.empty(cap, np.uint32)
        dst = np.empty(cap, np.uint32)
        cnt = C.c_uint64()
        check(load().gary_gen_ba(spec.n, spec.m, spec.seed, src.ctypes.data, dst.ctypes.data, C.byref(cnt)),
              "gary_gen_ba")
        return src[: cnt.value], dst[: cnt.value]
    scale = max(1, math.ceil(math.log2(spec.n)))
    s, d = gen_rmat(scale, spec.seed, 8 * spec.n)
    keep = (s < spec.n) & (d < spec.n)
    return s[keep], d[keep]


class Batch:
    """The disjoint union of the graphs on the device, ranked per graph."""

    def __init__(self, specs, graph: Graph, group_off: np.ndarray, sym_nnz: int):
        self.specs = specs
        self.graph = graph
        self.group_off = group_off
        self.sym_nnz = sym_nnz

    @classmethod
    def build(cls, specs, threads: int = 16, stream=None) -> "Batch":
        import torch

        with ThreadPoolExecutor(threads) as ex:
            edges = list(ex.map(generate, specs))
        ns = np.array([s.n for s in specs], np.uint64)
        off = np.zeros(len(specs) + 1, np.uint64)
        np.cumsum(ns, out=off[1:])
        total_n = int(off[-1])
        m = sum(len(s) for s, _ in edges)
        src = torch.empty(m, dtype=torch.int32, pin_memory=True)
        dst = torch.empty(m, dtype=torch.int32, pin_memory=True)
        sv, dv = src.numpy().view(np.uint32), dst.numpy().view(np.uint32)
        pos = 0
        for (s, d), o in zip(edges, off[:-1]):
            k = len(s)
            sv[pos:pos + k] = s + np.uint32(o)
            dv[pos:pos + k] = d + np.uint32(o)
            pos += k
        del edges
        csr = csr_from_edges_device(src.cuda(), dst.cuda(), total_n, stream)
        del src, dst
        p, i = csr.device_ptrs()
        _, nnz = csr.shape()
        out = C.c_void_p()
        check(load().gary_batch_upload(off.ctypes.data, len(specs), p, i, total_n, nnz, GARY_INPUT_DEVICE,
                                       _s(stream), C.byref(out)), "gary_batch_upload")
        csr.free()
        torch.cuda.empty_cache()
        return cls(specs, Graph(out.value), off, nnz)

    def count(self, sched: int = GARY_SCHED_PLAIN, stream=None):
        """(per-graph counts numpy uint64, total) through one batched launch."""
        import torch

        counts = torch.zeros(len(self.specs), dtype=torch.int64, device="cuda")
        total = torch.zeros(1, dtype=torch.int64, device="cuda")
        check(load().gary_batch_count_async(self.graph.handle, sched, counts.data_ptr(), total.data_ptr(),
                                            _s(stream)), "gary_batch_count_async")
        torch.cuda.synchronize()
        return counts.cpu().numpy().view(np.uint64), int(total.item())

    def capture(self, stream, sched: int = GARY_SCHED_PLAIN) -> "Exec":
        import torch

        counts = torch.zeros(len(self.specs), dtype=torch.int64, device="cuda")
        total = torch.zeros(1, dtype=torch.int64, device="cuda")
        e = C.c_void_p()
        check(load().gary_batch_capture(self.graph.handle, sched, counts.data_ptr(), total.data_ptr(),
                                        _s(stream), C.byref(e)), "gary_batch_capture")
        return Exec(e.value, counts, total)

    def free(self):
        self.graph.free()


class Exec:
    """A captured batched count (CUDA graph); results land in .counts/.total."""

    def __init__(self, handle, counts, total):
        self.h = C.c_void_p(handle)
        self.counts = counts
        self.total = total

    def launch(self, stream) -> None:
        check(load().gary_exec_launch(self.h, _s(stream)), "gary_exec_launch")

    def free(self):
        if self.h:
            load().gary_exec_free(self.h)
            self.h = C.c_void_p()


def per_graph_graphs(specs, threads: int = 16) -> list[Graph]:
    """Each graph uploaded on its own (the sequential-launch baseline)."""
    with ThreadPoolExecutor(threads) as ex:
        edges = list(ex.map(generate, specs))
    graphs = []
    for spec, (s, d) in zip(specs, edges):
        with csr_from_edges_device(s, d, spec.n) as csr:
            p, i = csr.device_ptrs()
            _, nnz = csr.shape()
            out = C.c_void_p()
            check(load().gary_graph_upload(p, i, spec.n, nnz, GARY_INPUT_DEVICE, None, C.byref(out)),
                  "gary_graph_upload")
            graphs.append(Graph(out.value))
    return graphs


def _s(stream) -> int:
    if stream is None:
        return 0
    return stream if isinstance(stream, int) else stream.cuda_stream


__all__ = ["GraphSpec", "make_specs", "generate", "Batch", "Exec", "per_graph_graphs", "DeviceCsr"]
