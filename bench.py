"""Benchmark: triangle counting on RMAT scale 24, edge factor 32.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full triangle count of the degree-oriented RMAT-24 ef32 graph
(a,b,c,d = .57,.19,.19,.05, seeded, deduplicated, no loops, symmetrised) with
the graph resident in HBM.  `value` is oriented edges / second over all ranks.
Multi-GPU (torchrun, one rank per GPU): every rank holds the whole graph and
counts its shard of the tile plan; the shard counts are summed with one 8-byte
all-reduce (strong scaling).

`learned` times the same count under the learned schedule (the cost model in
gary_b200/data) right after the plain one, in the same process.

`e2e` runs the same count through the public C ABI from pinned HOST buffers:
upload (H2D copy, orientation, relabel, padding) + count + the 8-byte D2H read
of the result, every step.  The host graph is the reference's input form for
this path by default: the id-oriented DAG CSR (csr_dag.bin, each edge once in
the row of its larger endpoint); --e2e-input symmetric uploads both directions.

`cpu_baseline` (rank 0, N=1) and `--impl reference` time the reference's own CPU
path: the same seeded edges (the oracle's restatement of the generator, so the
product library is not loaded), deduplicated, then the reference's own graph
pipeline (GraphCOO::symmetrize -> toCSR_ -> toCOO -> orientation -> toCSR_,
src/Graph.cpp, compiled in place under oracle/_ref) and its cpuTriCount
(test/TriQueryTest.cu:17-37) on a bounded, evenly strided vertex sample, with
all host threads.

`batch` and `setops` (N=1; --no-extras skips them) summarise the batched
4096-graph launch and the set-intersection microbench on a 2^20-pair batch;
`--workload batch|setops|patterns` runs each in full.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "triangle-count edges/sec at RMAT-24: learned-sched vs plain GPU vs CPU; HBM GB/s"
UNIT = "edges/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--ef", type=int, default=32)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--sched", choices=["plain", "learned"], default="plain")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--e2e-input", choices=["dag", "symmetric"], default="dag",
                    help="host CSR the e2e leg uploads: the reference's id-oriented DAG or the symmetric graph")
    ap.add_argument("--pool-keep-gb", type=float, default=None,
                    help="freed construction scratch the library's memory pool keeps mapped (GB)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU sample time")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip timing the reference GPU kernel")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--workload", choices=["tc", "setops", "batch", "patterns"], default="tc",
                    help="tc: the headline triangle count; setops: the set-intersection microbench; "
                         "batch: 4096 graphs in one launch; patterns: triangle / 4-cycle / 4-clique "
                         "counts on the RMAT graph")
    ap.add_argument("--cpu-scale", type=int, default=16,
                    help="patterns: RMAT scale of the graph the CPU oracle counts beside the GPU")
    ap.add_argument("--patterns", default="3,4,5",
                    help="patterns workload: 3 triangle, 4 four-cycle, 5 four-clique")
    ap.add_argument("--graphs", type=int, default=4096, help="batch: number of graphs")
    ap.add_argument("--no-autotune", action="store_true", help="batch: keep the default tile shapes")
    ap.add_argument("--pairs-log2", type=int, default=24, help="setops: total pairs = 2^k")
    ap.add_argument("--batch-log2", type=int, default=20, help="setops: pairs per generated batch")
    ap.add_argument("--overlaps", default="0,0.1,0.25,0.5", help="setops: planted overlap fractions")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-schedule leg")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batch and set-intersection summaries of the default line")
    return ap.parse_args()


# ---------------------------------------------------------------- plumbing
class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "power_w_max": max(power) if power else None}


def build_graph(gb, torch, scale, ef, seed):
    """RMAT edges generated on the device, symmetric CSR built on the device."""
    n = 1 << scale
    src, dst = gb.gen_rmat_device(scale, seed, ef << scale)
    csr = gb.csr_from_edges_device(src, dst, n)
    del src, dst
    torch.cuda.empty_cache()
    return n, csr


def upload_from_device_csr(gb, csr, n):
    from gary_b200 import _lib

    p, i = csr.device_ptrs()
    _, nnz = csr.shape()
    out = C.c_void_p()
    _lib.check(_lib.load().gary_graph_upload(p, i, n, nnz, _lib.GARY_INPUT_DEVICE, None, C.byref(out)),
               "gary_graph_upload")
    return gb.Graph(out.value)


def id_oriented_dag(torch, hp, hi, n):
    """Pinned host (ptr, idx, nnz) of the graph with every edge kept once, in
    the row of its larger endpoint (v < u in row u), from the pinned symmetric
    CSR; computed on the device, outside any timed region."""
    ptr = hp.cuda()
    idx = hi.cuda()
    deg = (ptr[1:] - ptr[:-1])
    rows = torch.repeat_interleave(torch.arange(n, device="cuda", dtype=torch.int32), deg)
    keep = idx < rows
    del deg
    kept_rows = rows[keep]
    del rows
    dag_idx = idx[keep]
    del idx, keep
    cnt = torch.bincount(kept_rows, minlength=n)
    del kept_rows
    dptr = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    torch.cumsum(cnt, 0, out=dptr[1:])
    nnz = int(dptr[-1].item())
    op = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
    oi = torch.empty(nnz, dtype=torch.int32, pin_memory=True)
    op.copy_(dptr)
    oi.copy_(dag_idx)
    del dptr, dag_idx, cnt, ptr
    torch.cuda.empty_cache()
    return op, oi, nnz


def workload_config(args, world: int) -> dict:
    """The `config` both arms print (the same dict, so the lines compare)."""
    return {"workload": f"triangle count, RMAT scale {args.scale} edge factor {args.ef}, seed {args.seed}",
            "scale": args.scale, "ef": args.ef, "seed": args.seed,
            "l2": "inputs larger than L2: the graph's lists (GBs) against the 126 MB L2",
            "parallelism": f"dp{world} (tile shards, graph replicated)"}


# Sources the triangle kernel is built from: a counter capture stored under
# profiles/ applies to the build whose sources hash to its "kernel_src".
KERNEL_SOURCES = ("tc.cu", "tc.cuh", "warp_ops.cuh", "bulk.cuh", "internal.cuh", "graph.cuh")
# the 4-cycle and 4-clique count kernels
PATTERN_SOURCES = ("patterns.cu", "patterns.cuh", "pattern_rules.cuh", "warp_ops.cuh", "internal.cuh", "graph.cuh")


def kernel_source_hash(sources=KERNEL_SOURCES) -> str:
    import hashlib

    h = hashlib.sha256()
    for name in sources:
        h.update((ROOT / "gary_b200" / "csrc" / name).read_bytes())
    return h.hexdigest()[:16]


def measured_counters(workload: str, sources=KERNEL_SOURCES):
    """The ncu counters stored for `workload` (profiles/roofline_traffic.json:
    DRAM bytes, warp instructions and L2->SM bytes of one launch, or of one
    count call's kernels for the 4-vertex patterns), with `stale` true when
    they were captured on other kernel sources."""
    f = ROOT / "profiles" / "roofline_traffic.json"
    if not f.exists():
        return None
    try:
        rec = json.loads(f.read_text()).get(workload)
    except Exception:
        return None
    if not isinstance(rec, dict):
        return None
    rec = dict(rec)
    rec["stale"] = rec.get("kernel_src") != kernel_source_hash(sources)
    return rec


def peak_hbm():
    pk = ROOT / "MEASURED_PEAKS.json"
    peaks = json.loads(pk.read_text()) if pk.exists() else {}
    hbm = peaks.get("hbm_gbs")
    if hbm:
        return float(hbm), "MEASURED_PEAKS.json hbm_gbs (measured)"
    return 6650.0, "fallback 6650 GB/s"


def reference_dag(scale: int, ef: int, seed: int):
    """The reference's oriented CSR of the workload, built without the product
    library: the oracle's restatement of the seeded generator, the duplicate
    and loop removal the workload defines, then the reference's own pipeline
    (symmetrize -> toCSR_ -> toCOO -> orientation -> toCSR_, src/Graph.cpp; the
    orientation keeps src > dst, as convert.cpp writes csr_dag.bin).
    Returns (RefCSR, out-degrees, oriented edges, seconds)."""
    import numpy as np

    from oracle import oracle as O

    n = 1 << scale
    t0 = time.perf_counter()
    src, dst = O.gen_rmat(scale, seed, ef << scale)
    us, vs = O.unique_edges(n, src, dst)
    del src, dst
    ref = O.RefCSR.dag_from_edges(n, us.view(np.int32), vs.view(np.int32))
    m = len(us)
    del us, vs
    ptr, _ = ref.arrays()
    deg = np.diff(ptr)
    return ref, deg, m, time.perf_counter() - t0


def reference_stride(ref, deg, n: int, target_s: float) -> int:
    """Vertex stride whose strided sample takes about target_s seconds."""
    stride = 4096
    while True:
        edges = int(deg[::stride].sum())
        t0 = time.perf_counter()
        ref.tri_count(0, n, stride, 0)
        dt = time.perf_counter() - t0
        if dt >= 0.5 or stride == 1:
            break
        stride = max(1, stride // 8)
    rate = edges / max(dt, 1e-9)
    return max(1, int(int(deg.sum()) / max(rate * target_s, 1)))


def reference_sample_line(ref, deg, m: int, n: int, stride: int, times: list, threads: int, prep_s: float):
    edges = int(deg[::stride].sum())
    dt = sum(times) / len(times)
    sample = (f"every {stride}-th vertex of the reference's id-oriented DAG of the same graph (~{edges} of {m} "
              f"oriented edges per step, offset rotated per step; input built by the reference's own "
              f"pipeline in {prep_s:.0f} s, untimed)")
    return edges / dt, dt, sample


# ---------------------------------------------------------------- arms
def run_reference(args, dist):
    """--impl reference: the reference's CPU path, rank 0 only.  Nothing of the
    product library is loaded: the input comes from the oracle's generator
    restatement and the reference's own pipeline."""
    from oracle import oracle as O

    if dist.rank != 0:
        return 0
    n = 1 << args.scale
    ref, deg, m, prep_s = reference_dag(args.scale, args.ef, args.seed)
    threads = O.ref_cpu().ref_omp_max_threads()
    stride = reference_stride(ref, deg, n, args.cpu_seconds / 2)
    for _ in range(args.warmup):
        ref.tri_count(0, n, stride * 4, 0)
    times = []
    for k in range(args.steps):
        t0 = time.perf_counter()
        ref.tri_count(k % stride, n, stride, 0)
        times.append(time.perf_counter() - t0)
    value, dt, sample = reference_sample_line(ref, deg, m, n, stride, times, threads, prep_s)
    ref.free()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": workload_config(args, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "path": "cpuTriCount (test/TriQueryTest.cu:17-37, uint64 accumulators) over the reference's GraphCSR",
    }
    print(json.dumps(line), flush=True)
    return 0


def time_counts(L, g, sched, dist, stream, out, steps: int, warmup: int, clocks=None):
    """Per-step kernel ms (CUDA events on the counting stream) of `steps`
    counts after `warmup`, bracketed by barriers and synchronisations; then
    the launch status is checked.  Returns (ms list, local count)."""
    import ctypes as C

    import torch

    from gary_b200 import _lib

    def step():
        _lib.check(L.gary_count_shard_async(g.handle, _lib.GARY_PATTERN_TRIANGLE, sched, dist.rank, dist.world,
                                            C.c_void_p(stream.cuda_stream), C.c_void_p(out.data_ptr())),
                   "gary_count_shard_async")

    with torch.cuda.stream(stream):
        for _ in range(max(warmup, 1)):
            step()
    stream.synchronize()
    count_local = int(out.item())
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    with torch.cuda.stream(stream):
        for k in range(steps):
            evs[k][0].record(stream)
            step()
            evs[k][1].record(stream)
    stream.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    # the launches' own status (bounded waits, table capacity): never a silent count
    _lib.check(L.gary_count_status(g.handle, C.c_void_p(stream.cuda_stream)), "gary_count_status")
    assert int(out.item()) == count_local, "count changed between steps"
    return [a.elapsed_time(b) for a, b in evs], count_local, clk


def run_ours(args, dist):
    import ctypes as C

    import numpy as np
    import torch

    import gary_b200 as gb
    from gary_b200 import _lib

    dist.init()
    dev = dist.local
    if args.pool_keep_gb is not None:
        _lib.check(_lib.load().gary_tune(b"pool_keep_bytes", int(args.pool_keep_gb * 1e9)), "gary_tune")
    sched = {"plain": _lib.GARY_SCHED_PLAIN, "learned": _lib.GARY_SCHED_LEARNED}[args.sched]
    if args.sched == "learned" or not args.no_learned:
        from gary_b200.costmodel import CostModel

        CostModel.load().install()
    t_build = time.perf_counter()
    n, csr = build_graph(gb, torch, args.scale, args.ef, args.seed)
    _, sym_nnz = csr.shape()
    g = upload_from_device_csr(gb, csr, n)
    build_s = time.perf_counter() - t_build
    info = g.info()
    m = info["m"]
    stream = torch.cuda.Stream()
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    L = _lib.load()

    # ---- timed region: K steps, device events on the launching stream
    per, count_local, clk = time_counts(L, g, sched, dist, stream, out, args.steps, args.warmup, Clocks(dev))
    stats = g.last_stats()
    ms_local = sum(per) / len(per)
    ms = dist.allreduce(ms_local, "max")
    count = dist.allreduce(count_local, "sum")
    value = m / (ms / 1e3)

    # ---- the other schedule on the same graph, same process, same timing rules
    learned = None
    if not args.no_learned:
        other = _lib.GARY_SCHED_PLAIN if args.sched == "learned" else _lib.GARY_SCHED_LEARNED
        lper, lcount, _ = time_counts(L, g, other, dist, stream, out, args.steps, args.warmup)
        lstats = g.last_stats()
        lms = dist.allreduce(sum(lper) / len(lper), "max")
        lcount = dist.allreduce(lcount, "sum")
        learned_ms, plain_ms = (lms, ms) if other == _lib.GARY_SCHED_LEARNED else (ms, lms)
        learned = {"value": m / (learned_ms / 1e3), "unit": UNIT, "ms": learned_ms, "plain_ms": plain_ms,
                   "ratio_vs_plain": plain_ms / learned_ms, "count_equal": lcount == count,
                   "balance": balance_of(lstats),
                   "model": "gary_b200/data/cost_model.gmlp (6-64-64-4 MLP, per-vertex variant and tile weights)"}
        assert lcount == count, f"learned schedule count {lcount} != plain {count}"

    # ---- end to end through the public API from pinned host memory
    e2e = None
    if args.e2e_steps > 0:
        hp = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
        hi = torch.empty(sym_nnz, dtype=torch.int32, pin_memory=True)
        hp_np = hp.numpy().view(np.uint64)
        hi_np = hi.numpy().view(np.uint32)
        csr.download(hp_np, hi_np)
        csr.free()
        e2e_flags, e2e_nnz = 0, sym_nnz
        if args.e2e_input == "dag":
            # the reference's input form (csr_dag.bin: GraphCOO::orientation keeps
            # src > dst, so row u lists its neighbours v < u), built here, untimed
            hp, hi, e2e_nnz = id_oriented_dag(torch, hp, hi, n)
            e2e_flags = _lib.GARY_INPUT_DAG
        e2e_times = []
        for k in range(args.e2e_steps + 1):
            dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            gh = C.c_void_p()
            _lib.check(L.gary_graph_upload(hp.data_ptr(), hi.data_ptr(), n, e2e_nnz, e2e_flags,
                                           C.c_void_p(stream.cuda_stream), C.byref(gh)), "upload")
            dres = torch.empty(1, dtype=torch.int64, device="cuda")
            _lib.check(L.gary_count_shard_async(gh, _lib.GARY_PATTERN_TRIANGLE, sched, dist.rank, dist.world,
                                                C.c_void_p(stream.cuda_stream), C.c_void_p(dres.data_ptr())),
                       "count")
            with torch.cuda.stream(stream):  # 8-byte D2H read of the result, on the counting stream
                hres = dres.to("cpu", non_blocking=True)
            stream.synchronize()
            res = int(hres.item())
            dt = time.perf_counter() - t0
            _lib.check(L.gary_count_status(gh, C.c_void_p(stream.cuda_stream)), "gary_count_status")
            L.gary_graph_free(gh)
            if k > 0:  # first one warms the allocator
                e2e_times.append(dt)
            assert res == count_local, "e2e count differs from the resident-graph count"
        # the median step, with the mean and every step beside it: a rare step pays
        # for a slow driver call on a host shared with other jobs
        e2e_s = dist.allreduce(statistics.median(e2e_times), "max")
        e2e_mean = dist.allreduce(sum(e2e_times) / len(e2e_times), "max")
        form = ("id-oriented DAG CSR, rows list neighbours v < u (the reference's csr_dag input)"
                if args.e2e_input == "dag" else "symmetric CSR")
        e2e = {"value": m / e2e_s, "unit": UNIT, "h2d_bytes_per_step": (n + 1) * 8 + e2e_nnz * 4,
               "d2h_bytes_per_step": 8, "ms_per_step": e2e_s * 1e3, "statistic": "median of the steps",
               "mean_ms_per_step": e2e_mean * 1e3, "step_ms": [round(t * 1e3, 2) for t in e2e_times],
               "path": f"gary_graph_upload(pinned host {form}) + gary_count_shard_async + D2H of the count"}
    else:
        csr.free()

    line = None
    if dist.rank == 0:
        cfg = workload_config(args, dist.world)
        alg = info["alg_bytes"]
        hbm, peak_src = peak_hbm()
        # per-launch kernel time at N ranks: each rank runs one launch over its shard
        achieved = (alg / dist.world) / (ms_local / 1e3) / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                    "traffic": None, "peak_source": peak_src, "alg_bytes_per_launch": alg / dist.world,
                    "alg_bytes_definition": "sum over oriented edges of 4(d+(u)+d+(v)) + 24: both lists read "
                                            "once per edge, as the reference's kernel reads them; the "
                                            "middle-vertex walk reads far less, so this frac exceeds 1"}
        mc = measured_counters(cfg["workload"]) if dist.world == 1 else None
        sm_hz = (clk.get("sm_mhz") or 1965.0) * 1e6 if clk else 1965.0 * 1e6
        if mc:
            t = ms_local / 1e3
            roofline["traffic"] = mc["dram_bytes"]
            roofline["measured"] = {
                "source": mc.get("profile"), "kernel_src": mc.get("kernel_src"), "stale": mc["stale"],
                # DRAM: the bytes one launch moved (ncu) over its live duration
                "dram": {"gbs": mc["dram_bytes"] / t / 1e9, "frac": mc["dram_bytes"] / t / 1e9 / hbm},
                # instruction issue: warp instructions (ncu) over 148 SMs x 4 schedulers x clock
                "issue": {"warp_inst_per_launch": mc.get("warp_inst"),
                          "ceiling_per_s": sm_count() * 4 * sm_hz,
                          "frac": (mc["warp_inst"] / t) / (sm_count() * 4 * sm_hz) if mc.get("warp_inst") else None},
                # L2 -> SM bytes (ncu) and the L2's own throughput fraction (ncu's peak)
                "l2": {"bytes_to_sm": mc.get("l2_to_sm_bytes"),
                       "gbs": mc["l2_to_sm_bytes"] / t / 1e9 if mc.get("l2_to_sm_bytes") else None,
                       "throughput_pct_of_peak": mc.get("l2_pct_of_peak")},
            }
        work = stats.get("work") or 0
        roofline["probes"] = {"per_launch": work, "per_s": work / (ms_local / 1e3) if work else None,
                              "definition": "ids of in-neighbour suffixes tested against a set of N+(v)"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic", "sched": args.sched,
            "config": cfg,
            "graph": {"n": n, "oriented_edges": m, "sym_nnz": sym_nnz, "max_out_degree": info["max_out_degree"],
                      "wedges": info["wedges"], "alg_bytes": alg, "adj_gb": info["adj_words"] * 4 / 1e9},
            "count": count,
            "roofline": roofline,
            "learned": learned,
            "e2e": e2e,
            "gpu_launches": args.steps,
            "clocks": clk,
            "build_s": build_s,
            "cta_path_tiles": stats.get("cta_path_tiles"),
            # the last timed launch's makespan against the mean CTA finish: how much any other
            # assignment of the same tiles to CTAs could gain
            "balance": balance_of(stats),
        }
    g_dag = None
    if dist.rank == 0 and dist.world == 1 and not args.no_ref_gpu:
        g_dag = g.download()
    g.free()
    torch.cuda.empty_cache()

    if dist.rank == 0 and dist.world == 1:
        from oracle import oracle as O  # CPU baseline / reference legs only

        if g_dag is not None and O.have_ref_gpu():
            dptr, didx, _ = g_dag
            # the reference's own triangleCountHom<true,32> built for sm_100a, same DAG
            ref = O.RefGpuGraph(dptr.astype(np.int64), didx.astype(np.int32))
            ref.tri_count(0)
            tms = []
            for _ in range(3):
                c, t = ref.tri_count(0)
                tms.append(t)
                assert c == count, f"reference kernel count {c} != ours {count}"
            ref.free()
            tr = statistics.median(tms)
            line["ref_gpu_kernel"] = {"value": m / (tr / 1e3), "unit": UNIT, "ms": tr,
                                      "kernel": "graph_query::triangleCountHom<true,32> (sm_100a build)",
                                      "count_equal": True}
        del g_dag
        if not args.no_cpu and O.have_ref_cpu():
            ref, deg, rm, prep_s = reference_dag(args.scale, args.ef, args.seed)
            threads = O.ref_cpu().ref_omp_max_threads()
            stride = reference_stride(ref, deg, n, args.cpu_seconds)
            t0 = time.perf_counter()
            ref.tri_count(0, n, stride, 0)
            dt = time.perf_counter() - t0
            v, _, sample = reference_sample_line(ref, deg, rm, n, stride, [dt], threads, prep_s)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                                    "sample": sample}
            ref.free()
        if not args.no_extras:
            line["batch"] = batch_summary(args)
            line["setops"] = setops_summary(args)
    if line is not None:
        print(json.dumps(line), flush=True)
    dist.close()
    return 0


def balance_of(stats: dict) -> dict:
    mk, mean = stats.get("makespan_ms") or 0.0, stats.get("mean_cta_finish_ms") or 0.0
    return {"makespan_ms": mk, "mean_cta_finish_ms": mean, "schedule_bound": mk / mean if mean else None}


def sm_count() -> int:
    import torch

    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count


def run_setops(args, dist):
    import torch

    torch.cuda.set_device(dist.local)
    overlaps = [float(x) for x in args.overlaps.split(",")]
    print(json.dumps(setops_measure(args, args.pairs_log2, args.batch_log2, overlaps, not args.no_cpu)), flush=True)
    return 0


def setops_summary(args) -> dict:
    """The microbench on one 2^20-pair batch at planted overlap 0.1, for the
    default line: pairs/s per variant (count only), the best variant's HBM
    fraction, the CPU merge baseline, and whether every variant agreed."""
    line = setops_measure(args, 20, 20, [0.1], True)
    per = {k.split(":")[1]: round(r["pairs_per_s"]) for k, r in line["variants"].items() if k.endswith(":count")}
    return {"metric": "set-intersection pairs/s", "pairs": 1 << 20, "overlap": 0.1, "pairs_per_s": per,
            "best": line["best"], "best_pairs_per_s": line["value"], "roofline": line["roofline"],
            "cpu_baseline": line["cpu_baseline"], "variants_agree": True,
            "full_run": "python bench.py --workload setops (2^24 pairs per overlap, overlaps 0-0.5)"}


def setops_measure(args, pairs_log2: int, batch_log2: int, overlaps: list, with_cpu: bool) -> dict:
    """Set-intersection microbench: 2^pairs_log2 pairs of sorted uint32 lists,
    Zipf(1.2) lengths on [1, 65536], values in [0, 2^26), per planted overlap;
    merge / two-phase search / bitmap / auto, count-only and materialised.
    Pairs are generated on the device in batches (not timed).  Each variant's
    kernel is timed with CUDA events on every batch, output buffers prepared
    beforehand, so the timed region is the one launch.  A batch holds about
    14 GB of lists, far above L2.  The CPU baseline merges a sample of the first
    batch's pairs on the host cores (std::set_intersection semantics)."""
    import numpy as np
    import torch

    from gary_b200 import setops as so
    from oracle import oracle as O

    cdf = so.zipf_table(65536, 1.2)
    total_pairs = 1 << pairs_log2
    bsz = min(1 << batch_log2, total_pairs)
    variants = ["merge", "search", "bitmap", "auto"]
    res = {}
    stream = torch.cuda.Stream()
    counts = torch.empty(bsz, dtype=torch.int64, device="cuda")
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    queue = torch.zeros(1, dtype=torch.int64, device="cuda")
    cpu = None
    launches = 0
    for ov in overlaps:
        acc = {(v, m): [0.0, 0] for v in variants for m in (False, True)}
        bytes_in = 0
        for first in range(0, total_pairs, bsz):
            with torch.cuda.stream(stream):
                batch = so.PairBatch.generate(args.seed, first, bsz, cdf, ov, stream=stream)
                outs = so.output_buffers(batch)
            stream.synchronize()
            bytes_in += batch.input_bytes()
            for v in variants:
                for mat in (False, True):
                    kw = dict(stream=stream, counts=counts, queue=queue, total=tot, outputs=outs if mat else None)
                    with torch.cuda.stream(stream):
                        so.intersect(batch, so.VARIANTS[v], mat, **kw)  # warm
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        so.intersect(batch, so.VARIANTS[v], mat, **kw)
                        e1.record(stream)
                    stream.synchronize()
                    launches += 1
                    acc[(v, mat)][0] += e0.elapsed_time(e1)
                    acc[(v, mat)][1] += int(tot.item())
            if cpu is None and with_cpu:
                # CPU merge on a sample of this batch, checked against the GPU counts
                S = min(bsz, 1 << 16)
                so.intersect(batch, so.VARIANTS["auto"], False, stream=stream, counts=counts, queue=queue, total=tot)
                stream.synchronize()
                gpu_counts = counts[:S].cpu().numpy()
                a_off = batch.a_off[:S + 1].cpu().numpy()
                b_off = batch.b_off[:S + 1].cpu().numpy()
                a = batch.a[:int(a_off[-1])].cpu().numpy().view(np.uint32)
                b = batch.b[:int(b_off[-1])].cpu().numpy().view(np.uint32)
                la, lb = batch.la[:S].cpu().numpy(), batch.lb[:S].cpu().numpy()
                threads = os.cpu_count() or 1
                O.intersect_batch(a_off, la, a, b_off, lb, b, threads)  # warm
                t0 = time.perf_counter()
                reps = 0
                while True:
                    c_cpu, _ = O.intersect_batch(a_off, la, a, b_off, lb, b, threads)
                    reps += 1
                    if time.perf_counter() - t0 > 2.0:
                        break
                dt = (time.perf_counter() - t0) / reps
                assert np.array_equal(c_cpu, gpu_counts), "CPU merge and GPU counts differ"
                cpu = {"value": S / dt, "unit": "pairs/s", "cores": threads, "kind": "port",
                       "sample": f"first {S} pairs of the overlap-{ov} batch (merge, OpenMP over pairs), "
                                 f"counts equal to the GPU's"}
            del batch, outs
        for (v, mat), (ms, hits) in acc.items():
            b = bytes_in + (4 * hits if mat else 0)
            res[f"ov{ov}:{v}:{'mat' if mat else 'count'}"] = {
                "pairs_per_s": total_pairs / (ms / 1e3), "ms": ms, "GB_per_s": b / (ms / 1e3) / 1e9,
                "intersection_total": hits}
        # every variant agrees on the total
        totals = {k: r["intersection_total"] for k, r in res.items() if k.startswith(f"ov{ov}:")}
        assert len(set(totals.values())) == 1, totals
    best = max((r["pairs_per_s"], k) for k, r in res.items() if k.endswith(":count"))
    hbm, peak_src = peak_hbm()
    bk = res[best[1]]
    line = {"metric": f"set-intersection pairs/sec (2^{pairs_log2} Zipf(1.2) pairs)", "value": best[0],
            "unit": "pairs/s",
            "best": best[1], "n_gpus": 1, "steps": len(overlaps), "warmup": 1, "higher_is_better": True,
            "dtype": "u32", "data": "synthetic",
            "config": {"workload": f"set-intersection microbench, 2^{pairs_log2} pairs per overlap, "
                                   f"Zipf(1.2) lengths on [1, 65536], values in [0, 2^26)",
                       "batch_pairs": bsz, "overlaps": overlaps, "seed": args.seed,
                       "l2": "inputs larger than L2 (each batch holds ~14 GB of lists)"},
            "roofline": {"bound": "hbm", "achieved": bk["GB_per_s"], "peak": hbm, "unit": "GB/s",
                         "frac": bk["GB_per_s"] / hbm, "traffic": None, "peak_source": peak_src},
            "cpu_baseline": cpu, "gpu_launches": launches, "variants": res}
    return line


def run_batch(args, dist):
    import torch

    torch.cuda.set_device(dist.local)
    line = batch_measure(args, args.steps, args.warmup)
    print(json.dumps(line), flush=True)
    return 1 if line["mismatched_graphs"] else 0


def batch_summary(args) -> dict:
    """The batched workload for the default line: graphs/s of the captured
    launch, the sequential per-graph launches, their ratio and the number of
    graphs whose counts differ (batched vs sequential)."""
    line = batch_measure(args, 5, 3)
    keep = ("value", "unit", "ms_per_step", "sequential_ms_per_step", "speedup_vs_sequential",
            "oriented_edges_per_s", "mismatched_graphs", "total_triangles", "build_s")
    return {"metric": line["metric"], **{k: line[k] for k in keep}, "graphs": line["config"]["graphs"],
            "autotuned": line["config"]["autotuned"], "full_run": "python bench.py --workload batch"}


def batch_measure(args, steps: int, warmup: int) -> dict:
    """Batched counting: 4096 graphs (n log-uniform in [1e3, 2e5], half BA with
    m in 2..16, half RMAT ef8) in one autotuned, CUDA-graph-captured persistent
    launch, against 4096 sequential per-graph launches of the plain kernel on
    one stream.  Graph construction and plan building are not timed."""
    import numpy as np
    import torch

    from gary_b200 import autotune as at
    from gary_b200 import batch as B

    t0 = time.perf_counter()
    specs = B.make_specs(args.graphs, seed=args.seed)
    batch = B.Batch.build(specs)
    inf = batch.graph.info()
    build_s = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    counts = torch.zeros(len(specs), dtype=torch.int64, device="cuda")
    total = torch.zeros(1, dtype=torch.int64, device="cuda")
    L = load_lib()

    def one():
        from gary_b200._lib import check
        check(L.gary_batch_count_async(batch.graph.handle, 0, counts.data_ptr(), total.data_ptr(),
                                       stream.cuda_stream), "batch count")

    if args.no_autotune:
        tuned = {"config": "defaults", "ms": None, "trials": []}
    else:
        with torch.cuda.stream(stream):
            tuned = at.autotune(batch.graph, one)
    exe = batch.capture(stream)
    for _ in range(warmup):
        exe.launch(stream)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        exe.launch(stream)
    e1.record(stream)
    stream.synchronize()
    ms_batch = e0.elapsed_time(e1) / steps
    from gary_b200._lib import check
    check(L.gary_count_status(batch.graph.handle, stream.cuda_stream), "gary_count_status")
    bcounts = exe.counts.cpu().numpy().view(np.uint64).copy()
    # sequential baseline: the same graphs uploaded one by one, one launch each
    t1 = time.perf_counter()
    graphs = B.per_graph_graphs(specs)
    outs = torch.zeros(len(specs), dtype=torch.int64, device="cuda")
    with torch.cuda.stream(stream):
        for k, g in enumerate(graphs):  # plans built outside the timed region
            g.count_async(outs[k:k + 1], stream=stream)
    stream.synchronize()
    seq_build_s = time.perf_counter() - t1
    e0.record(stream)
    for _ in range(steps):
        with torch.cuda.stream(stream):
            for k, g in enumerate(graphs):
                g.count_async(outs[k:k + 1], stream=stream)
    e1.record(stream)
    stream.synchronize()
    ms_seq = e0.elapsed_time(e1) / steps
    scounts = outs.cpu().numpy().view(np.uint64)
    direct, _ = batch.count()  # the batched count without the CUDA graph
    bad = np.nonzero(scounts != bcounts)[0]
    mismatch = []
    if len(bad):
        from oracle import oracle as O  # checker for the diagnosis only
        for i in bad[:4]:
            s_, d_ = B.generate(specs[i])
            ptr, idx = O.sym_csr(s_, d_, specs[i].n)
            dp, di = O.orient(ptr, idx)
            mismatch.append({"graph": int(i), "n": specs[i].n, "kind": specs[i].kind, "batched": int(bcounts[i]),
                             "direct": int(direct[i]), "sequential": int(scounts[i]),
                             "oracle": O.tri_count(dp, di)})
    line = {"metric": "batched triangle count: graphs/s (4096 graphs, one captured launch)",
            "value": len(specs) / (ms_batch / 1e3), "unit": "graphs/s", "n_gpus": 1, "steps": steps,
            "warmup": warmup, "ms_per_step": ms_batch, "higher_is_better": True, "dtype": "u32",
            "data": "synthetic",
            "config": {"workload": f"{len(specs)} graphs, n log-uniform in [1e3, 2e5], even BA (m in 2..16), "
                                   f"odd RMAT ef8, seed {args.seed}",
                       "graphs": len(specs), "vertices": inf["n"], "oriented_edges": inf["m"],
                       "autotuned": tuned["config"]},
            "sequential_ms_per_step": ms_seq, "speedup_vs_sequential": ms_seq / ms_batch,
            "oriented_edges_per_s": inf["m"] / (ms_batch / 1e3), "total_triangles": int(bcounts.sum()),
            "build_s": build_s, "sequential_build_s": seq_build_s,
            "autotune_trials": tuned["trials"], "mismatched_graphs": int(len(bad)), "mismatch_samples": mismatch}
    exe.free()
    for g in graphs:
        g.free()
    batch.free()
    at.apply({})
    torch.cuda.empty_cache()
    return line


def pattern_roofline(workload: str, ms: float):
    """DRAM and issue fractions of one 4-cycle / 4-clique count call: the ncu
    counters stored for the workload (all the call's count kernels, summed)
    over the call's live CUDA-event time; None when none are stored."""
    mc = measured_counters(workload, PATTERN_SOURCES)
    if not mc:
        return None
    hbm, src = peak_hbm()
    t = ms / 1e3
    ceiling = sm_count() * 4 * 1965e6  # 4 schedulers per SM at the maximum SM clock
    return {"bound": "hbm", "achieved": mc["dram_bytes"] / t / 1e9, "peak": hbm, "unit": "GB/s",
            "frac": mc["dram_bytes"] / t / 1e9 / hbm, "traffic": mc["dram_bytes"], "peak_source": src,
            "achieved_basis": "ncu DRAM bytes of the call's count kernels over the call's CUDA-event time",
            "issue": {"warp_inst_per_call": mc["warp_inst"], "ceiling_per_s": ceiling,
                      "frac": mc["warp_inst"] / t / ceiling},
            "kernels": mc.get("kernels"), "source": mc.get("profile"), "kernel_src": mc.get("kernel_src"),
            "stale": mc["stale"]}


def run_patterns(args, dist):
    """Triangle, 4-cycle and 4-clique counts of the seeded RMAT graph (one GPU):
    per pattern the first call (plan building included, wall clock) and the
    mean of `steps` counts after `warmup` (CUDA events on the counting stream,
    plan cached).  Beside it, the same pattern on RMAT scale --cpu-scale
    (default 16) counted by the GPU and by the CPU oracle (all host threads),
    with equal counts: the oracle cannot count the full graph in reasonable
    time.  One JSON line per pattern."""
    import numpy as np
    import torch

    import gary_b200 as gb
    from oracle import oracle as O  # the small-graph CPU baseline only

    torch.cuda.set_device(dist.local)
    n, csr = build_graph(gb, torch, args.scale, args.ef, args.seed)
    g = upload_from_device_csr(gb, csr, n)
    csr.free()
    m = g.info()["m"]
    # the small graph for the CPU comparison
    sn = 1 << args.cpu_scale
    ss, sd = gb.gen_rmat(args.cpu_scale, args.seed, args.ef << args.cpu_scale)
    sptr, sidx = gb.csr_from_edges(ss, sd, sn)
    dptr, didx = O.orient(sptr, sidx)
    small = gb.Graph.upload(sptr, sidx, sn)
    stream = torch.cuda.Stream()
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    names = {3: "triangle", 4: "4-cycle", 5: "4-clique"}

    def timed(graph, pat, steps):
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                graph.count_async(out, pat, stream=stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                graph.count_async(out, pat, stream=stream)
            e1.record(stream)
        stream.synchronize()
        graph.check_status(stream)
        return e0.elapsed_time(e1) / max(steps, 1), int(out.item())

    for pat in (int(x) for x in args.patterns.split(",")):
        with torch.cuda.stream(stream):
            t0 = time.perf_counter()
            g.count_async(out, pat, stream=stream)
            stream.synchronize()
            first_s = time.perf_counter() - t0
        ms, cnt = timed(g, pat, args.steps)
        sms, scnt = timed(small, pat, max(args.steps, 5))
        oracle = {3: lambda: O.tri_count(dptr, didx), 4: lambda: O.c4_count(sptr, sidx),
                  5: lambda: O.k4_count(dptr, didx)}[pat]
        t0 = time.perf_counter()
        ocnt = oracle()
        cpu_s = time.perf_counter() - t0
        assert ocnt == scnt, f"{names[pat]}: oracle {ocnt} != GPU {scnt} on the small graph"
        workload = f"{names[pat]} count, RMAT scale {args.scale} edge factor {args.ef}, seed {args.seed}"
        print(json.dumps({"metric": f"{names[pat]} count time", "value": ms, "unit": "ms", "higher_is_better": False,
                          "pattern": names[pat], "count": cnt, "first_call_s": first_s,
                          "oriented_edges_per_s": m / (ms / 1e3),
                          "steps": args.steps, "warmup": args.warmup, "n_gpus": 1, "data": "synthetic",
                          "config": {"workload": workload},
                          "roofline": pattern_roofline(workload, ms),
                          "small_graph": {"workload": f"RMAT scale {args.cpu_scale} edge factor {args.ef}",
                                          "gpu_ms": sms, "count": scnt,
                                          "cpu_baseline": {"value": cpu_s * 1e3, "unit": "ms", "kind": "port",
                                                           "cores": os.cpu_count(),
                                                           "sample": "the whole small graph, CPU oracle"},
                                          "gpu_vs_cpu": cpu_s * 1e3 / sms}}), flush=True)
    small.free()
    g.free()
    return 0


def load_lib():
    from gary_b200 import _lib
    return _lib.load()


def main():
    from gary_b200.dist import Dist

    args = parse()
    dist = Dist.from_env()
    if args.workload == "setops":
        return run_setops(args, dist)
    if args.workload == "batch":
        return run_batch(args, dist)
    if args.workload == "patterns":
        return run_patterns(args, dist)
    if args.impl == "reference":
        return run_reference(args, dist)
    return run_ours(args, dist)


if __name__ == "__main__":
    sys.exit(main())
