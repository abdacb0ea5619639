"""The N>1 path on CPU: two gloo ranks run the same host code the benchmark
runs under torchrun (gary_b200.dist), with a shard counter in place of the
GPU kernel.  Shards of a count must sum to the oracle's total; max/gather
reductions must be exact; a rank that fails before a collective must end the
other rank's collective with an error, not a hang."""
from __future__ import annotations

import multiprocessing as mp
import os
import socket
import time

import numpy as np
import pytest

from oracle import oracle as O


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _graph(seed=3, n=600, m=6000):
    r = np.random.default_rng(seed)
    s = r.integers(0, n, m).astype(np.uint32)
    d = (r.integers(0, n, m) ** 1).astype(np.uint32)
    ptr, idx = O.sym_csr(s, d, n)
    return O.orient(ptr, idx)


def _shard_count(dptr, didx, shard, nshards):
    """Triangles whose lowest-ordered vertex lies in the shard's row range."""
    n = len(dptr) - 1
    lo, hi = shard * n // nshards, (shard + 1) * n // nshards
    t = 0
    for u in range(lo, hi):
        nu = didx[dptr[u]:dptr[u + 1]]
        for v in nu:
            t += len(np.intersect1d(nu, didx[dptr[v]:dptr[v + 1]], assume_unique=True))
    return t


def _worker(rank, world, port, mode, out_q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from gary_b200.dist import Dist, sharded_total

    d = Dist.from_env(timeout_s=20.0).init(backend="gloo")
    try:
        if mode == "count":
            dptr, didx = _graph()
            local, total = sharded_total(d, lambda s, k: _shard_count(dptr, didx, s, k))
            out_q.put((rank, "count", local, total))
        elif mode == "reduce":
            mx = d.allreduce(1.5 + rank, "max")
            mn = d.allreduce(7 - rank, "min")
            big = d.allreduce((1 << 40) + rank, "sum")
            g = d.gather(10 * rank + 1)
            d.barrier()
            out_q.put((rank, "reduce", mx, mn, big, g))
        elif mode == "fail":
            if rank == 1:
                raise SystemExit(3)  # leaves before the collective
            t0 = time.time()
            try:
                d.allreduce(1, "sum")
                out_q.put((rank, "fail", "no error", time.time() - t0))
            except Exception as e:  # noqa: BLE001 - any error ends the wait
                out_q.put((rank, "fail", type(e).__name__, time.time() - t0))
    finally:
        if mode != "fail":
            d.close()


def _run(mode, world=2, limit=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    deadline = time.time() + limit
    for p in procs:
        p.join(max(1.0, deadline - time.time()))
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
        p.join()
    assert not alive, f"{mode}: ranks still running after {limit}s"
    res = []
    while not q.empty():
        res.append(q.get())
    return sorted(res), [p.exitcode for p in procs]


def test_sharded_count_sums_to_oracle():
    res, codes = _run("count")
    assert codes == [0, 0]
    dptr, didx = _graph()
    want = O.tri_count(dptr, didx)
    locals_ = [r[2] for r in res]
    assert len(res) == 2 and all(r[3] == want for r in res)
    assert sum(locals_) == want and min(locals_) > 0


def test_reductions_exact():
    res, codes = _run("reduce")
    assert codes == [0, 0]
    for r in res:
        _, _, mx, mn, big, g = r
        assert mx == 2.5 and mn == 6 and big == 2 * (1 << 40) + 1 and g == [1, 11]


@pytest.mark.timeout(180)
def test_failed_rank_ends_collective_with_error():
    res, codes = _run("fail", limit=150)
    assert codes[1] == 3
    (rank, _, err, waited), = res
    assert rank == 0 and err != "no error" and waited < 60
