"""The learned cost model of the triangle kernel: data collection, training
(on the device, through the project's own MLP kernels), files, evaluation.

    python -m gary_b200.costmodel train --scales 18,19,20,21,22 \
        --out gary_b200/data/cost_model.gmlp
    python -m gary_b200.costmodel eval --model gary_b200/data/cost_model.gmlp --scale 24 [--bound]

Training data is logged by the instrumented plain kernel itself: for every
middle vertex of the triangle kernel, clock64 cycles with each intersection
variant forced in turn (hash, search, regs: at most 8 ids in registers, bitmap), next to the vertex's
six features.  A sample carries targets only for the variants that are legal
for it.  The network predicts log2 cycles per variant; GARY_SCHED_LEARNED
picks the cheapest legal variant per vertex and weights tiles by it.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time
from pathlib import Path

import numpy as np

from ._lib import GARY_PATTERN_TRIANGLE, GARY_SCHED_LEARNED, GARY_SCHED_PLAIN, check, load

N_IN, N_OUT = 6, 4
VARIANTS = ("hash", "search", "regs", "bitmap")
DEFAULT_MODEL = Path(__file__).resolve().parent / "data" / "cost_model.gmlp"


def n_params() -> int:
    return int(load().gary_mlp_param_count())


class CostModel:
    def __init__(self, params: np.ndarray):
        self.params = np.ascontiguousarray(params, np.float32)
        assert self.params.size == n_params()

    @classmethod
    def init(cls, seed: int = 0) -> "CostModel":
        p = np.zeros(n_params(), np.float32)
        check(load().gary_mlp_init(seed, p.ctypes.data), "gary_mlp_init")
        return cls(p)

    @classmethod
    def load(cls, path=DEFAULT_MODEL) -> "CostModel":
        p = np.zeros(n_params(), np.float32)
        check(load().gary_mlp_load(str(path).encode(), p.ctypes.data), "gary_mlp_load")
        return cls(p)

    def save(self, path) -> None:
        Path(path).parent.mkdir(parents=True, exist_ok=True)
        check(load().gary_mlp_save(str(path).encode(), self.params.ctypes.data), "gary_mlp_save")

    def install(self) -> None:
        """Make this the process-wide model of GARY_SCHED_LEARNED."""
        check(load().gary_set_cost_model(self.params.ctypes.data), "gary_set_cost_model")

    def predict(self, x: np.ndarray) -> np.ndarray:
        """Raw features [n, 6] -> predicted log2 cycles [n, 4] (on the device)."""
        import torch

        dp = torch.from_numpy(self.params).cuda()
        dx = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
        dy = torch.empty((len(x), N_OUT), dtype=torch.float32, device="cuda")
        check(load().gary_mlp_forward(dp.data_ptr(), dx.data_ptr(), len(x), 1, dy.data_ptr(), None),
              "gary_mlp_forward")
        return dy.cpu().numpy()


def profile(g, variants=(0, 1, 2, 3), repeats: int = 1):
    """(features [n,6], legal [n], {variant: cycles [n]}, count) of graph g."""
    import torch

    n = g.info()["n"]
    L = load()
    x = torch.empty((n, N_IN), dtype=torch.float32, device="cuda")
    legal = torch.empty(n, dtype=torch.uint8, device="cuda")
    check(L.gary_tc_features(g.handle, x.data_ptr(), legal.data_ptr(), None), "gary_tc_features")
    cyc = torch.empty(n, dtype=torch.int64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    out, counts = {}, set()
    for v in variants:
        acc = np.zeros(n, np.float64)
        for _ in range(repeats):
            check(L.gary_tc_profile(g.handle, v, cyc.data_ptr(), cnt.data_ptr(), None), "gary_tc_profile")
            torch.cuda.synchronize()
            acc += cyc.cpu().numpy().astype(np.float64)
            counts.add(int(cnt.item()))
        out[v] = acc / repeats
    assert len(counts) == 1, f"variants disagree on the count: {counts}"
    return x.cpu().numpy(), legal.cpu().numpy(), out, counts.pop()


def dataset(x, legal, cycles, max_rows: int, seed: int = 0):
    """Rows with at least one measured legal variant: (X, T=log2 cycles, mask)."""
    rows = np.nonzero(legal)[0]
    rng = np.random.default_rng(seed)
    if len(rows) > max_rows:
        rows = np.sort(rng.choice(rows, max_rows, replace=False))
    T = np.zeros((len(rows), N_OUT), np.float32)
    M = np.zeros(len(rows), np.uint8)
    for k, c in cycles.items():
        ok = ((legal[rows] >> k) & 1).astype(bool) & (c[rows] > 0)
        T[ok, k] = np.log2(c[rows][ok])
        M[ok] |= np.uint8(1 << k)
    keep = M != 0
    return x[rows][keep].astype(np.float32), T[keep], M[keep]


def train(X, T, M, epochs: int = 30, batch: int = 4096, lr: float = 2e-3, seed: int = 0,
          val_frac: float = 0.1, log=print) -> tuple[CostModel, dict]:
    """Fit the network on the device with gary_mlp_grad / gary_mlp_adam."""
    import torch

    L = load()
    rng = np.random.default_rng(seed)
    perm = rng.permutation(len(X))
    nval = max(1, int(len(X) * val_frac))
    vi, ti = perm[:nval], perm[nval:]
    model = CostModel.init(seed)
    p = model.params
    mu_x, sd_x = X[ti].mean(0), X[ti].std(0) + 1e-6
    mu_y = np.zeros(N_OUT, np.float32)
    sd_y = np.ones(N_OUT, np.float32)
    for k in range(N_OUT):
        sel = ((M[ti] >> k) & 1).astype(bool)
        if sel.any():
            mu_y[k] = T[ti][sel, k].mean()
            sd_y[k] = T[ti][sel, k].std() + 1e-6
    p[0:6], p[6:12], p[12:16], p[16:20] = mu_x, sd_x, mu_y, sd_y
    Xs = ((X - mu_x) / sd_x).astype(np.float32)
    Ts = ((T - mu_y) / sd_y).astype(np.float32)
    dev = "cuda"
    dX, dT, dM = (torch.from_numpy(a).to(dev) for a in (Xs, Ts, M))
    dP = torch.from_numpy(p.copy()).to(dev)
    dG = torch.zeros_like(dP)
    dm = torch.zeros_like(dP)
    dv = torch.zeros_like(dP)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    train_idx = torch.from_numpy(ti).to(dev)
    step = 0
    hist = []
    for ep in range(epochs):
        order = train_idx[torch.randperm(len(ti), device=dev, generator=torch.Generator(device=dev).manual_seed(seed + ep))]
        tot = 0.0
        cells = 0
        for b0 in range(0, len(order), batch):
            idx = order[b0:b0 + batch]
            bx, bt, bm = dX[idx].contiguous(), dT[idx].contiguous(), dM[idx].contiguous()
            nc = int(sum(((bm >> k) & 1).sum().item() for k in range(N_OUT)))
            check(L.gary_mlp_grad(dP.data_ptr(), bx.data_ptr(), bt.data_ptr(), bm.data_ptr(), len(idx),
                                  float(max(nc, 1)), dG.data_ptr(), loss.data_ptr(), None), "gary_mlp_grad")
            step += 1
            check(L.gary_mlp_adam(dP.data_ptr(), dG.data_ptr(), dm.data_ptr(), dv.data_ptr(), step, lr, None),
                  "gary_mlp_adam")
            tot += float(loss.item())
            cells += nc
        hist.append(tot / max(cells, 1))
        if log and (ep % 5 == 0 or ep == epochs - 1):
            log(f"epoch {ep}: train mse (standardised) {hist[-1]:.4f}")
    model = CostModel(dP.cpu().numpy())
    # validation in log2-cycle units
    pred = model.predict(X[vi])
    stats = {"train_rows": int(len(ti)), "val_rows": int(nval), "loss_curve": hist}
    for k, name in enumerate(VARIANTS):
        sel = ((M[vi] >> k) & 1).astype(bool)
        if sel.sum() > 10:
            err = pred[sel, k] - T[vi][sel, k]
            var = T[vi][sel, k].var()
            stats[f"val_rmse_log2_{name}"] = float(np.sqrt((err ** 2).mean()))
            stats[f"val_r2_{name}"] = float(1 - (err ** 2).mean() / max(var, 1e-9))
    return model, stats


def time_scheds(g, steps: int = 5):
    """Kernel ms of the plain and learned plans on graph g (CUDA events)."""
    import torch

    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    res = {}
    for name, sched in (("plain", GARY_SCHED_PLAIN), ("learned", GARY_SCHED_LEARNED)):
        for _ in range(2):
            g.count_async(out, GARY_PATTERN_TRIANGLE, sched)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            g.count_async(out, GARY_PATTERN_TRIANGLE, sched)
        e1.record()
        torch.cuda.synchronize()
        res[name] = {"ms": e0.elapsed_time(e1) / steps, "count": int(out.item())}
    return res


def variant_bound(g, model: "CostModel | None" = None) -> dict:
    """What per-vertex variant choice can gain on graph g: every warp-class
    middle vertex is run with each legal variant forced; returns the summed
    cycles of the plain dispatch, of the best legal variant per vertex (the
    bound), and (with a model) of the model's choices."""
    x, legal, cyc, cnt = profile(g, variants=(-1, 0, 1, 2, 3))
    w = legal != 0
    C_ = np.stack([cyc[k][w] for k in range(N_OUT)], 1)
    ok = np.stack([((legal[w] >> k) & 1).astype(bool) & (cyc[k][w] > 0) for k in range(N_OUT)], 1)
    best = np.where(ok, C_, np.inf).min(1)
    best = np.where(np.isfinite(best), best, cyc[-1][w])
    res = {"warp_vertices": int(w.sum()), "plain_cycles": float(cyc[-1][w].sum()),
           "best_cycles": float(best.sum()), "bound_gain": float(cyc[-1][w].sum() / best.sum()),
           "count": cnt}
    if model is not None and w.any():
        pred = model.predict(x[w])
        choice = np.where(ok, pred, np.inf).argmin(1)
        res["model_cycles"] = float(C_[np.arange(len(C_)), choice].sum())
    return res


def _graph(scale: int, ef: int, seed: int):
    import torch

    import gary_b200 as gb

    n = 1 << scale
    src, dst = gb.gen_rmat_device(scale, seed, ef << scale)
    csr = gb.csr_from_edges_device(src, dst, n)
    del src, dst
    torch.cuda.empty_cache()
    p, i = csr.device_ptrs()
    _, nnz = csr.shape()
    out = C.c_void_p()
    from ._lib import GARY_INPUT_DEVICE

    check(load().gary_graph_upload(p, i, n, nnz, GARY_INPUT_DEVICE, None, C.byref(out)), "gary_graph_upload")
    csr.free()
    return gb.Graph(out.value)


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--scales", default="18,19,20,21,22")
    t.add_argument("--ef", type=int, default=16)
    t.add_argument("--rows", type=int, default=250_000, help="samples per training graph")
    t.add_argument("--epochs", type=int, default=40)
    t.add_argument("--out", default=str(DEFAULT_MODEL))
    t.add_argument("--report", default=None, help="write a JSON training report here")
    e = sub.add_parser("eval")
    e.add_argument("--model", default=str(DEFAULT_MODEL))
    e.add_argument("--scale", type=int, default=24)
    e.add_argument("--ef", type=int, default=32)
    e.add_argument("--bound", action="store_true",
                   help="also profile every variant per vertex and report the per-vertex choice bound")
    a = ap.parse_args(argv)
    if a.cmd == "train":
        Xs, Ts, Ms = [], [], []
        t0 = time.time()
        for i, sc in enumerate(int(x) for x in a.scales.split(",")):
            g = _graph(sc, a.ef, 100 + i)
            x, legal, cyc, cnt = profile(g)
            X, T, M = dataset(x, legal, cyc, a.rows, seed=i)
            Xs.append(X), Ts.append(T), Ms.append(M)
            print(f"rmat{sc} ef{a.ef}: {len(X)} samples, triangles {cnt}", flush=True)
            g.free()
        X, T, M = np.concatenate(Xs), np.concatenate(Ts), np.concatenate(Ms)
        model, stats = train(X, T, M, epochs=a.epochs)
        model.save(a.out)
        stats["seconds"] = time.time() - t0
        stats["scales"] = a.scales
        print(json.dumps({k: v for k, v in stats.items() if k != "loss_curve"}), flush=True)
        if a.report:
            Path(a.report).write_text(json.dumps(stats, indent=1))
    else:
        model = CostModel.load(a.model)
        model.install()
        g = _graph(a.scale, a.ef, 1)
        res = {"scale": a.scale, "ef": a.ef, **time_scheds(g)}
        if a.bound:
            res["variant_choice"] = variant_bound(g, model)
        print(json.dumps(res), flush=True)
        g.free()


if __name__ == "__main__":
    main()
