"""Batched set operations (include/ops of the reference): generator checks on
the CPU, kernel parity against the oracle's std::set_intersection restatement
and the reference's own search templates on the GPU."""
from __future__ import annotations

import numpy as np
import pytest

from gary_b200 import setops as so
from gary_b200 import _lib
from oracle import oracle as O
from vectors import search_case, unpack_bits


@pytest.fixture(scope="module")
def cdf():
    return so.zipf_table(65536, 1.2)


def test_zipf_table(cdf):
    assert cdf[-1] == np.iinfo(np.uint64).max
    assert np.all(np.diff(cdf.astype(np.float64)) >= 0)
    # P(len = 1) = 1 / H(65536, 1.2)
    H = np.sum(np.arange(1, 65537, dtype=np.float64) ** -1.2)
    assert abs(float(cdf[0]) / 2**64 - 1 / H) < 1e-9


def test_pair_generator_host(cdf):
    lens = []
    for p in range(2000):
        a, b = so.gen_pair_host(7, p, cdf, 0.25)
        for x in (a, b):
            assert len(x) >= 1 and len(x) <= 65536
            assert np.all(np.diff(x.astype(np.int64)) > 0) and x[-1] < so.RANGE
        lens += [len(a), len(b)]
        # planted overlap: at least some of the shorter list is in the longer one
        s, l = (a, b) if len(a) <= len(b) else (b, a)
        if len(s) >= 64 and len(l) >= 2 * len(s):
            frac = len(np.intersect1d(s, l)) / len(s)
            assert 0.1 < frac < 0.4
    lens = np.array(lens)
    assert 5 <= np.median(lens) <= 20
    a2, b2 = so.gen_pair_host(7, 5, cdf, 0.25)
    a3, b3 = so.gen_pair_host(7, 5, cdf, 0.25)
    assert np.array_equal(a2, a3) and np.array_equal(b2, b3)


def test_no_overlap_is_sparse(cdf):
    hits = tot = 0
    for p in range(300):
        a, b = so.gen_pair_host(3, p, cdf, 0.0)
        hits += O.intersect(a, b)
        tot += min(len(a), len(b))
    assert hits <= 0.01 * tot + 5


@pytest.mark.gpu
def test_device_generator_matches_host(cdf, cuda):
    batch = so.PairBatch.generate(11, 1000, 512, cdf, 0.1)
    la, lb = batch.la.cpu().numpy(), batch.lb.cpu().numpy()
    ao, bo = batch.a_off.cpu().numpy(), batch.b_off.cpu().numpy()
    A, B = batch.a.cpu().numpy().view(np.uint32), batch.b.cpu().numpy().view(np.uint32)
    for i in range(512):
        a, b = so.gen_pair_host(11, 1000 + i, cdf, 0.1)
        assert la[i] == len(a) and lb[i] == len(b)
        assert np.array_equal(A[ao[i]:ao[i] + la[i]], a)
        assert np.array_equal(B[bo[i]:bo[i] + lb[i]], b)
        assert ao[i] % 4 == 0 and np.all(A[ao[i] + la[i]:ao[i + 1]] == 0xFFFFFFFF)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["auto", "merge", "search", "bitmap"])
@pytest.mark.parametrize("overlap", [0.0, 0.5])
def test_intersect_counts_and_outputs(cdf, cuda, variant, overlap):
    npairs = 3000
    batch = so.PairBatch.generate(5, 77, npairs, cdf, overlap)
    counts, total, out, out_off = so.intersect(batch, so.VARIANTS[variant], materialise=True)
    counts = counts.cpu().numpy()
    out = out.cpu().numpy().view(np.uint32)
    out_off = out_off.cpu().numpy()
    want_total = 0
    for i in range(npairs):
        a, b = so.gen_pair_host(5, 77 + i, cdf, overlap)
        ref = O.intersect(a, b, materialise=True)
        assert counts[i] == len(ref), (variant, i)
        assert np.array_equal(out[out_off[i]:out_off[i] + counts[i]], ref), (variant, i)
        want_total += len(ref)
    assert int(total.item()) == want_total
    # count-only run agrees
    c2, t2 = so.intersect(batch, so.VARIANTS[variant])
    assert int(t2.item()) == want_total


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["merge", "search", "bitmap"])
def test_intersect_edge_cases(cuda, variant):
    import torch

    cases = [([], [1, 2]), ([5], [5]), ([5], [6]), (list(range(31)), list(range(0, 62, 2))),
             (list(range(32)), list(range(32))), (list(range(33)), list(range(1, 34))),
             (list(range(0, 3000, 3)), list(range(0, 3000, 2))), ([0, 4294967294], [4294967294]),
             (list(range(100000, 101000)), list(range(200000, 201000))),
             (list(range(0, 2_000_000, 7)), [7 * 1000, 7 * 99999, 5])]
    cases = [(np.array(sorted(set(a)), np.uint32), np.array(sorted(set(b)), np.uint32)) for a, b in cases]
    la = np.array([len(a) for a, _ in cases], np.int32)
    lb = np.array([len(b) for _, b in cases], np.int32)
    ao = np.concatenate([[0], np.cumsum((la + 3) // 4 * 4)]).astype(np.int64)
    bo = np.concatenate([[0], np.cumsum((lb + 3) // 4 * 4)]).astype(np.int64)
    A = np.full(max(ao[-1], 4), 0xFFFFFFFF, np.uint32)
    B = np.full(max(bo[-1], 4), 0xFFFFFFFF, np.uint32)
    for i, (a, b) in enumerate(cases):
        A[ao[i]:ao[i] + len(a)] = a
        B[bo[i]:bo[i] + len(b)] = b
    t = lambda x, dt: torch.from_numpy(np.ascontiguousarray(x).view(dt)).cuda()  # noqa: E731
    batch = so.PairBatch(len(cases), t(la, np.int32), t(lb, np.int32), t(ao, np.int64), t(bo, np.int64),
                         t(A, np.int32), t(B, np.int32))
    counts, total, out, out_off = so.intersect(batch, so.VARIANTS[variant], materialise=True)
    counts = counts.cpu().numpy()
    out = out.cpu().numpy().view(np.uint32)
    for i, (a, b) in enumerate(cases):
        ref = np.intersect1d(a, b)
        assert counts[i] == len(ref), (variant, i)
        o = int(out_off[i].item())
        assert np.array_equal(out[o:o + counts[i]], ref), (variant, i)


@pytest.mark.gpu
def test_search_matches_reference_golden(golden, cuda):
    """gary_search_batch against the reference's own binary_search /
    binary_search_2phase results (tests/golden)."""
    import torch

    for c in golden["search"]:
        lst, keys = search_case(c["seed"], c["n_list"], c["n_keys"], c["lo"], c["hi"], c["sort_keys"])
        f1 = unpack_bits(c["found"], c["n_keys"])
        f2 = unpack_bits(c["found_2phase"], c["n_keys"])
        dl = torch.from_numpy(lst.astype(np.int32)).cuda()
        dk = torch.from_numpy(keys.astype(np.int32)).cuda()
        for cache, want in ((0, f1), (32, f2), (256, f2), (8192, f2)):
            found, count = so.search(dl, dk, cache)
            assert np.array_equal(found.cpu().numpy(), want), (c["seed"], cache)
            assert int(count.item()) == int(want.sum())


@pytest.mark.gpu
def test_search_large(cuda):
    import torch

    lst, keys = search_case(9, 4 << 20, 1 << 16, 1 << 29, 1 << 30, False)
    dl = torch.from_numpy(lst).cuda()
    dk = torch.from_numpy(keys).cuda()
    want = np.isin(keys, lst).astype(np.uint8)
    for cache in (0, 32, 4096):
        found, count = so.search(dl, dk, cache)
        assert np.array_equal(found.cpu().numpy(), want)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["auto", "merge", "search", "bitmap"])
def test_intersect_num_bounded_and_filtered(cdf, cuda, variant):
    """The intersect_num family: members below a per-pair bound and outside a
    per-pair list of excluded ids (with repeats), against the oracle's merge."""
    import torch

    npairs = 2000
    batch = so.PairBatch.generate(9, 300, npairs, cdf, 0.5)
    rng = np.random.default_rng(3)
    bound = rng.integers(0, 1 << 26, npairs).astype(np.uint32)
    bound[::7] = 0xFFFFFFFF  # no effective bound
    bound[::11] = 0          # empty range
    pairs = [so.gen_pair_host(9, 300 + i, cdf, 0.5) for i in range(npairs)]
    ex, ex_off = [], [0]
    for a, b in pairs:
        common = O.intersect(a, b, materialise=True)
        k = int(rng.integers(0, 5))
        pick = list(rng.choice(common, size=min(k, len(common)), replace=False)) if len(common) else []
        pick += [int(rng.integers(0, 1 << 26))]          # usually not a member
        if pick:
            pick.append(pick[0])                          # a repeat is excluded once
        ex += pick
        ex_off.append(len(ex))
    dev = lambda x, dt: torch.from_numpy(np.asarray(x, dt).view(dt)).cuda()  # noqa: E731
    tb = dev(bound.view(np.int32), np.int32)
    teo = dev(ex_off, np.int64)
    tex = dev(np.asarray(ex, np.uint32).view(np.int32), np.int32)
    counts, total = so.intersect_num(batch, tb, teo, tex, so.VARIANTS[variant])
    counts = counts.cpu().numpy()
    want_total = 0
    for i, (a, b) in enumerate(pairs):
        common = O.intersect(a, b, materialise=True)
        excl = set(ex[ex_off[i]:ex_off[i + 1]])
        want = sum(1 for x in common if x < bound[i] and int(x) not in excl)
        assert counts[i] == want, (variant, i)
        want_total += want
    assert int(total.item()) == want_total
    # no bound and no exclusions: the plain counts
    c0, t0 = so.intersect_num(batch, variant=so.VARIANTS[variant])
    c1, t1 = so.intersect(batch, so.VARIANTS[variant])
    assert torch.equal(c0, c1) and int(t0.item()) == int(t1.item())
