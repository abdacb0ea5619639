"""Regenerate the input graphs named by the golden fixtures."""
from __future__ import annotations

import itertools

import numpy as np

import gary_b200 as gb
from vectors import edge_checksum


def edges_of(case) -> tuple[int, np.ndarray, np.ndarray]:
    gen = case["gen"]
    if gen == "explicit":
        e = np.array(case["edges"], np.uint32).reshape(-1, 2)
        src, dst, n = e[:, 0].copy(), e[:, 1].copy(), case["n"]
    elif gen == "er+clique":
        a = case["gen_args"]
        s, d = gb.gen_er(a["n"], a["m"], a["seed"])
        cl = np.array(list(itertools.combinations(range(*a["clique"]), 2)), np.uint32)
        src = np.concatenate([s, cl[:, 0]])
        dst = np.concatenate([d, cl[:, 1]])
        n = a["n"]
    elif gen == "er":
        a = case["gen_args"]
        src, dst = gb.gen_er(a["n"], a["m"], a["seed"])
        n = a["n"]
    elif gen == "rmat":
        a = case["gen_args"]
        src, dst = gb.gen_rmat(a["scale"], a["seed"], a["ef"] << a["scale"])
        n = 1 << a["scale"]
    else:
        raise ValueError(gen)
    assert edge_checksum(src, dst) == case["edge_digest"], f"{case['name']}: generator drifted"
    return n, src, dst
