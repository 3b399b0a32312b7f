"""The device BVH build reproduces Builder.subdivide's in-place partition
(src/bvh.zig:175-182, a Lomuto partition) without running it sequentially:
position q < mid receives the left-going element of rank q; position
q >= mid keeps s_q when s_q goes right, else receives G(rank(q)), with
G(k) = s_k if s_k goes right, else G(rank(k)).  This checks the formula, as
the device kernels evaluate it (prefix counts, then pointer jumping), against
the sequential loop on random inputs.
"""
import numpy as np


def lomuto(s, left):
    r = list(s)
    mid = 0
    for j in range(len(r)):
        if left[r[j]]:
            r[mid], r[j] = r[j], r[mid]
            mid += 1
    return r


def by_formula(s, left):
    n = len(s)
    L = np.array([left[e] for e in s], bool)
    rank = np.concatenate([[0], np.cumsum(L)[:-1]]).astype(np.int64)
    mid = int(L.sum())
    nxt = np.where(L, rank, np.arange(n))  # pointer jumping: root(p) = p for right-going, else root(rank(p))
    for _ in range(max(1, int(np.ceil(np.log2(max(n, 2)))))):
        nxt = nxt[nxt]
    out = np.empty(n, np.int64)
    out[rank[L]] = np.asarray(s)[L]  # left-going elements in order
    q = np.arange(mid, n)
    out[q] = np.where(L[q], np.asarray(s)[nxt[rank[q]]], np.asarray(s)[q])
    return list(out)


def test_formula_matches_lomuto():
    rng = np.random.default_rng(0)
    for trial in range(2000):
        n = int(rng.integers(1, 80))
        s = list(rng.permutation(1000)[:n])
        p = rng.uniform(0.05, 0.95)
        left = {e: bool(rng.random() < p) for e in s}
        assert by_formula(s, left) == lomuto(s, left), (s, left)


def test_formula_edge_patterns():
    for pattern in ("LLLL", "RRRR", "LRLR", "RLRL", "RRLL", "LLRR", "RLLLR", "L", "R"):
        s = list(range(len(pattern)))
        left = {i: c == "L" for i, c in enumerate(pattern)}
        assert by_formula(s, left) == lomuto(s, left)
