"""Shared helpers for the PPR / adjoint tests."""
import numpy as np


def seed_teleports(g, k, rng, max_seeds=64):
    """k teleport columns, each uniform over a log-uniform-sized seed set of
    non-isolated vertices."""
    n = g.num_nodes
    cand = np.nonzero(np.diff(g.out_offsets) > 0)[0]
    T = np.zeros((n, k), np.float32)
    for c in range(k):
        size = int(np.exp(rng.uniform(0, np.log(max_seeds))))
        seeds = rng.choice(cand, size=min(size, cand.size), replace=False)
        T[seeds, c] = np.float32(1.0 / seeds.size)
    return T


def in_weights(g, ew):
    """Weight of each in-CSR entry (v -> u) looked up in v's out-row."""
    n = g.num_nodes
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(g.out_offsets))
    key_out = src * n + g.out_neighbors
    dst = np.repeat(np.arange(n, dtype=np.int64), np.diff(g.in_offsets))
    key_in = g.in_neighbors.astype(np.int64) * n + dst
    pos = np.searchsorted(key_out, key_in)
    assert np.all(key_out[pos] == key_in)
    return ew[pos].astype(np.float64)


def row_sums(g, ew):
    out = np.zeros(g.num_nodes, np.float64)
    src = np.repeat(np.arange(g.num_nodes), np.diff(g.out_offsets))
    np.add.at(out, src, ew.astype(np.float64))
    return out
