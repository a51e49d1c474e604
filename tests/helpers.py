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


def depths_from_parents(parent, src):
    """Depth of every vertex along BFS parent pointers (-1 unreached)."""
    n = parent.size
    d = np.full(n, -1, np.int32)
    d[src] = 0
    level = np.array([src])
    k = 0
    not_src = np.arange(n) != src
    while level.size:
        nxt = np.nonzero(np.isin(parent, level) & (d == -1) & not_src)[0]
        k += 1
        d[nxt] = k
        level = nxt
    return d
