"""Definitions of the measured workloads, shared by bench.py, suite.py, the
fixture scripts and the tests.  Pure numpy: importing this module loads
neither the engine nor the oracle, so the CPU reference arm of bench.py can
build the very same inputs without touching libgpm.so.

Workloads (seeded synthetic graphs; the public datasets the reference lists
are not available here):
  tc       R-MAT scale 22, edge factor 16, (a,b,c,d) = (.57,.19,.19,.05),
           seed 1 (+ rank), symmetrised and simple, degree-oriented
  clique   4- and 5-cliques of R-MAT scale 20 (same law, seed 1)
  motif    256 Chung-Lu graphs: n log-uniform in [1e3, 1e6], exponent
           U[2.1, 2.8], mean degree U[8, 64] (member parameters from
           numpy seed 5, member m drawn with seed 11 + m), all 3- and
           4-vertex induced motifs
  match    R-MAT scale 21 (edge factor 16, seed 3) with 8 Zipf(1.2) vertex
           labels (seed 3); five queries walked on the data graph (numpy
           seed 3): triangle, 4-cycle, diamond, house, 6-vertex pyramid
           (an apex over a 5-cycle), labels copied from the walked vertices
"""
from __future__ import annotations

import numpy as np

RMAT_ABC = (0.57, 0.19, 0.19)
EDGE_FACTOR = 16
TC_SCALE, TC_SEED = 22, 1
CLIQUE_SCALE, CLIQUE_SEED = 20, 1
MATCH_SCALE, MATCH_SEED, MATCH_LABELS, MATCH_ZIPF = 21, 3, 8, 1.2
BATCH_COUNT, BATCH_NMIN, BATCH_NMAX, BATCH_PARAM_SEED, BATCH_SEED = 256, 1e3, 1e6, 5, 11

# query shapes of the labelled workload (edges); pyramid-6 = apex over a 5-cycle
SHAPES = {
    "triangle": (3, [(0, 1), (1, 2), (2, 0)]),
    "cycle4": (4, [(0, 1), (1, 2), (2, 3), (3, 0)]),
    "diamond": (4, [(0, 1), (0, 2), (0, 3), (1, 2), (2, 3)]),
    "house": (5, [(0, 1), (0, 4), (1, 2), (1, 4), (2, 3), (3, 4)]),
    "pyramid6": (6, [(0, 1), (0, 2), (0, 3), (0, 4), (0, 5), (1, 2), (2, 3), (3, 4), (4, 5), (5, 1)]),
}


def walk_query(off, idx, labels, shape, rng, tries=2000):
    """An embedding of `shape` found by a seeded randomised walk (depth-first,
    random neighbour order); returns the walked vertices' labels."""
    k, edges = shape
    adj = [set() for _ in range(k)]
    for a, b in edges:
        adj[a].add(b)
        adj[b].add(a)
    n = len(off) - 1
    deg = np.diff(off)

    def nbrs(v):
        return idx[off[v]:off[v + 1]]

    def has(a, b):
        lst = nbrs(a)
        i = np.searchsorted(lst, b)
        return i < len(lst) and lst[i] == b

    for _ in range(tries):
        start = int(rng.integers(n))
        if deg[start] < len(adj[0]):
            continue
        emb = [start]

        def extend(i):
            if i == k:
                return True
            parent = next(j for j in range(i) if j in adj[i])
            cand = nbrs(emb[parent])
            for v in rng.permutation(cand)[:64]:
                v = int(v)
                if v in emb or deg[v] < len(adj[i]):
                    continue
                if all(has(emb[j], v) for j in range(i) if j in adj[i]):
                    emb.append(v)
                    if extend(i + 1):
                        return True
                    emb.pop()
            return False

        if extend(1):
            return labels[np.array(emb)]
    raise RuntimeError("no embedding found")


def walk_queries(off, idx, labels, seed=MATCH_SEED):
    """The five labelled queries of the match workload, in SHAPES order:
    {name: (k, edges int32[m, 2], labels int32[k])}."""
    rng = np.random.default_rng(seed)
    out = {}
    for name, shape in SHAPES.items():
        ql = walk_query(off, idx, labels, shape, rng)
        out[name] = (shape[0], np.array(shape[1], np.int32), np.asarray(ql, np.int32))
    return out


def batch_members(count=BATCH_COUNT, nmax=BATCH_NMAX, seed=BATCH_PARAM_SEED, nmin=BATCH_NMIN):
    """Member parameters of the batched motif workload: (n, exponent, mean degree)."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(nmin), np.log(nmax), count)).astype(np.int64)
    gam = rng.uniform(2.1, 2.8, count)
    md = rng.uniform(8, 64, count)
    return n, gam, md


def mix64(x: int) -> int:
    """splitmix64's finaliser (the engine's per-member seed: member m of a
    batch generated with seed s draws with mix64(s + m))."""
    M = (1 << 64) - 1
    x = (x + 0x9E3779B97F4A7C15) & M
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M
    return x ^ (x >> 31)


def member_seed(m: int, seed: int = BATCH_SEED) -> int:
    return mix64((seed + m) & ((1 << 64) - 1))
