"""Counts of the reference's own sub_ceci matcher for query graphs of 16 to 64
vertices, as a golden fixture (ceci_wide.npz).

    python tests/golden/make_ceci_wide_golden.py [--timeout 600]

sub_ceci is built from the reference's sources into oracle/_ref/myceci
(`make -C oracle ref`); it accepts queries of up to 64 vertices
(sub_ceci/configuration/config.h:12).  Data graphs: seeded uniform random
labelled graphs (numpy default_rng(20261204)).  Queries: a connected vertex
set of the data graph grown from a random start by random frontier picks
(so every query has at least one embedding), labels copied from the data
graph, edges = a spanning tree of the growth plus a random share of the other
edges among the set (0, half or all of them).  Each (graph, query) pair is
written in sub_ceci's t/v/e format and run as

    myceci -d data.graph -q query.graph -filter CECI -order CECI -engine CECI

rows whose run exceeds --timeout seconds are left out.  ceci_wide.npz holds
the graphs (concatenated edge and label arrays with lengths), the queries
(sizes, concatenated edges, labels) and sub_ceci's #Embeddings per query.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from make_golden import run_ceci, write_tve  # noqa: E402

SIZES = (16, 17, 20, 24, 32, 40, 48, 64)
CHORD_SHARES = (0.0, 0.5, 1.0)


def grow_query(rng, n, adj, k, share):
    """k connected data vertices and the query edges among them."""
    while True:
        start = int(rng.integers(0, n))
        verts, seen = [start], {start}
        tree = []
        frontier = [(start, w) for w in adj[start]]
        while len(verts) < k and frontier:
            i = int(rng.integers(0, len(frontier)))
            a, b = frontier.pop(i)
            if b in seen:
                continue
            seen.add(b)
            verts.append(b)
            tree.append((a, b))
            frontier.extend((b, w) for w in adj[b] if w not in seen)
        if len(verts) == k:
            break
    pos = {v: i for i, v in enumerate(verts)}
    tset = {(min(a, b), max(a, b)) for a, b in tree}
    chords = sorted({(min(a, b), max(a, b)) for a in verts for b in adj[a] if b in pos} - tset)
    keep = [c for c in chords if rng.random() < share]
    edges = [(pos[a], pos[b]) for a, b in list(tset) + keep]
    return np.array(verts, np.int64), np.array(sorted(edges), np.int32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--timeout", type=float, default=600)
    a = ap.parse_args()
    myceci = os.path.join(ROOT, "oracle", "_ref", "myceci")
    rng = np.random.default_rng(20261204)
    graphs, queries = [], []
    with tempfile.TemporaryDirectory() as td:
        for gi, (gn, deg, nl) in enumerate(((200, 6.0, 4), (400, 5.0, 8), (800, 4.0, 12))):
            gm = int(gn * deg / 2)
            ge = rng.integers(0, gn, size=(gm, 2)).astype(np.int32)
            ge = ge[ge[:, 0] != ge[:, 1]]
            gl = rng.integers(0, nl, size=gn).astype(np.int32)
            adj = [set() for _ in range(gn)]
            for x, y in ge:
                adj[int(x)].add(int(y))
                adj[int(y)].add(int(x))
            adj = [sorted(s) for s in adj]
            dpath = os.path.join(td, f"g{gi}.graph")
            write_tve(dpath, gn, ge, gl)
            graphs.append((gn, ge, gl))
            for k in SIZES:
                for share in CHORD_SHARES:
                    verts, qe = grow_query(rng, gn, adj, k, share)
                    ql = gl[verts].astype(np.int32)
                    qpath = os.path.join(td, f"q{gi}_{k}_{share}.graph")
                    write_tve(qpath, k, qe, ql)
                    try:
                        c = run_ceci_timed(myceci, dpath, qpath, a.timeout)
                    except subprocess.TimeoutExpired:
                        print(f"graph {gi} k {k} share {share}: over {a.timeout} s, left out", flush=True)
                        continue
                    print(f"graph {gi} k {k} share {share}: {len(qe)} edges, {c} embeddings", flush=True)
                    queries.append((gi, k, qe, ql, c))
    np.savez_compressed(
        os.path.join(HERE, "ceci_wide.npz"),
        gn=np.array([g[0] for g in graphs]), ge=np.concatenate([g[1] for g in graphs]),
        ge_len=np.array([len(g[1]) for g in graphs]), gl=np.concatenate([g[2] for g in graphs]),
        q_graph=np.array([q[0] for q in queries]), q_n=np.array([q[1] for q in queries]),
        q_e=np.concatenate([q[2] for q in queries]), q_e_len=np.array([len(q[2]) for q in queries]),
        q_lab=np.concatenate([q[3] for q in queries]),
        expected=np.array([q[4] for q in queries], np.uint64))
    print("wrote ceci_wide.npz:", len(queries), "queries")


def run_ceci_timed(myceci, data, query, timeout):
    import re
    out = subprocess.run([myceci, "-d", data, "-q", query, "-filter", "CECI", "-order", "CECI", "-engine", "CECI"],
                         capture_output=True, text=True, check=True, timeout=timeout).stdout
    return int(re.search(r"#Embeddings: (\d+)", out).group(1))


if __name__ == "__main__":
    main()
