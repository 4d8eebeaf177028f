"""Labelled subgraph matching (sub_ceci semantics) on the GPU vs known answers."""
import os

import numpy as np
import pytest

import gpm
import _oracle as orc

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def edges_of(off, idx):
    src = np.repeat(np.arange(len(off) - 1), np.diff(off)).astype(np.int32)
    keep = src < idx
    return src[keep], idx[keep]


def test_hprd_known_answers():
    z = np.load(os.path.join(GOLD, "hprd_kat.npz"))
    s, d = edges_of(z["off"], z["idx"])
    g = gpm.Graph.from_edges(len(z["off"]) - 1, s, d, labels=z["labels"])
    po = pi = pl = 0
    for i, m in enumerate(z["qn"]):
        qo = z["qoff"][po: po + m + 1]
        po += m + 1
        qi = z["qidx"][pi: pi + qo[-1]]
        pi += qo[-1]
        ql = z["qlab"][pl: pl + m]
        pl += m
        qs, qd = edges_of(qo, qi)
        assert g.match(gpm.Query(int(m), qs, qd, ql)) == int(z["expected"][i]), i


def test_reference_subceci_random_graphs():
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import SHAPES
    z = np.load(os.path.join(GOLD, "ceci_random.npz"))
    starts = np.concatenate([[0], np.cumsum(z["ge_len"])])
    lstarts = np.concatenate([[0], np.cumsum(z["gn"])])
    shapes = list(SHAPES.values())
    for row in z["rows"]:
        gi, si = int(row[0]), int(row[1])
        e = z["ge"][starts[gi]: starts[gi + 1]]
        g = gpm.Graph.from_edges(int(z["gn"][gi]), e[:, 0], e[:, 1], labels=z["gl"][lstarts[gi]: lstarts[gi + 1]])
        sn, sedges = shapes[si]
        se = np.array(sedges, np.int32)
        q = gpm.Query(sn, se[:, 0], se[:, 1], np.array(row[2: 2 + sn], np.int32))
        assert g.match(q) == int(row[-1]), (gi, si)


@pytest.mark.parametrize("scale,nl", [(9, 4), (10, 8), (11, 8)])
def test_rmat_zipf_labels_vs_oracle(scale, nl):
    # sizes keep the embedding counts in the millions: enumeration cost is
    # proportional to the count on both sides
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import SHAPES
    n, s, d = gpm.gen_rmat(scale, 8, seed=scale)
    lab = gpm.gen_zipf_labels(n, nl, 1.2, seed=5)
    off, idx = orc.build_csr(n, s, d)
    g = gpm.Graph.from_edges(n, s, d, labels=lab)
    rng = np.random.default_rng(scale)
    for name, (sn, sedges) in SHAPES.items():
        se = np.array(sedges, np.int32)
        ql = lab[rng.integers(0, n, size=sn)]
        qo, qi = orc.build_csr(sn, se[:, 0], se[:, 1])
        want = orc.match(off, idx, lab, qo, qi, ql)
        assert g.match(gpm.Query(sn, se[:, 0], se[:, 1], ql)) == want, name


def test_single_vertex_and_errors():
    g = gpm.Graph.from_edges(4, [0, 1], [1, 2], labels=[1, 1, 2, 1])
    assert g.match(gpm.Query(1, [], [], [1])) == 3
    with pytest.raises(gpm.GpmError):
        gpm.Query(65, [0], [1], np.zeros(65))
    g2 = gpm.Graph.from_edges(4, [0, 1], [1, 2])
    with pytest.raises(gpm.GpmError):
        g2.match(gpm.Query(2, [0], [1], [0, 0]))


def brute_embeddings(off, idx, lab, qn, qedges, qlab):
    """All injective, label-preserving maps of the query that send every
    query edge to a data edge (sub_ceci's embeddings), by backtracking."""
    adj = [set(idx[off[v]:off[v + 1]].tolist()) for v in range(len(off) - 1)]
    qadj = [set() for _ in range(qn)]
    for a, b in qedges:
        qadj[a].add(b)
        qadj[b].add(a)
    out, emb = [], [-1] * qn

    def go(i):
        if i == qn:
            out.append(tuple(emb))
            return
        for v in range(len(off) - 1):
            if lab[v] != qlab[i] or v in emb[:i]:
                continue
            if all(emb[j] in adj[v] for j in range(i) if j in qadj[i]):
                emb[i] = v
                go(i + 1)
                emb[i] = -1

    go(0)
    return out


QUERIES = {
    "vertex": (1, [], [0]),
    "edge": (2, [(0, 1)], [0, 1]),
    "triangle": (3, [(0, 1), (1, 2), (2, 0)], [0, 1, 0]),
    "path3": (3, [(0, 1), (1, 2)], [1, 0, 1]),
    "cycle4": (4, [(0, 1), (1, 2), (2, 3), (3, 0)], [0, 1, 0, 1]),
    "tailed": (4, [(0, 1), (1, 2), (2, 0), (2, 3)], [0, 0, 1, 1]),
}


@pytest.mark.parametrize("name", sorted(QUERIES))
def test_listing_and_limit_vs_brute_force(name):
    """gpm_match_list returns every embedding when the limit allows (as a set
    equal to a brute-force enumeration), and a limit below the total gives
    exactly `limit` distinct valid embeddings; gpm_match_limit = min(total,
    limit) (sub_ceci's -num)."""
    rng = np.random.default_rng(21)
    n = 40
    e = rng.integers(0, n, size=(160, 2)).astype(np.int32)
    lab = rng.integers(0, 2, size=n).astype(np.int32)
    off, idx = orc.build_csr(n, e[:, 0], e[:, 1])
    g = gpm.Graph.from_edges(n, e[:, 0], e[:, 1], labels=lab)
    qn, qe, ql = QUERIES[name]
    qa = np.array([a for a, _ in qe], np.int32)
    qb = np.array([b for _, b in qe], np.int32)
    q = gpm.Query(qn, qa, qb, np.array(ql, np.int32))
    want = set(brute_embeddings(off, idx, lab, qn, qe, ql))
    total = g.match(q)
    assert total == len(want) > 0
    rows = g.match_list(q, total + 5)
    assert len(rows) == total and set(map(tuple, rows.tolist())) == want
    for lim in (1, total // 2 + 1, total):
        assert g.match(q, limit=lim) == min(total, lim)
        part = g.match_list(q, lim)
        got = set(map(tuple, part.tolist()))
        assert len(part) == lim and len(got) == lim and got <= want
    assert g.match(q, limit=0) == 0 and len(g.match_list(q, 0)) == 0


def test_limit_stops_a_large_enumeration():
    """On a graph with ~10^9 embeddings a small limit returns at once with
    exactly that many (the grid stops early)."""
    import time
    n, s, d = gpm.gen_rmat(14, 16, seed=9)
    lab = np.zeros(n, np.int32)
    g = gpm.Graph.from_edges(n, s, d, labels=lab)
    q = gpm.Query(4, np.array([0, 1, 2, 3], np.int32), np.array([1, 2, 3, 0], np.int32), np.zeros(4, np.int32))
    t = time.perf_counter()
    assert g.match(q, limit=1000) == 1000
    rows = g.match_list(q, 1000)
    assert time.perf_counter() - t < 30
    off, idx = g.csr()
    assert len(set(map(tuple, rows.tolist()))) == 1000
    for r in rows[:50]:
        nb = [set(idx[off[v]:off[v + 1]].tolist()) for v in r]
        assert len(set(r.tolist())) == 4
        assert r[1] in nb[0] and r[2] in nb[1] and r[3] in nb[2] and r[0] in nb[3]
