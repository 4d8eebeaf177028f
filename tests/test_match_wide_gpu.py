"""Query graphs of 16 to 64 vertices (sub_ceci's limit,
sub_ceci/configuration/config.h:12): counts equal the reference's own sub_ceci
on seeded random labelled graphs (tests/golden/ceci_wide.npz, written by
make_ceci_wide_golden.py), in single calls, in batches that mix 16-vertex
queries with wider ones (all of them run by the 64-wide kernel), in a
disjoint union with member ids, and as listed embeddings."""
import os

import numpy as np
import pytest

import gpm

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def wide_cases():
    z = np.load(os.path.join(GOLD, "ceci_wide.npz"))
    gs = np.concatenate([[0], np.cumsum(z["ge_len"])])
    ls = np.concatenate([[0], np.cumsum(z["gn"])])
    graphs = [(int(z["gn"][i]), z["ge"][gs[i]:gs[i + 1]], z["gl"][ls[i]:ls[i + 1]]) for i in range(len(z["gn"]))]
    qs = np.concatenate([[0], np.cumsum(z["q_e_len"])])
    qls = np.concatenate([[0], np.cumsum(z["q_n"])])
    queries = [(int(z["q_graph"][i]), int(z["q_n"][i]), z["q_e"][qs[i]:qs[i + 1]], z["q_lab"][qls[i]:qls[i + 1]],
                int(z["expected"][i])) for i in range(len(z["q_n"]))]
    return graphs, queries


def make_query(k, qe, ql):
    return gpm.Query(k, qe[:, 0], qe[:, 1], ql)


def test_wide_queries_equal_subceci():
    graphs, queries = wide_cases()
    assert max(q[1] for q in queries) == 64 and min(q[1] for q in queries) == 16
    gg = [gpm.Graph.from_edges(n, e[:, 0], e[:, 1], labels=lab) for n, e, lab in graphs]
    for i, (gi, k, qe, ql, want) in enumerate(queries):
        assert gg[gi].match(make_query(k, qe, ql)) == want, (i, gi, k)


def test_batches_mixing_narrow_and_wide_queries():
    graphs, queries = wide_cases()
    for gi, (n, e, lab) in enumerate(graphs):
        g = gpm.Graph.from_edges(n, e[:, 0], e[:, 1], labels=lab)
        mine = [q for q in queries if q[0] == gi]
        want = [q[4] for q in mine]
        b = gpm.MatchBatch(g, [make_query(k, qe, ql) for _, k, qe, ql, _ in mine])
        assert b.run(use_graph=False)[:, 0].tolist() == want
        assert b.run(use_graph=True)[:, 0].tolist() == want
        b.autotune()
        assert b.run(use_graph=True)[:, 0].tolist() == want
        # the 16-vertex queries alone take the narrow kernel
        narrow = [q for q in mine if q[1] <= 16]
        bn = gpm.MatchBatch(g, [make_query(k, qe, ql) for _, k, qe, ql, _ in narrow])
        assert bn.run(use_graph=True)[:, 0].tolist() == [q[4] for q in narrow]


def test_wide_queries_on_a_union_with_members():
    graphs, queries = wide_cases()
    base = np.cumsum([0] + [g[0] for g in graphs])
    src = np.concatenate([e[:, 0] + base[i] for i, (_, e, _) in enumerate(graphs)]).astype(np.int32)
    dst = np.concatenate([e[:, 1] + base[i] for i, (_, e, _) in enumerate(graphs)]).astype(np.int32)
    lab = np.concatenate([g[2] for g in graphs]).astype(np.int32)
    member = np.repeat(np.arange(len(graphs), dtype=np.int32), [g[0] for g in graphs])
    u = gpm.Graph.from_edges(int(base[-1]), src, dst, labels=lab)
    gg = [gpm.Graph.from_edges(n, e[:, 0], e[:, 1], labels=l) for n, e, l in graphs]
    qq = [make_query(k, qe, ql) for _, k, qe, ql, _ in queries]
    out = gpm.MatchBatch(u, qq, member=member, nmembers=len(graphs)).run(use_graph=True)
    for i, (gi, _, _, _, want) in enumerate(queries):
        assert int(out[i, gi]) == want, i
        for m in range(len(graphs)):
            assert int(out[i, m]) == gg[m].match(qq[i]), (i, m)


def test_wide_listing_and_limit():
    graphs, queries = wide_cases()
    gg = [gpm.Graph.from_edges(n, e[:, 0], e[:, 1], labels=lab) for n, e, lab in graphs]
    adj = []
    for n, e, _ in graphs:
        s = [set() for _ in range(n)]
        for a, b in e:
            s[int(a)].add(int(b))
            s[int(b)].add(int(a))
        adj.append(s)
    listed = 0
    for gi, k, qe, ql, want in queries:
        if k <= 16 or want > 5000:
            continue
        q = make_query(k, qe, ql)
        rows = gg[gi].match_list(q, want + 3)
        assert len(rows) == want and len({tuple(r) for r in rows.tolist()}) == want
        lab = graphs[gi][2]
        for r in rows:
            assert len(set(r.tolist())) == k and (lab[r] == ql).all()
            assert all(int(r[b]) in adj[gi][int(r[a])] for a, b in qe)
        lim = max(1, want // 3)
        assert gg[gi].match(q, limit=lim) == lim
        listed += 1
    assert listed >= 20
    # a large wide enumeration stops at its limit
    big = max(queries, key=lambda q: q[4])
    assert big[1] > 16 and big[4] > 10**7
    assert gg[big[0]].match(make_query(*big[1:4]), limit=1000) == 1000
