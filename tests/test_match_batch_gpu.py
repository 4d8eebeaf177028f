"""Batched labelled matching: many queries (and many member graphs of one
disjoint union) counted in one persistent launch, replayed from a CUDA graph,
with the task split chosen by the autotuner -- every count must equal a
single gpm_match call of the same query on the same graph, and the oracle."""
import numpy as np
import pytest

import gpm
import _oracle as orc
import workloads as W

pytestmark = pytest.mark.gpu


def queries_of(off, idx, lab, seed):
    qs = W.walk_queries(off, idx, lab, seed=seed)
    out = [gpm.Query(k, e[:, 0], e[:, 1], ql) for k, e, ql in qs.values()]
    # a one-vertex and a two-vertex query (counted without the DFS kernel)
    out.append(gpm.Query(1, [], [], [int(lab[0])]))
    out.append(gpm.Query(2, [0], [1], [int(lab[0]), int(lab[1])]))
    return out


def test_batch_equals_single_queries():
    n, s, d = gpm.gen_rmat(14, 8, seed=21)
    lab = gpm.gen_zipf_labels(n, 4, 1.2, seed=21)
    g = gpm.Graph.from_edges(n, s, d, labels=lab)
    off, idx = g.csr()
    qs = queries_of(off, idx, lab, seed=4)
    want = np.array([g.match(q) for q in qs], np.uint64)
    b = gpm.MatchBatch(g, qs)
    assert b.run(use_graph=False)[:, 0].tolist() == want.tolist()
    assert b.run(use_graph=True)[:, 0].tolist() == want.tolist()
    assert b.run(use_graph=True)[:, 0].tolist() == want.tolist()  # replay
    span = b.autotune()
    assert span in (0, 16384, 2048, 256)
    assert b.run(use_graph=True)[:, 0].tolist() == want.tolist()
    ntasks, _ = b.info()
    assert ntasks > 0


def test_batch_every_split_span_keeps_counts():
    # hub-heavy graph: tasks of 4+ vertex queries split into many chunks
    n, s, d = gpm.gen_chung_lu(6000, 2.1, 24.0, seed=9)
    lab = gpm.gen_zipf_labels(n, 3, 1.2, seed=9)
    g = gpm.Graph.from_edges(n, s, d, labels=lab)
    off, idx = g.csr()
    qs = queries_of(off, idx, lab, seed=5)[:4]
    want = [g.match(q) for q in qs]
    b = gpm.MatchBatch(g, qs)
    base_tasks, _ = b.info()
    b.autotune()  # builds and runs the task list of every candidate span
    got = b.run(use_graph=True)[:, 0].tolist()
    assert got == want
    assert b.info()[0] >= base_tasks


def test_batch_members_of_a_union():
    """Six random labelled graphs as one disjoint union with member ids:
    per-member counts equal each graph matched on its own and the oracle."""
    rng = np.random.default_rng(33)
    parts, labels, member, base = [], [], [], 0
    graphs = []
    for m in range(6):
        gn = int(rng.integers(50, 400))
        e = rng.integers(0, gn, size=(gn * 4, 2)).astype(np.int32)
        gl = rng.integers(0, 3, size=gn).astype(np.int32)
        graphs.append((gn, e, gl))
        parts.append(e + base)
        labels.append(gl)
        member.append(np.full(gn, m, np.int32))
        base += gn
    e = np.concatenate(parts)
    lab = np.concatenate(labels)
    mem = np.concatenate(member)
    g = gpm.Graph.from_edges(base, e[:, 0], e[:, 1], labels=lab)
    shapes = list(W.SHAPES.values())
    qs = []
    for k, edges in shapes:
        ee = np.array(edges, np.int32)
        qs.append((k, ee, rng.integers(0, 3, size=k).astype(np.int32)))
    b = gpm.MatchBatch(g, [gpm.Query(k, ee[:, 0], ee[:, 1], ql) for k, ee, ql in qs], member=mem, nmembers=6)
    got = b.run(use_graph=True)
    assert got.shape == (len(qs), 6)
    for m, (gn, ge, gl) in enumerate(graphs):
        gm = gpm.Graph.from_edges(gn, ge[:, 0], ge[:, 1], labels=gl)
        off, idx = orc.build_csr(gn, ge[:, 0], ge[:, 1])
        for qi, (k, ee, ql) in enumerate(qs):
            single = gm.match(gpm.Query(k, ee[:, 0], ee[:, 1], ql))
            qo, qx = orc.build_csr(k, ee[:, 0], ee[:, 1])
            assert got[qi, m] == single == orc.match(off, idx, gl, qo, qx, ql), (qi, m)


def test_batch_rejects_bad_member_ids():
    n, s, d = gpm.gen_rmat(8, 4, seed=2)
    lab = gpm.gen_zipf_labels(n, 2, 1.2, seed=2)
    g = gpm.Graph.from_edges(n, s, d, labels=lab)
    q = gpm.Query(3, [0, 1, 2], [1, 2, 0], [0, 0, 1])
    with pytest.raises(gpm.GpmError):
        gpm.MatchBatch(g, [q], member=np.full(n, 5, np.int32), nmembers=2)
