"""Batched motif counting: many graphs in one union, one launch per stage,
replayed from a captured CUDA graph, autotuned thresholds -- per-member counts
must equal the single-graph path and the oracle."""
import numpy as np
import pytest

import gpm
import _oracle as orc

pytestmark = pytest.mark.gpu


def members(seed, count, nmax=4000):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(30), np.log(nmax))))
        gam = rng.uniform(2.1, 2.8)
        md = rng.uniform(4, 24)
        _, s, d = gpm.gen_chung_lu(n, gam, md, seed=seed * 1000 + i)
        out.append((n, s, d))
    return out


def test_batch_matches_members_and_oracle():
    mem = members(1, 24)
    b = gpm.Batch.from_edges(mem)
    assert b.info()[0] == 24
    res_direct = b.motif(use_graph=False)
    res_graph = b.motif(use_graph=True)
    res_graph2 = b.motif(use_graph=True)
    assert (res_direct == res_graph).all() and (res_graph == res_graph2).all()
    for i, (n, s, d) in enumerate(mem):
        off, idx = orc.build_csr(n, s, d)
        boff, bidx = b.member_csr(i)
        assert (boff == off).all() and (bidx == idx).all()
        g = gpm.Graph.from_edges(n, s, d)
        assert res_graph[i, :2].tolist() == g.motif(3).tolist()
        assert res_graph[i, 2:].tolist() == g.motif(4).tolist()
        if i < 8:
            assert res_graph[i, 2:].tolist() == orc.motif4(off, idx).tolist()


def test_autotune_keeps_counts():
    b = gpm.Batch.from_edges(members(2, 12, 20000))
    before = b.motif(use_graph=True)
    tuned = b.autotune()
    assert len(tuned) == 3 and all(t > 0 for t in tuned)
    after = b.motif(use_graph=True)
    assert (before == after).all()


def test_device_generated_batch():
    n = np.array([1000, 3000, 500, 20000], np.int64)
    gam = np.array([2.1, 2.5, 2.8, 2.3])
    md = np.array([8.0, 32.0, 16.0, 64.0])
    b = gpm.Batch.chung_lu(n, gam, md, seed=7)
    res = b.motif()
    for i in range(len(n)):
        off, idx = b.member_csr(i)
        g = gpm.Graph.from_csr(off, idx)
        assert res[i, 2:].tolist() == g.motif(4).tolist()
        if n[i] <= 3000:
            assert res[i, 2:].tolist() == orc.motif4(off, idx).tolist()


def test_empty_and_tiny_members():
    mem = [(5, np.array([], np.int32), np.array([], np.int32)), (3, np.array([0, 1, 2]), np.array([1, 2, 0])),
           (4, np.array([0, 0, 0]), np.array([1, 2, 3]))]
    res = gpm.Batch.from_edges(mem).motif()
    assert res[0].tolist() == [0] * 8
    assert res[1].tolist() == [0, 1, 0, 0, 0, 0, 0, 0]
    assert res[2].tolist() == [3, 0, 1, 0, 0, 0, 0, 0]
