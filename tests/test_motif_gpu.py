"""3/4-vertex motifs and the named patterns P1..P8 / Motif4 on the GPU vs the oracle."""
import numpy as np
import pytest

import gpm
import _oracle as orc

pytestmark = pytest.mark.gpu


def sym(n, s, d):
    return orc.build_csr(n, s, d)


@pytest.mark.parametrize("seed", range(10))
def test_small_random_vs_bruteforce(seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(5, 60))
    e = rng.integers(0, n, size=(int(n * rng.uniform(1, 6)), 2)).astype(np.int32)
    off, idx = sym(n, e[:, 0], e[:, 1])
    bf = orc.bruteforce(off, idx)
    g = gpm.Graph.from_edges(n, e[:, 0], e[:, 1])
    assert g.motif(3).tolist() == bf[:2].tolist()
    assert g.motif(4).tolist() == bf[2:].tolist()


@pytest.mark.parametrize("gamma,mean,seed", [(2.1, 8.0, 1), (2.5, 16.0, 2), (2.8, 32.0, 3)])
def test_chung_lu_vs_g2miner_restatement(gamma, mean, seed):
    n, s, d = gpm.gen_chung_lu(3000, gamma, mean, seed=seed)
    off, idx = sym(n, s, d)
    doff, didx = orc.orient(off, idx)
    g = gpm.Graph.from_edges(n, s, d)
    assert g.motif(4).tolist() == orc.motif4(off, idx).tolist()
    assert g.motif(3).tolist() == orc.motif3(off, idx, orc.tc(doff, didx)).tolist()


def test_rmat_vs_g2miner_restatement():
    n, s, d = gpm.gen_rmat(12, 16, seed=7)
    off, idx = sym(n, s, d)
    g = gpm.Graph.rmat(12, 16, seed=7)
    assert g.motif(4).tolist() == orc.motif4(off, idx).tolist()


def test_simple_mtx_fixture():
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_small.npz"))
    e = z["simple_mtx"]
    g = gpm.Graph.from_edges(4, e[:, 0], e[:, 1])
    assert g.motif(4).tolist() == [0, 1, 0, 0, 0, 0]
    assert g.motif(3).tolist() == [2, 0]


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("family", [gpm.G2MINER, gpm.PATTERN_SOLVER])
def test_named_patterns(seed, family):
    rng = np.random.default_rng(200 + seed)
    n = int(rng.integers(20, 70))
    e = rng.integers(0, n, size=(int(n * rng.uniform(2, 5)), 2)).astype(np.int32)
    off, idx = sym(n, e[:, 0], e[:, 1])
    g = gpm.Graph.from_edges(n, e[:, 0], e[:, 1])
    for p in range(1, 9):
        want = orc.pattern_g2miner(off, idx, p)
        res, cnt = g.pattern(f"P{p}", family)
        assert res == want, (p, res, want)
        if family == gpm.PATTERN_SOLVER:
            assert res == orc.pattern_solver(off, idx, p)[0]
    res, cnt = g.pattern("Motif4", family)
    m4 = orc.motif4(off, idx)
    assert cnt.tolist() == m4.tolist()
    assert res == (int(m4[0]) if family == gpm.G2MINER else (int(m4[1]) - int(m4[2])) % 2**64)


def test_patterns_on_rmat():
    n, s, d = gpm.gen_rmat(10, 8, seed=3)
    off, idx = sym(n, s, d)
    g = gpm.Graph.from_edges(n, s, d)
    for p in (2, 3, 5, 6, 7, 8):
        assert g.pattern(f"P{p}")[0] == orc.pattern_g2miner(off, idx, p, 0), p


def test_unknown_pattern():
    g = gpm.Graph.from_edges(3, [0, 1], [1, 2])
    with pytest.raises(gpm.GpmError) as e:
        g.pattern("P9")
    assert e.value.status == 1


def test_hub_lists_longer_than_the_sort_buffer():
    """A 3999-leaf hub: its relabelled list (3999 ids) is beyond the
    1024-key sort buffer of the relabel and takes the segmented-sort
    fallback; the motif counts stay exact."""
    n = 4000
    rng = np.random.default_rng(11)
    other = rng.integers(1, n, size=(30000, 2))
    s = np.concatenate([np.zeros(n - 1, np.int64), other[:, 0]]).astype(np.int32)
    d = np.concatenate([np.arange(1, n), other[:, 1]]).astype(np.int32)
    off, idx = sym(n, s, d)
    assert np.diff(off).max() > 1024
    g = gpm.Graph.from_edges(n, s, d)
    assert g.motif(4).tolist() == orc.motif4(off, idx).tolist()


def c4_of(m4):
    """Non-induced 4-cycles from the induced counts: cycle + diamond + 3 x clique."""
    return (int(m4[3]) + int(m4[4]) + 3 * int(m4[5])) % 2**64


@pytest.mark.parametrize("graph", ["chung_lu", "rmat"])
def test_every_hub_task_in_key_range_chunks(graph, monkeypatch):
    """GPM_C4_BIG_MIN=0 sends every 4-cycle task above the warp bound to the
    chunked shared-memory kernel (lane groups of 1..32 lanes per neighbour)."""
    monkeypatch.setenv("GPM_C4_BIG_MIN", "0")
    if graph == "chung_lu":
        n, s, d = gpm.gen_chung_lu(3000, 2.2, 24.0, seed=9)
    else:
        n, s, d = gpm.gen_rmat(12, 16, seed=5)
    off, idx = sym(n, s, d)
    g = gpm.Graph.from_edges(n, s, d)
    assert g.motif(4).tolist() == orc.motif4(off, idx).tolist()


def test_giant_tasks_many_chunks_and_wide_counters():
    """Two non-adjacent hubs on 250,000 vertices: the 70,000-neighbour hub's
    task needs 32-bit counters and five key chunks, the 20,000-neighbour hub
    16-bit counters and three; medium hubs among their neighbours take the
    whole-warp walk.  Checked against the closed-form count, alone and as a
    member of a batch (nonzero base rank)."""
    off, idx = orc.two_hub_graph(250000, 1000000, 70000, 20000, [300, 450, 800, 1500, 2500], seed=5)
    want = orc.c4_two_hubs(off, idx, 0, 1)
    g = gpm.Graph.from_csr(off, idx)
    assert c4_of(g.motif(4)) == want
    n = len(off) - 1
    src = np.repeat(np.arange(n), np.diff(off)).astype(np.int32)
    sn, ss, sd = gpm.gen_chung_lu(5000, 2.3, 12.0, seed=3)
    b = gpm.Batch.from_edges([(sn, ss, sd), (n, src, idx), (sn, ss, sd)])
    r = b.motif(use_graph=False)
    assert c4_of(r[1, 2:]) == want
    assert r[0].tolist() == r[2].tolist()
    soff, sidx = sym(sn, ss, sd)
    assert r[0, 2:].tolist() == orc.motif4(soff, sidx).tolist()


def test_cached_pipelines_repeat_exactly():
    """The first call of each motif size keeps its pipeline with the graph;
    later calls, interleaved with the other size, only relaunch it and give
    the same counts."""
    n, s, d = gpm.gen_chung_lu(5000, 2.2, 20.0, seed=21)
    off, idx = sym(n, s, d)
    want4 = orc.motif4(off, idx).tolist()
    want3 = orc.motif3(off, idx, orc.tc(*orc.orient(off, idx))).tolist()
    g = gpm.Graph.from_edges(n, s, d)
    for _ in range(3):
        assert g.motif(4).tolist() == want4
        assert g.motif(3).tolist() == want3
