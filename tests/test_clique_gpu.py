"""k-clique counting (CFSolver semantics) on the GPU vs the CPU oracle."""
import itertools

import numpy as np
import pytest

import gpm
import _oracle as orc

pytestmark = pytest.mark.gpu


def dag(n, s, d):
    off, idx = orc.build_csr(n, s, d)
    return off, idx, *orc.orient(off, idx)


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("k", [3, 4, 5, 6])
def test_random_small(seed, k):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(10, 80))
    e = rng.integers(0, n, size=(int(n * rng.uniform(2, 8)), 2)).astype(np.int32)
    off, idx, doff, didx = dag(n, e[:, 0], e[:, 1])
    g = gpm.Graph.from_edges(n, e[:, 0], e[:, 1]).orient()
    assert g.clique(k) == orc.clique(doff, didx, k)


@pytest.mark.parametrize("scale,k", [(12, 4), (14, 4), (14, 5), (16, 4), (16, 5)])
def test_rmat_against_oracle(scale, k):
    n, s, d = gpm.gen_rmat(scale, 16, seed=scale)
    off, idx, doff, didx = dag(n, s, d)
    g = gpm.Graph.rmat(scale, 16, seed=scale).orient()
    assert g.clique(k) == orc.clique(doff, didx, k)


def test_k3_equals_triangles():
    g = gpm.Graph.rmat(17, 16, seed=3).orient()
    assert g.clique(3) == g.tc(gpm.V_CENTRIC)


def test_dense_hubs_cta_and_slab_paths():
    # out-lists of several hundred force CTA tasks; > ~560 spills rows to the slab
    rng = np.random.default_rng(11)
    n = 1000
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(len(iu)) < 0.9  # near-complete: DAG out-lists up to ~n
    a, b = iu[keep].astype(np.int32), ju[keep].astype(np.int32)
    off, idx, doff, didx = dag(n, a, b)
    assert np.diff(doff).max() > 560
    g = gpm.Graph.from_edges(n, a, b).orient()
    assert g.clique(3) == orc.tc(doff, didx)
    n2 = 300
    a2 = rng.integers(0, n2, size=25000)
    b2 = rng.integers(0, n2, size=25000)
    off2, idx2, doff2, didx2 = dag(n2, a2, b2)
    g2 = gpm.Graph.from_edges(n2, a2, b2).orient()
    assert g2.clique(4) == orc.clique(doff2, didx2, 4)


def test_unoriented_graph_uses_reference_sum():
    # CFSolver sums over stored edges; on a symmetric graph every k-clique is
    # counted once per ordering of its vertices: k! times.
    rng = np.random.default_rng(4)
    n = 40
    e = rng.integers(0, n, size=(300, 2)).astype(np.int32)
    off, idx, doff, didx = dag(n, e[:, 0], e[:, 1])
    g = gpm.Graph.from_edges(n, e[:, 0], e[:, 1])
    assert g.clique(4) == 24 * orc.clique(doff, didx, 4)
    assert g.clique(3) == 6 * orc.clique(doff, didx, 3)


@pytest.mark.parametrize("k", [3, 4, 5])
def test_complete_graphs(k):
    from math import comb
    n = 40
    pairs = np.array(list(itertools.combinations(range(n), 2)), np.int32)
    g = gpm.Graph.from_edges(n, pairs[:, 0], pairs[:, 1]).orient()
    assert g.clique(k) == comb(n, k)


def test_bad_k():
    g = gpm.Graph.from_edges(3, [0], [1]).orient()
    with pytest.raises(gpm.GpmError):
        g.clique(2)
    with pytest.raises(gpm.GpmError):
        g.clique(9)


def test_cached_schedules_repeat_exactly():
    """Each k's schedule is built on its first call and kept with the graph;
    interleaved repeated calls (and the edge-centric kernel between them)
    give the oracle's counts every time."""
    n, s, d = gpm.gen_rmat(13, 16, seed=23)
    off, idx, doff, didx = dag(n, s, d)
    want = {k: orc.clique(doff, didx, k) for k in (3, 4, 5)}
    g = gpm.Graph.rmat(13, 16, seed=23).orient()
    for _ in range(3):
        for k in (5, 3, 4):
            assert g.clique(k) == want[k], k
        assert g.clique(4, edge_centric=True) == want[4]
