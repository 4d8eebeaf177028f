"""Triangle counting on the GPU through the C ABI, bit-exact against the oracle."""
import numpy as np
import pytest

import gpm
import _oracle as orc

pytestmark = pytest.mark.gpu
VARIANTS = [gpm.TC_BSEARCH, gpm.TC_MERGE, gpm.TC_HASH, gpm.TC_BITMAP]


def tc_all_variants(g):
    import torch
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    res = []
    for v in VARIANTS:
        g.tc_async(v, torch.cuda.current_stream().cuda_stream, out.data_ptr())
        torch.cuda.synchronize()
        res.append(int(out.item()))
    return res


def oracle_graph(n, src, dst):
    off, idx = orc.build_csr(n, src, dst)
    doff, didx = orc.orient(off, idx)
    return off, idx, doff, didx


def test_device_csr_matches_oracle_build():
    n, s, d = gpm.gen_er(3000, 20000, seed=11)
    off, idx, doff, didx = oracle_graph(n, s, d)
    g = gpm.Graph.from_edges(n, s, d)
    o2, i2 = g.csr()
    assert (o2 == off).all() and (i2 == idx).all()
    assert g.info().max_degree == int(np.diff(off).max())
    g.orient()
    o3, i3 = g.csr()
    assert (o3 == doff).all() and (i3 == didx).all()


def test_device_generator_matches_host_generator():
    n, s, d = gpm.gen_rmat(12, 8, seed=3)
    off, idx = orc.build_csr(n, s, d)
    g = gpm.Graph.rmat(12, 8, seed=3)
    o2, i2 = g.csr()
    assert (o2 == off).all() and (i2 == idx).all()


def test_er_config():
    # G(n=16384, m=131072 draws), self-loops/duplicates removed, degree-oriented.
    n, s, d = gpm.gen_er(16384, 131072, seed=1)
    off, idx, doff, didx = oracle_graph(n, s, d)
    want = orc.tc(doff, didx)
    assert want == orc.tc_merge(doff, didx)
    g = gpm.Graph.from_edges(n, s, d).orient()
    assert g.tc(gpm.V_CENTRIC) == want
    assert g.tc(gpm.E_CENTRIC) == want
    assert tc_all_variants(g) == [want] * len(VARIANTS)


@pytest.mark.parametrize("scale,ef,seed", [(10, 16, 1), (14, 16, 2), (16, 16, 3), (17, 8, 4)])
def test_rmat_against_oracle(scale, ef, seed):
    n, s, d = gpm.gen_rmat(scale, ef, seed=seed)
    off, idx, doff, didx = oracle_graph(n, s, d)
    want = orc.tc(doff, didx)
    g = gpm.Graph.rmat(scale, ef, seed=seed).orient()
    assert tc_all_variants(g) == [want] * len(VARIANTS)
    g2 = gpm.Graph.rmat(scale, ef, seed=seed).orient(relabel=True)
    assert tc_all_variants(g2) == [want] * len(VARIANTS)


def test_hub_chunking_beyond_one_table():
    # a vertex with out-degree > 1024 in the DAG forces the chunked CTA path
    n = 3000
    hub_src, hub_dst = [], []
    rng = np.random.default_rng(5)
    # 1500 vertices of degree ~40 pointing among themselves + clique-ish core
    e = rng.integers(1000, 2600, size=(40000, 2))
    core = rng.integers(2600, 3000, size=(60000, 2))
    s = np.concatenate([e[:, 0], core[:, 0]]).astype(np.int32)
    d = np.concatenate([e[:, 1], core[:, 1]]).astype(np.int32)
    off, idx, doff, didx = oracle_graph(n, s, d)
    assert np.diff(doff).max() > 100
    want = orc.tc(doff, didx)
    g = gpm.Graph.from_edges(n, s, d).orient()
    assert tc_all_variants(g) == [want] * len(VARIANTS)


def test_unoriented_sum_semantics():
    # TCSolver sums |N(u) & N(v)| over stored edges; on a symmetric graph = 6T
    n, s, d = gpm.gen_er(500, 3000, seed=9)
    off, idx, doff, didx = oracle_graph(n, s, d)
    g = gpm.Graph.from_edges(n, s, d)
    assert tc_all_variants(g) == [6 * orc.tc(doff, didx)] * len(VARIANTS)


@pytest.mark.parametrize("case", ["empty", "single_edge", "triangle", "k5", "star"])
def test_edge_cases(case):
    if case == "empty":
        n, s, d = 4, [], []
    elif case == "single_edge":
        n, s, d = 2, [0], [1]
    elif case == "triangle":
        n, s, d = 3, [0, 1, 2], [1, 2, 0]
    elif case == "k5":
        pairs = [(a, b) for a in range(5) for b in range(a + 1, 5)]
        n, s, d = 5, [p[0] for p in pairs], [p[1] for p in pairs]
    else:
        n, s, d = 50, [0] * 49, list(range(1, 50))
    s, d = np.array(s, np.int32), np.array(d, np.int32)
    want = {"empty": 0, "single_edge": 0, "triangle": 1, "k5": 10, "star": 0}[case]
    g = gpm.Graph.from_edges(n, s, d).orient()
    assert tc_all_variants(g) == [want] * len(VARIANTS)
    assert g.tc(gpm.V_CENTRIC) == want


def test_host_csr_end_to_end():
    n, s, d = gpm.gen_rmat(15, 16, seed=8)
    off, idx, doff, didx = oracle_graph(n, s, d)
    want = orc.tc(doff, didx)
    for v in VARIANTS:
        assert gpm.tc_host_csr(off, idx, v) == want


def core_words(kmin, kmax):
    """(and_words, clear_words) of a core owner's bitmap based at kmin
    rounded down to 128 (multiples of four words)."""
    base = kmin & ~127
    return (((kmax - base) >> 5) + 4) & ~3, (((kmax - base + 1) >> 5) + 4) & ~3


def plan_numpy(off, idx, core=16384, core_min=128, dense_pct=100, cta_words=6144):
    """The fixed plan's work restated in numpy: rank by (degree, id), DAG
    edges upward, owner = endpoint with the longer out-list (ties to the
    source), segment = the partner's list clipped to [min, max] of the
    owner's list (owners with fewer than 2 keys have none).  Dense core:
    ranks from core_base = (n - core) rounded down to 128; a vertex with at
    least core_min keys there has a row (no rows at all when a row would be
    wider than cta_words words); a segment is dense when its owner's keys all
    lie in the core, its partner has a row and its keys are at least
    dense_pct % of the owner's bitmap words.  Returns (segments,
    keys of the non-dense segments, owner keys, owner tasks, dense segments,
    their words)."""
    n = len(off) - 1
    deg = np.diff(off)
    order = np.lexsort((np.arange(n), deg))
    rank = np.empty(n, np.int64)
    rank[order] = np.arange(n)
    rs, rd = rank[np.repeat(np.arange(n), deg)], rank[idx]
    up = rd > rs
    us, vs = rs[up], rd[up]
    o = np.lexsort((vs, us))
    us, vs = us[o], vs[o]
    dp = np.bincount(us, minlength=n)
    roff = np.zeros(n + 1, np.int64)
    roff[1:] = np.cumsum(dp)
    du, dv = dp[us], dp[vs]
    own_u = dv <= du
    owner, partner = np.where(own_u, us, vs), np.where(own_u, vs, us)
    kmin = vs[np.minimum(roff[:-1], len(vs) - 1)]
    kmax = vs[np.maximum(roff[1:] - 1, 0)]
    key = us * (n + 1) + vs
    a = np.searchsorted(key, partner * (n + 1) + kmin[owner], "left")
    b = np.searchsorted(key, partner * (n + 1) + kmax[owner], "right")
    clip = np.where(np.maximum(du, dv) >= 2, np.maximum(b - a, 0), 0)
    seg = clip > 0
    tasks = np.unique(owner[seg])
    dense = np.zeros_like(seg)
    aw = np.zeros(len(seg), np.int64)
    cb = max(0, n - core) & ~127
    row_words = ((n - cb + 127) >> 7) << 2
    rowed = np.bincount(us[vs >= cb], minlength=n) >= max(1, core_min)
    if core > 0 and n > 0 and row_words <= cta_words and rowed.any():
        ko, kx = kmin[owner].astype(np.int64), kmax[owner].astype(np.int64)
        aw, _ = core_words(ko, kx)
        dense = seg & (ko >= cb) & rowed[partner] & (100 * clip >= dense_pct * aw)
    return (int(seg.sum()), int(clip[~dense].sum()), int(dp[tasks].sum()), len(tasks), int(dense.sum()),
            int(aw[dense].sum()))


@pytest.mark.parametrize("kind", ["rmat", "er"])
def test_plan_segments_match_numpy(kind):
    """The plan streams exactly the clipped segments: their number, their
    keys, the owner keys and the owner tasks equal the numpy restatement."""
    if kind == "rmat":
        n, s, d = gpm.gen_rmat(13, 16, seed=7)
    else:
        n, s, d = gpm.gen_er(20000, 300000, seed=7)
    off, idx = orc.build_csr(n, s, d)
    g = gpm.Graph.from_csr(off, idx).orient()
    assert g.plan_stats() == plan_numpy(off, idx)


@pytest.mark.parametrize("case", [("rmat", 4096, 2, 0), ("rmat", 1 << 20, 1, 0), ("rmat", 8192, 16, 50),
                                  ("er", 1 << 20, 1, 0), ("clique", 16384, 128, 100)])
def test_dense_core_rows(case, monkeypatch):
    """Dense core segments (core bitmap rows ANDed with the owner's bitmap)
    count the same triangles: the thresholds lowered so that most segments of
    core owners are dense, on R-MAT, Erdos-Renyi and a graph with a
    1200-clique; the plan's dense segments and words equal the numpy
    restatement."""
    kind, core, core_min, pct = case
    monkeypatch.setenv("GPM_TC_CORE", str(core))
    monkeypatch.setenv("GPM_TC_CORE_MIN", str(core_min))
    monkeypatch.setenv("GPM_TC_DENSE_PCT", str(pct))
    if kind == "rmat":
        n, s, d = gpm.gen_rmat(14, 16, seed=5)
    elif kind == "er":
        n, s, d = gpm.gen_er(6000, 400000, seed=5)
    else:
        n = 5000
        iu, ju = np.triu_indices(1200, 1)
        fr = np.random.default_rng(4).integers(0, n, size=(20000, 2))
        s = np.concatenate([iu, fr[:, 0]]).astype(np.int32)
        d = np.concatenate([ju, fr[:, 1]]).astype(np.int32)
    off, idx, doff, didx = oracle_graph(n, s, d)
    want = orc.tc(doff, didx)
    g = gpm.Graph.from_edges(n, s, d).orient()
    stats = g.plan_stats()
    assert stats == plan_numpy(off, idx, core, core_min, pct)
    assert stats[4] > 0
    assert tc_all_variants(g) == [want] * len(VARIANTS)
    assert gpm.tc_host_csr(off, idx, gpm.TC_AUTO) == want


def test_lists_longer_than_the_sort_buffer():
    """Relabelled lists longer than the 1024-key sort buffer take the
    segmented-sort fallback: a 1200-clique (DAG out-lists up to 1199) with a
    sparse random fringe, through the oriented graph and the host-CSR path."""
    n = 5000
    iu, ju = np.triu_indices(1200, 1)
    fr = np.random.default_rng(3).integers(0, n, size=(20000, 2))
    s = np.concatenate([iu, fr[:, 0]]).astype(np.int32)
    d = np.concatenate([ju, fr[:, 1]]).astype(np.int32)
    off, idx, doff, didx = oracle_graph(n, s, d)
    assert np.diff(doff).max() > 1024
    want = orc.tc(doff, didx)
    g = gpm.Graph.from_edges(n, s, d).orient()
    assert tc_all_variants(g) == [want] * len(VARIANTS)
    assert gpm.tc_host_csr(off, idx, gpm.TC_AUTO) == want
    assert g.plan_stats() == plan_numpy(off, idx)
