"""The CPU oracle against the reference's own known answers (no GPU).

Pins: sub_ceci's 200 HPRD known-answer tests, the counts the reference's
sub_ceci (built from its sources) printed for seeded random labelled graphs,
and an independent brute-force census for the unlabelled restatements.
"""
import os

import numpy as np
import pytest

import _oracle as orc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def kat():
    z = np.load(os.path.join(GOLD, "hprd_kat.npz"))
    qoffs, qidxs, qlabs = [], [], []
    po = pi = pl = 0
    for m in z["qn"]:
        qo = z["qoff"][po: po + m + 1]
        po += m + 1
        qi = z["qidx"][pi: pi + qo[-1]]
        pi += qo[-1]
        ql = z["qlab"][pl: pl + m]
        pl += m
        qoffs.append(qo)
        qidxs.append(qi)
        qlabs.append(ql)
    return z, qoffs, qidxs, qlabs


def test_hprd_known_answers():
    z, qo, qi, ql = kat()
    got = [orc.match(z["off"], z["idx"], z["labels"], qo[i], qi[i], ql[i]) for i in range(200)]
    assert got == [int(x) for x in z["expected"]]


def ceci_random_cases():
    z = np.load(os.path.join(GOLD, "ceci_random.npz"))
    from make_golden import SHAPES  # noqa: F401  (shapes table lives with the generator)
    return z


def test_reference_subceci_on_random_graphs():
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import SHAPES
    z = np.load(os.path.join(GOLD, "ceci_random.npz"))
    starts = np.concatenate([[0], np.cumsum(z["ge_len"])])
    lstarts = np.concatenate([[0], np.cumsum(z["gn"])])
    shapes = list(SHAPES.values())
    for row in z["rows"]:
        gi, si = int(row[0]), int(row[1])
        n = int(z["gn"][gi])
        e = z["ge"][starts[gi]: starts[gi + 1]]
        lab = z["gl"][lstarts[gi]: lstarts[gi + 1]]
        off, idx = orc.build_csr(n, e[:, 0], e[:, 1])
        sn, sedges = shapes[si]
        se = np.array(sedges, np.int32)
        qo, qi = orc.build_csr(sn, se[:, 0], se[:, 1])
        ql = np.array(row[2: 2 + sn], np.int32)
        assert orc.match(off, idx, lab, qo, qi, ql) == int(row[-1]), (gi, si)


def test_reference_subceci_wide_queries():
    """Query graphs of 16..64 vertices: the oracle equals the counts the
    reference's own sub_ceci printed (ceci_wide.npz)."""
    z = np.load(os.path.join(GOLD, "ceci_wide.npz"))
    gs = np.concatenate([[0], np.cumsum(z["ge_len"])])
    ls = np.concatenate([[0], np.cumsum(z["gn"])])
    qs = np.concatenate([[0], np.cumsum(z["q_e_len"])])
    qls = np.concatenate([[0], np.cumsum(z["q_n"])])
    assert len(z["q_n"]) >= 60 and int(z["q_n"].max()) == 64
    for i in range(len(z["q_n"])):
        gi = int(z["q_graph"][i])
        e = z["ge"][gs[gi]: gs[gi + 1]]
        off, idx = orc.build_csr(int(z["gn"][gi]), e[:, 0], e[:, 1])
        k = int(z["q_n"][i])
        qe = z["q_e"][qs[i]: qs[i + 1]]
        qo, qi = orc.build_csr(k, qe[:, 0], qe[:, 1])
        got = orc.match(off, idx, z["gl"][ls[gi]: ls[gi + 1]], qo, qi, z["q_lab"][qls[i]: qls[i + 1]])
        assert got == int(z["expected"][i]), i


def test_sample_dataset_counts():
    z = np.load(os.path.join(GOLD, "ref_small.npz"))
    off, idx = orc.build_csr(5, z["sample_e"][:, 0], z["sample_e"][:, 1])
    for key, want in (("q1", 0), ("q2", 1)):
        qe = z[key + "_e"]
        qn = len(z[key + "_lab"])
        qo, qi = orc.build_csr(qn, qe[:, 0], qe[:, 1])
        assert orc.match(off, idx, z["sample_lab"], qo, qi, z[key + "_lab"]) == int(z["sample_counts"][want])


def test_simple_mtx_known_answers():
    # datasets/simple.mtx: the 4-path 1-2-3-4 -> no triangle, one induced 4-path.
    z = np.load(os.path.join(GOLD, "ref_small.npz"))
    e = z["simple_mtx"]
    off, idx = orc.build_csr(4, e[:, 0], e[:, 1])
    doff, didx = orc.orient(off, idx)
    assert orc.tc(doff, didx) == 0
    assert orc.motif4(off, idx).tolist() == [0, 1, 0, 0, 0, 0]
    assert orc.bruteforce(off, idx).tolist() == [2, 0, 0, 1, 0, 0, 0, 0]


@pytest.mark.parametrize("seed", range(12))
def test_restatements_match_bruteforce(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(4, 50))
    m = int(rng.integers(0, 5 * n))
    e = rng.integers(0, n, size=(m, 2)).astype(np.int32)
    off, idx = orc.build_csr(n, e[:, 0], e[:, 1])
    doff, didx = orc.orient(off, idx)
    bf = orc.bruteforce(off, idx)
    tri = orc.tc(doff, didx)
    assert tri == orc.tc_merge(doff, didx) == bf[1] == orc.clique(doff, didx, 3)
    assert orc.motif4(off, idx).tolist() == bf[2:].tolist()
    assert orc.clique(doff, didx, 4) == bf[7]
    assert orc.motif3(off, idx, tri).tolist() == bf[:2].tolist()
    for p in range(1, 9):
        r, _ = orc.pattern_solver(off, idx, p)
        assert r == orc.pattern_g2miner(off, idx, p), p
    r, cnt = orc.pattern_solver(off, idx, 0)
    assert cnt.tolist() == bf[2:].tolist()


def test_orientation_rule():
    # graph.h:128-129: keep u->v iff d(v) > d(u) or (equal and v > u)
    rng = np.random.default_rng(7)
    e = rng.integers(0, 30, size=(80, 2)).astype(np.int32)
    off, idx = orc.build_csr(30, e[:, 0], e[:, 1])
    doff, didx = orc.orient(off, idx)
    deg = np.diff(off)
    for u in range(30):
        kept = set(didx[doff[u]:doff[u + 1]].tolist())
        for v in idx[off[u]:off[u + 1]]:
            want = deg[v] > deg[u] or (deg[v] == deg[u] and v > u)
            assert (int(v) in kept) == want
    assert len(didx) * 2 == len(idx)


def test_weighted_triangle_sum():
    """orc_tc_weighted with unit weights is the triangle count; with
    out-degree weights it is checked against a plain loop."""
    rng = np.random.default_rng(8)
    n = 300
    e = rng.integers(0, n, size=(2500, 2)).astype(np.int32)
    off, idx = orc.build_csr(n, e[:, 0], e[:, 1])
    doff, didx = orc.orient(off, idx)
    assert orc.tc_weighted(doff, didx, np.ones(n, np.int64)) == orc.tc(doff, didx)
    dp = np.diff(doff)
    want = 0
    for u in range(n):
        nu = set(didx[doff[u]:doff[u + 1]].tolist())
        for v in didx[doff[u]:doff[u + 1]]:
            for w in didx[doff[v]:doff[v + 1]]:
                if w in nu:
                    want += int(dp[w])
    assert orc.tc_weighted(doff, didx, dp.astype(np.int64)) == want


@pytest.mark.parametrize("seed", range(3))
def test_c4_two_hubs_formula_matches_oracle(seed):
    """The closed-form 4-cycle count used for hub graphs too large for the
    enumerating oracle agrees with it on small two-hub graphs."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(500, 3000))
    off, idx = orc.two_hub_graph(n, 2 * n, n // 6, n // 15, [40, 70], seed=seed)
    m4 = orc.motif4(off, idx)
    assert orc.c4_two_hubs(off, idx, 0, 1) == int(m4[3] + m4[4] + 3 * m4[5])
