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
        gpm.Query(17, [0], [1], np.zeros(17))
    g2 = gpm.Graph.from_edges(4, [0, 1], [1, 2])
    with pytest.raises(gpm.GpmError):
        g2.match(gpm.Query(2, [0], [1], [0, 0]))
