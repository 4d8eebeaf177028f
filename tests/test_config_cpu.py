"""The full-size workload graphs on the CPU: the oracle's restated
generators rebuild exactly the graphs the reference's own solvers counted
(size and CSR checksum recorded beside their counts in ref_config.npz), and
the oracle's triangle count of the R-MAT 22 graph equals the reference's."""
import os

import numpy as np
import pytest

import _oracle as orc
import workloads as W

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def checksum(off, idx):
    pos = np.arange(1, len(idx) + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        s = np.sum(pos * (idx.astype(np.uint64) + np.uint64(1)), dtype=np.uint64)
        s += np.sum(off.astype(np.uint64), dtype=np.uint64)
    return int(s)


@pytest.fixture(scope="module")
def ref():
    return np.load(os.path.join(GOLD, "ref_config.npz"))


@pytest.mark.parametrize("wl,scale,seed", [("motif", 18, 1), ("clique", W.CLIQUE_SCALE, W.CLIQUE_SEED),
                                           ("tc", W.TC_SCALE, W.TC_SEED)])
def test_oracle_rebuilds_the_reference_graphs(ref, wl, scale, seed):
    n, s, d = orc.gen_rmat(scale, W.EDGE_FACTOR, *W.RMAT_ABC, seed=seed)
    off, idx = orc.build_csr(n, s, d)
    assert n == int(ref[f"{wl}_n"]) and len(idx) == int(ref[f"{wl}_nnz"])
    assert checksum(off, idx) == int(ref[f"{wl}_checksum"])
    if wl == "tc":
        doff, didx = orc.orient(off, idx)
        assert orc.tc(doff, didx) == int(ref["tc_e_centric"]) == int(ref["tc_v_centric"])
