"""Parity at the full sizes of the measured workloads.

The counts come from the reference itself, run on the same graphs:
  ref_config.npz      the reference's own GPU solvers (make_ref_config_golden.py):
                      TCSolver e- and v-centric on R-MAT 22, CFSolver k = 4, 5 on
                      R-MAT 20, G2MinerSolver Motif4 on R-MAT 18
  ceci_config.npz     the reference's sub_ceci matcher (make_ceci_config_golden.py)
                      on R-MAT 16, 18, 21 with 8 Zipf labels and the walked queries
  batch256_oracle.npz the CPU oracle on every member of the 256-graph motif batch
                      with at most 100,000 vertices (make_batch_golden.py)
Each graph is regenerated from its seed and its CSR checksum compared with the
one recorded beside the counts, so a changed generator cannot pass as a
changed count.
"""
import os

import numpy as np
import pytest

import gpm
import workloads as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture(name):
    path = os.path.join(GOLD, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not recorded yet")
    return np.load(path)


def checksum(off, idx):
    pos = np.arange(1, len(idx) + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        s = np.sum(pos * (idx.astype(np.uint64) + np.uint64(1)), dtype=np.uint64)
        s += np.sum(off.astype(np.uint64), dtype=np.uint64)
    return int(s)


def rmat_graph(z, wl, seed):
    scale = {"tc": W.TC_SCALE, "clique": W.CLIQUE_SCALE, "motif": 18}[wl]
    g = gpm.Graph.rmat(scale, W.EDGE_FACTOR, *W.RMAT_ABC, seed=seed)
    off, idx = g.csr()
    assert len(off) - 1 == int(z[f"{wl}_n"]) and len(idx) == int(z[f"{wl}_nnz"])
    assert checksum(off, idx) == int(z[f"{wl}_checksum"]), "generator changed: re-record the fixture"
    return g


def test_tc_rmat22_equals_reference_solvers():
    z = fixture("ref_config.npz")
    want = int(z["tc_e_centric"])
    assert want == int(z["tc_v_centric"])
    g = rmat_graph(z, "tc", W.TC_SEED).orient()
    gpm.Sched.pretrained().attach(g)  # the shipped weights drive TC_LEARNED
    out = np.zeros(1, np.uint64)
    import torch
    d = torch.zeros(1, dtype=torch.int64, device="cuda")
    sp = torch.cuda.current_stream().cuda_stream
    for v in (gpm.TC_AUTO, gpm.TC_BITMAP, gpm.TC_LEARNED, gpm.TC_HASH):
        g.tc_async(v, sp, d.data_ptr())
        torch.cuda.synchronize()
        out[0] = int(d.item())
        assert int(out[0]) == want, v
    assert g.tc(gpm.E_CENTRIC) == want


def test_tc_rmat22_end_to_end_from_host():
    z = fixture("ref_config.npz")
    g = rmat_graph(z, "tc", W.TC_SEED)
    off, idx = g.csr()
    assert gpm.tc_host_csr(off, idx) == int(z["tc_e_centric"])


def test_cliques_rmat20_equal_cfsolver():
    z = fixture("ref_config.npz")
    g = rmat_graph(z, "clique", W.CLIQUE_SEED).orient()
    assert g.clique(4) == int(z["clique_k4"])
    assert g.clique(5) == int(z["clique_k5"])
    assert g.clique(4, edge_centric=True) == int(z["clique_k4"])


def test_motif4_rmat18_equals_g2miner():
    z = fixture("ref_config.npz")
    g = rmat_graph(z, "motif", 1)
    assert g.motif(4).tolist() == z["motif_g2miner"].tolist()
    assert g.pattern("Motif4", gpm.G2MINER)[1].tolist() == z["motif_g2miner"].tolist()


def labelled(scale):
    n, s, d = gpm.gen_rmat(scale, W.EDGE_FACTOR, *W.RMAT_ABC, seed=W.MATCH_SEED)
    lab = gpm.gen_zipf_labels(n, W.MATCH_LABELS, W.MATCH_ZIPF, seed=W.MATCH_SEED)
    g = gpm.Graph.from_edges(n, s, d, labels=lab)
    return g, W.walk_queries(*g.csr(), lab)


@pytest.mark.parametrize("scale", [16, 18, 21])
def test_labelled_matching_equals_sub_ceci(scale):
    z = fixture("ceci_config.npz")
    rows = [(r, lab) for r, lab in zip(z["rows"], z["labels"]) if r[0] == scale]
    if not rows:
        pytest.skip(f"no sub_ceci counts recorded at R-MAT {scale}")
    g, queries = labelled(scale)
    names = list(W.SHAPES)
    for r, lab in rows:
        k, e, ql = queries[names[int(r[1])]]
        assert ql.tolist() == lab[:k].tolist(), "walked query changed: re-record the fixture"
        assert g.match(gpm.Query(k, e[:, 0], e[:, 1], ql)) == int(r[2]), (scale, names[int(r[1])])


def test_batch256_members_equal_single_graphs_and_oracle():
    z = fixture("batch256_oracle.npz")
    nv, gam, md = W.batch_members()
    members = [gpm.gen_chung_lu(int(nv[i]), gam[i], md[i], seed=W.member_seed(i)) for i in range(len(nv))]
    b = gpm.Batch.from_edges(members)
    got = b.motif(use_graph=True)
    again = b.motif(use_graph=True)
    assert (got == again).all()
    oracle = dict(zip(z["members"].tolist(), z["counts"]))
    assert len(oracle) >= 150
    for i in range(len(nv)):
        if i in oracle:
            assert int(z["m"][list(z["members"]).index(i)]) == len(members[i][1])
            assert got[i].tolist() == oracle[i].tolist(), i
        off, idx = b.member_csr(i)
        g = gpm.Graph.from_csr(off, idx)
        assert got[i, 2:].tolist() == g.motif(4).tolist(), i
        assert got[i, :2].tolist() == g.motif(3).tolist(), i
        g.close()
