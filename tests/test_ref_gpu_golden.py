"""Counts printed by the reference's own GPU solvers (compiled from its
sources into oracle/_ref and run on a B200 by tests/golden/make_ref_gpu_golden.py)
pin the oracle (CPU tests) and the engine (GPU tests) for TC, CFSolver,
G2MinerSolver and PatternSolver."""
import os

import numpy as np
import pytest

import _oracle as orc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PATTERNS = [f"P{i}" for i in range(1, 9)]


def cases():
    z = np.load(os.path.join(GOLD, "ref_gpu.npz"))
    keys = [str(k) for k in z["keys"]]
    starts = np.concatenate([[0], np.cumsum(z["elen"])])
    for gi, n in enumerate(z["n"]):
        e = z["edges"][starts[gi]: starts[gi + 1]]
        rec = dict(zip(keys, (int(v) for v in z["table"][gi])))
        off, idx = orc.build_csr(int(n), e[:, 0], e[:, 1])
        yield gi, int(n), e, off, idx, rec


def test_oracle_matches_reference_gpu_solvers():
    for gi, n, e, off, idx, rec in cases():
        doff, didx = orc.orient(off, idx)
        tri = orc.tc(doff, didx)
        assert tri == rec["tc_e"] == rec["tc_v"], gi
        assert orc.clique(doff, didx, 4) == rec["cf4"], gi
        assert orc.clique(doff, didx, 5) == rec["cf5"], gi
        for p in PATTERNS:
            assert orc.pattern_g2miner(off, idx, int(p[1])) == rec[f"g2_{p}"], (gi, p)
            assert orc.pattern_solver(off, idx, int(p[1]))[0] == rec[f"ps_{p}"], (gi, p)
        assert orc.motif4(off, idx).tolist() == [rec[f"g2_m4_{i}"] for i in range(6)], gi


def test_patternsolver_motif4_double_processing_is_the_reference_bug():
    # PatternSolver.cuh:233-234 resets the work cursors to 0 while every warp
    # starts at its own warp id, so edges [0, #warps) run twice in
    # Motif4_edge_warp / P4_edge_warp.  On graphs whose stored edges all fall
    # below #warps the reference's counters 1..5 are exactly doubled; the
    # engine processes each edge once.
    for gi, n, e, off, idx, rec in cases():
        if len(idx) > 1000:
            continue
        m4 = orc.motif4(off, idx)
        assert rec["ps_m4_0"] == m4[0]
        assert [rec[f"ps_m4_{i}"] for i in range(1, 6)] == [2 * int(x) for x in m4[1:]], gi


@pytest.mark.gpu
def test_engine_matches_reference_gpu_solvers():
    import gpm
    for gi, n, e, off, idx, rec in cases():
        g = gpm.Graph.from_csr(off, idx)
        m4 = g.motif(4)
        assert m4.tolist() == [rec[f"g2_m4_{i}"] for i in range(6)], gi
        for p in PATTERNS:
            assert g.pattern(p, gpm.G2MINER)[0] == rec[f"g2_{p}"], (gi, p)
            assert g.pattern(p, gpm.PATTERN_SOLVER)[0] == rec[f"ps_{p}"], (gi, p)
        assert g.pattern("Motif4", gpm.G2MINER)[0] == rec["g2_m4_0"]
        d = gpm.Graph.from_csr(off, idx).orient()
        assert d.tc(gpm.E_CENTRIC) == rec["tc_e"] and d.tc(gpm.V_CENTRIC) == rec["tc_v"], gi
        assert d.clique(4) == rec["cf4"] and d.clique(5) == rec["cf5"], gi
