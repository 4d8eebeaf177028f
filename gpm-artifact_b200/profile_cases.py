"""One workload kernel on a bounded case, for ncu captures.

    python gpm-artifact_b200/profile_cases.py CASE [--scale S] [--k K] [--query Q] [--members N]

Every case builds its input, runs the counting call once untimed (first-call
work: relabel, plan, label partition) and then once more, so `ncu -k <kernel>
-s <launches of that kernel in the first call> -c 1` captures a steady-state
launch.  Cases:
  tc      triangle count, R-MAT --scale (default 20), fixed schedule
  clique  k-clique count (--k, default 4), R-MAT --scale (default 20)
  motif   3/4-vertex motif census of the first --members (default 32) graphs
          of the batched workload (their n, exponent and mean degree), one
          union, CUDA-graph replay
  match   labelled matching, R-MAT --scale (default 18) with 8 Zipf labels,
          query --query (default cycle4) walked as in the workload
Prints the count(s) so a plain run can be checked before a capture, and the
wall time of the second call (clique, motif, match).
"""
from __future__ import annotations

import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import numpy as np  # noqa: E402

import gpm  # noqa: E402
import workloads as W  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["tc", "clique", "motif", "match"])
    ap.add_argument("--scale", type=int, default=None)
    ap.add_argument("--k", type=int, default=4)
    ap.add_argument("--query", default="cycle4")
    ap.add_argument("--members", type=int, default=32)
    a = ap.parse_args()
    if a.case == "tc":
        import torch
        g = gpm.Graph.rmat(a.scale or 20, W.EDGE_FACTOR, *W.RMAT_ABC, seed=1).orient()
        out = torch.zeros(1, dtype=torch.int64, device="cuda")
        sp = torch.cuda.current_stream().cuda_stream
        for _ in range(2):
            g.tc_async(gpm.TC_BITMAP, sp, out.data_ptr())
        torch.cuda.synchronize()
        print("triangles", int(out.item()))
    elif a.case == "clique":
        import time
        g = gpm.Graph.rmat(a.scale or 20, W.EDGE_FACTOR, *W.RMAT_ABC, seed=1).orient()
        first = g.clique(a.k)
        t = time.perf_counter()
        second = g.clique(a.k)
        print(f"{a.k}-cliques", [first, second], f"{(time.perf_counter() - t) * 1e3:.1f} ms (second call)")
    elif a.case == "motif":
        nv, gam, md = W.batch_members()
        mem = [gpm.gen_chung_lu(int(nv[i]), gam[i], md[i], seed=W.member_seed(i)) for i in range(a.members)]
        import time
        b = gpm.Batch.from_edges(mem)
        r = [b.motif(use_graph=True)]
        t = time.perf_counter()
        r.append(b.motif(use_graph=True))
        assert (r[0] == r[1]).all()
        print("motif instances", int(r[1].sum()), f"{(time.perf_counter() - t) * 1e3:.1f} ms (second call)")
    else:
        scale = a.scale or 18
        n, s, d = gpm.gen_rmat(scale, W.EDGE_FACTOR, *W.RMAT_ABC, seed=W.MATCH_SEED)
        lab = gpm.gen_zipf_labels(n, W.MATCH_LABELS, W.MATCH_ZIPF, seed=W.MATCH_SEED)
        g = gpm.Graph.from_edges(n, s, d, labels=lab)
        k, e, ql = W.walk_queries(*g.csr(), lab)[a.query]
        q = gpm.Query(k, e[:, 0], e[:, 1], ql)
        import time
        first = g.match(q)
        t = time.perf_counter()
        second = g.match(q)
        print(a.query, [first, second], f"{(time.perf_counter() - t) * 1e3:.1f} ms (second call)")


if __name__ == "__main__":
    main()
