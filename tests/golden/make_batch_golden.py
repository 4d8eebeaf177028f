"""Oracle counts of the batched motif workload's members, as a golden fixture.

    python tests/golden/make_batch_golden.py [--nmax 100000] [--threads 0]

The workload is 256 Chung-Lu graphs (member parameters and seeds in
gpm-artifact_b200/workloads.py).  For every member with at most --nmax
vertices this script builds the member from the oracle's restatement of the
engine's seeded generator, counts all 3- and 4-vertex induced motifs with the
CPU oracle (the Motif4_G2Miner restatement and the 3-vertex census from
degrees and triangles) and stores them in batch256_oracle.npz:
  members  int64[k]     member indices
  n, m     int64[k]     vertices, generated edge draws
  counts   uint64[k, 8] induced 2-paths, triangles, 3-star, 4-path,
                        tailed triangle, 4-cycle, diamond, 4-clique
The members above --nmax cost the CPU oracle hours (their hubs); the GPU test
checks those against the engine's single-graph path instead.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "gpm-artifact_b200"))
import _oracle as orc  # noqa: E402
import workloads as W  # noqa: E402

OUT = os.path.join(HERE, "batch256_oracle.npz")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nmax", type=int, default=100000)
    ap.add_argument("--threads", type=int, default=0)
    a = ap.parse_args()
    nv, gam, md = W.batch_members()
    sel = [i for i in range(len(nv)) if nv[i] <= a.nmax]
    rows, ms, t0 = [], [], time.time()
    for k, i in enumerate(sel):
        n, s, d = orc.gen_chung_lu(int(nv[i]), gam[i], md[i], seed=W.member_seed(i), threads=a.threads)
        off, idx = orc.build_csr(n, s, d)
        m4 = orc.motif4(off, idx, a.threads)
        doff, didx = orc.orient(off, idx)
        tri = orc.tc(doff, didx, a.threads)
        rows.append(np.concatenate([orc.motif3(off, idx, tri), m4]))
        ms.append(len(s))
        print(f"{k + 1}/{len(sel)} member {i} n={n} {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(OUT, members=np.array(sel, np.int64), n=nv[sel].astype(np.int64),
                        m=np.array(ms, np.int64), counts=np.array(rows, np.uint64))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
