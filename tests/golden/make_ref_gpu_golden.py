"""Records the reference's own GPU solvers' counts as golden fixtures.

Runs on a GPU box, with the reference drivers already compiled from the
reference sources into oracle/_ref (`make -C oracle refgpu` where the
reference is mounted; the binaries travel with the repository copy):

    python tests/golden/make_ref_gpu_golden.py

For every graph below it writes a sorted, symmetric, 1-indexed .mtx file (the
reference keeps input order, so sorted input gives it sorted lists) and runs

    test_engine            e-centric TCSolver            "Result: N"
    test_trianglecounting  v-centric (hash) TCSolver     "Pattern 0: N"
    ref_cf <k>             CFSolver, k = 4, 5            "Result: N"
    test_G2Miner <P>       G2MinerSolver, P1..P8, Motif4 "Result: N" / "Result<i>: N"
    test_patternEnum <P>   PatternSolver, P1..P8, Motif4

and stores the parsed counts in ref_gpu.npz next to this file.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, os.path.join(ROOT, "gpm-artifact_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import _oracle as orc  # noqa: E402
import gpm  # noqa: E402  (generators only)

PATTERNS = [f"P{i}" for i in range(1, 9)] + ["Motif4"]


def graphs():
    out = []
    rng = np.random.default_rng(20261203)
    for n, m in [(60, 300), (400, 3000), (1500, 9000)]:
        _, s, d = gpm.gen_er(n, m, seed=n)
        out.append(("er", s, d))
    for scale, ef in [(8, 8), (10, 8), (11, 4)]:
        _, s, d = gpm.gen_rmat(scale, ef, seed=scale)
        out.append(("rmat", s, d))
    for n, gam, md in [(800, 2.2, 8.0), (2000, 2.6, 12.0)]:
        _, s, d = gpm.gen_chung_lu(n, gam, md, seed=n)
        out.append(("chunglu", s, d))
    iu, ju = np.triu_indices(40, 1)
    keep = rng.random(len(iu)) < 0.5
    out.append(("dense", iu[keep].astype(np.int32), ju[keep].astype(np.int32)))
    return out


def compact(s, d):
    """Symmetric simple CSR without isolated vertices (the .mtx loader sizes
    the graph from the smallest and largest id present)."""
    ids = np.unique(np.concatenate([s, d]))
    remap = np.full(int(ids.max()) + 1, -1, np.int64)
    remap[ids] = np.arange(len(ids))
    ss, dd = remap[s].astype(np.int32), remap[d].astype(np.int32)
    keep = ss != dd
    off, idx = orc.build_csr(len(ids), ss[keep], dd[keep])
    deg = np.diff(off)
    live = np.nonzero(deg)[0]
    if len(live) < len(ids):
        return compact(np.repeat(np.arange(len(ids)), deg).astype(np.int32), idx)
    return len(ids), off, idx


def run(args):
    out = subprocess.run([os.path.join(REF, args[0]), *args[1:]], capture_output=True, text=True, timeout=300)
    if out.returncode != 0:
        raise RuntimeError(f"{args}: {out.returncode}\n{out.stdout[-2000:]}\n{out.stderr[-2000:]}")
    return out.stdout


def first(text, pattern):
    return int(re.findall(pattern, text)[0])


def main():
    rows = []
    edges, sizes = [], []
    with tempfile.TemporaryDirectory() as td:
        for gi, (kind, s, d) in enumerate(graphs()):
            n, off, idx = compact(s, d)
            src = np.repeat(np.arange(n), np.diff(off))
            path = os.path.join(td, f"g{gi}.mtx")
            with open(path, "w") as f:
                f.write(f"{n} {n} {len(idx)}\n")
                f.writelines(f"{a + 1} {b + 1}\n" for a, b in zip(src, idx))
            lab = os.path.join(td, f"g{gi}.lab")
            with open(lab, "w") as f:
                f.writelines(f"{v + 1} 1\n" for v in range(n))
            rec = {"graph": gi}
            rec["tc_e"] = first(run(["test_engine", path, lab]), r"Result: (\d+)")
            rec["tc_v"] = first(run(["test_trianglecounting", path]), r"Pattern 0: (\d+)")
            for k in (4, 5):
                rec[f"cf{k}"] = first(run(["ref_cf", path, str(k)]), r"Result: (\d+)")
            for fam, drv in (("g2", "test_G2Miner"), ("ps", "test_patternEnum")):
                for p in PATTERNS:
                    text = run([drv, path, p])
                    if p == "Motif4":
                        got = dict(re.findall(r"Result(\d): (\d+)", text))
                        for i in range(6):
                            rec[f"{fam}_m4_{i}"] = int(got[str(i)])
                    else:
                        rec[f"{fam}_{p}"] = first(text, r"Result: (\d+)")
            print(kind, n, len(idx) // 2, rec, flush=True)
            rows.append(rec)
            edges.append(np.stack([src, idx], 1))
            sizes.append(n)
    keys = sorted(rows[0])
    np.savez_compressed(os.path.join(HERE, "ref_gpu.npz"), keys=np.array(keys),
                        table=np.array([[r[k] for k in keys] for r in rows], np.uint64),
                        n=np.array(sizes), elen=np.array([len(e) for e in edges]),
                        edges=np.concatenate(edges).astype(np.int32))
    print("wrote ref_gpu.npz")


if __name__ == "__main__":
    main()
