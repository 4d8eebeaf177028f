"""Records the reference's own GPU solvers' counts on the full-size workload
graphs as golden fixtures.

Runs on a GPU box, with the reference drivers already compiled from the
reference sources into oracle/_ref (`make -C oracle refgpu` where the
reference is mounted; the binaries travel with the repository copy):

    python tests/golden/make_ref_config_golden.py [--only tc,clique,motif]

Graphs (the engine's seeded generators, restated in the oracle so this
script never loads the engine; symmetrised, self-loops and duplicates
dropped; isolated vertices removed by an order-preserving renumbering
because the reference's .mtx loader sizes the graph from the ids present,
which changes neither the degree orientation nor any count):

    tc      R-MAT scale 22, edge factor 16, seed 1: test_engine (e-centric
            TCSolver, "Result: N") and test_trianglecounting (v-centric,
            "Pattern 0: N")
    clique  R-MAT scale 20, edge factor 16, seed 1: ref_cf 4 and ref_cf 5
            (CFSolver, "Result: N")
    motif   R-MAT scale 18, edge factor 16, seed 1: test_G2Miner Motif4
            (G2MinerSolver, "Result<i>: N", i = 0..5)

Every R-MAT graph uses (a, b, c) = (0.57, 0.19, 0.19).  The fixture
ref_config.npz stores, per graph, its size and a checksum of its symmetric
CSR (so a test can tell a changed generator from a changed count) and the
counts the reference printed.
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, os.path.join(ROOT, "tests"))
import _oracle as orc  # noqa: E402

OUT = os.path.join(HERE, "ref_config.npz")
GRAPHS = {"tc": (22, 1), "clique": (20, 1), "motif": (18, 1)}  # workload -> (R-MAT scale, seed)


def csr_checksum(off, idx):
    """Order-sensitive checksum of a CSR: sum over stored entries of
    (position + 1) * (id + 1), modulo 2^64, plus the offsets' sum."""
    pos = np.arange(1, len(idx) + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        s = np.sum(pos * (idx.astype(np.uint64) + np.uint64(1)), dtype=np.uint64)
        s += np.sum(off.astype(np.uint64), dtype=np.uint64)
    return int(s)


def rmat_csr(scale, seed):
    n, s, d = orc.gen_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
    return n, *orc.build_csr(n, s, d)


def compact_csr(off, idx):
    deg = np.diff(off)
    live = np.nonzero(deg)[0]
    remap = np.full(len(deg), -1, np.int64)
    remap[live] = np.arange(len(live))
    off2 = np.zeros(len(live) + 1, np.int64)
    off2[1:] = np.cumsum(deg[live])
    return off2, remap[idx].astype(np.int32)


def run(args, timeout=3600):
    t = time.perf_counter()
    out = subprocess.run([os.path.join(REF, args[0]), *args[1:]], capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError(f"{args}: {out.returncode}\n{out.stdout[-2000:]}\n{out.stderr[-2000:]}")
    print(f"{args[0]} {' '.join(args[2:])}: {time.perf_counter() - t:.1f} s", flush=True)
    return out.stdout


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="tc,clique,motif")
    todo = ap.parse_args().only.split(",")
    rec = dict(np.load(OUT)) if os.path.exists(OUT) else {}
    with tempfile.TemporaryDirectory() as td:
        for wl in todo:
            scale, seed = GRAPHS[wl]
            n, off, idx = rmat_csr(scale, seed)
            rec[f"{wl}_n"] = np.int64(n)
            rec[f"{wl}_nnz"] = np.int64(len(idx))
            rec[f"{wl}_checksum"] = np.uint64(csr_checksum(off, idx))
            coff, cidx = compact_csr(off, idx)
            path = os.path.join(td, f"{wl}.mtx")
            orc.write_mtx(path, coff, cidx)
            if wl == "tc":
                lab = os.path.join(td, "tc.lab")
                with open(lab, "w") as f:
                    f.write("".join(f"{v} 1\n" for v in range(1, len(coff))))
                e = re.findall(r"Result: (\d+)", run(["test_engine", path, lab]))
                v = re.findall(r"Pattern 0: (\d+)", run(["test_trianglecounting", path]))
                rec["tc_e_centric"] = np.uint64(int(e[-1]))
                rec["tc_v_centric"] = np.uint64(int(v[-1]))
            elif wl == "clique":
                for k in (4, 5):
                    c = re.findall(r"Result: (\d+)", run(["ref_cf", path, str(k)]))
                    rec[f"clique_k{k}"] = np.uint64(int(c[-1]))
            elif wl == "motif":
                got = dict(re.findall(r"Result(\d): (\d+)", run(["test_G2Miner", path, "Motif4"])))
                rec["motif_g2miner"] = np.array([int(got[str(i)]) for i in range(6)], np.uint64)
            print(wl, {k: (v.tolist() if hasattr(v, "tolist") else v) for k, v in rec.items() if k.startswith(wl)},
                  flush=True)
    np.savez_compressed(OUT, **rec)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
