"""Regenerates the golden fixtures in tests/golden from the AntiRF reference.

Run in a container where the reference is mounted (REFERENCE_DIR, else
$GPM_REF_DIR, else oracle/Makefile's REF_DIR) and oracle/_ref/myceci has been
built (`make -C oracle`):

    python tests/golden/make_golden.py [REFERENCE_DIR]

Outputs (committed; the GPU box never reads the reference itself):
  hprd_kat.npz    sub_ceci's 200 HPRD known-answer tests
                  (sub_ceci/test/data_graph/HPRD.graph, query_graph/*,
                  expected_output.res) as CSR arrays + expected counts.
  ref_small.npz   the reference's tiny fixtures: datasets/simple.mtx (as its
                  loader reads it), sub_ceci/test/sample_dataset/* with the
                  counts sub_ceci prints for them, querysets/qg1..qg5 shapes.
  ceci_random.npz counts printed by the reference's own sub_ceci (compiled
                  from its sources into oracle/_ref) for seeded random
                  labelled graphs and the five query shapes used by the
                  labelled-matching workload.
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
sys.path.insert(0, os.path.join(ROOT, "tests"))
import _oracle as orc  # noqa: E402


def read_tve(path):
    lab, edges = {}, []
    for line in open(path):
        t = line.split()
        if not t:
            continue
        if t[0] == "v":
            lab[int(t[1])] = int(t[2])
        elif t[0] == "e":
            edges.append((int(t[1]), int(t[2])))
    n = max(lab) + 1
    labels = np.array([lab.get(i, 0) for i in range(n)], np.int32)
    e = np.array(edges, np.int32).reshape(-1, 2)
    return n, e, labels


def csr_of(n, e):
    return orc.build_csr(n, e[:, 0], e[:, 1], symmetrize=True)


def write_tve(path, n, e, labels):
    off, idx = csr_of(n, e)
    deg = np.diff(off)
    und = [(int(a), int(b)) for a, b in zip(np.repeat(np.arange(n), deg), idx) if a < b]
    with open(path, "w") as f:
        f.write(f"t {n} {len(und)}\n")
        for v in range(n):
            f.write(f"v {v} {int(labels[v])} {int(deg[v])}\n")
        for a, b in und:
            f.write(f"e {a} {b}\n")


def run_ceci(myceci, data, query):
    out = subprocess.run([myceci, "-d", data, "-q", query, "-filter", "CECI", "-order", "CECI", "-engine", "CECI"],
                         capture_output=True, text=True, check=True).stdout
    return int(re.search(r"#Embeddings: (\d+)", out).group(1))


# query shapes of the labelled workload (edges); pyramid-6 = apex over a 5-cycle
SHAPES = {
    "triangle": (3, [(0, 1), (1, 2), (2, 0)]),
    "cycle4": (4, [(0, 1), (1, 2), (2, 3), (3, 0)]),
    "diamond": (4, [(0, 1), (0, 2), (0, 3), (1, 2), (2, 3)]),
    "house": (5, [(0, 1), (0, 4), (1, 2), (1, 4), (2, 3), (3, 4)]),
    "pyramid6": (6, [(0, 1), (0, 2), (0, 3), (0, 4), (0, 5), (1, 2), (2, 3), (3, 4), (4, 5), (5, 1)]),
}


def default_ref_dir():
    if os.environ.get("GPM_REF_DIR"):
        return os.environ["GPM_REF_DIR"]
    for line in open(os.path.join(ROOT, "oracle", "Makefile")):
        if line.startswith("REF_DIR") and "?=" in line:
            return line.split("?=", 1)[1].strip()
    raise SystemExit("give the reference's directory (argument or GPM_REF_DIR)")


def main(ref=None):
    ref = ref or default_ref_dir()
    ceci = os.path.join(ref, "sub_ceci", "test")
    # ---- HPRD KATs
    n, e, lab = read_tve(os.path.join(ceci, "data_graph", "HPRD.graph"))
    off, idx = csr_of(n, e)
    exp = {}
    for line in open(os.path.join(ceci, "expected_output.res")):
        k, v = line.strip().split(":")
        exp[k] = int(v)
    qn, qoff_all, qidx_all, qlab_all, counts = [], [], [], [], []
    for i in range(1, 201):
        name = f"query_dense_16_{i}"
        m, qe, ql = read_tve(os.path.join(ceci, "query_graph", name + ".graph"))
        qo, qi = csr_of(m, qe)
        qn.append(m)
        qoff_all.append(qo)
        qidx_all.append(qi)
        qlab_all.append(ql)
        counts.append(exp[name])
    np.savez_compressed(os.path.join(HERE, "hprd_kat.npz"), off=off, idx=idx, labels=lab, qn=np.array(qn),
                        qoff=np.concatenate(qoff_all), qidx=np.concatenate(qidx_all),
                        qlab=np.concatenate(qlab_all), expected=np.array(counts, np.uint64))
    # ---- small reference fixtures
    mtx = [tuple(map(int, l.split())) for l in open(os.path.join(ref, "datasets", "simple.mtx"))
           if l.strip() and not l.startswith("%")][1:]
    mtx = np.array([p for p in mtx if p[0] != p[1]], np.int32) - 1  # vmin = 1 shift
    sd = os.path.join(ceci, "sample_dataset")
    dn, de, dl = read_tve(os.path.join(sd, "test_case_1.graph"))
    q1n, q1e, q1l = read_tve(os.path.join(sd, "query1_positive.graph"))
    q2n, q2e, q2l = read_tve(os.path.join(sd, "query2_positive.graph"))
    myceci = os.path.join(ROOT, "oracle", "_ref", "myceci")
    c1 = run_ceci(myceci, os.path.join(sd, "test_case_1.graph"), os.path.join(sd, "query1_positive.graph"))
    c2 = run_ceci(myceci, os.path.join(sd, "test_case_1.graph"), os.path.join(sd, "query2_positive.graph"))
    qg = {}
    for k in range(1, 6):
        _, qe_, _ = read_tve(os.path.join(ref, "querysets", f"qg{k}"))
        qg[f"qg{k}"] = qe_
    np.savez_compressed(os.path.join(HERE, "ref_small.npz"), simple_mtx=mtx, sample_e=de, sample_lab=dl,
                        q1_e=q1e, q1_lab=q1l, q2_e=q2e, q2_lab=q2l, sample_counts=np.array([c1, c2], np.uint64),
                        **qg)
    # ---- the reference's sub_ceci on seeded random labelled graphs
    rng = np.random.default_rng(20261203)
    rows = []
    graphs = []
    with tempfile.TemporaryDirectory() as td:
        for gi in range(6):
            gn = int(rng.integers(40, 120))
            gm = int(gn * rng.uniform(2.0, 5.0))
            ge = rng.integers(0, gn, size=(gm, 2)).astype(np.int32)
            ge = ge[ge[:, 0] != ge[:, 1]]
            nl = int(rng.integers(1, 4))
            gl = rng.integers(0, nl, size=gn).astype(np.int32)
            dpath = os.path.join(td, f"g{gi}.graph")
            write_tve(dpath, gn, ge, gl)
            graphs.append((gn, ge, gl))
            for si, (sname, (sn, sedges)) in enumerate(SHAPES.items()):
                sl = rng.integers(0, nl, size=sn).astype(np.int32)
                qpath = os.path.join(td, f"q{gi}_{si}.graph")
                write_tve(qpath, sn, np.array(sedges, np.int32), sl)
                rows.append((gi, si, *np.pad(sl, (0, 6 - sn)), run_ceci(myceci, dpath, qpath)))
    gsz = np.array([g[0] for g in graphs])
    np.savez_compressed(os.path.join(HERE, "ceci_random.npz"), rows=np.array(rows, np.int64), gn=gsz,
                        ge=np.concatenate([g[1] for g in graphs]), ge_len=np.array([len(g[1]) for g in graphs]),
                        gl=np.concatenate([g[2] for g in graphs]),
                        shapes=np.array(list(SHAPES.keys())))
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main(*sys.argv[1:])
