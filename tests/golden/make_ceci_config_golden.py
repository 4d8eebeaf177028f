"""Counts of the reference's own sub_ceci matcher on the labelled workload's
graphs, as a golden fixture.

    python tests/golden/make_ceci_config_golden.py [--scales 16,18,21] [--queries 21:triangle,cycle4,diamond]
                                                   [--workdir DIR] [--timeout 7200] [--jobs 4]

sub_ceci is built from the reference's sources into oracle/_ref/myceci
(`make -C oracle ref`).  For each R-MAT scale (edge factor 16, seed 3, 8
Zipf(1.2) labels with seed 3; the engine's seeded generators restated in the
oracle) the script writes the data graph in sub_ceci's t/v/e format, walks the
five workload queries on it (gpm-artifact_b200/workloads.py: triangle, 4-cycle,
diamond, house, 6-vertex pyramid; labels copied from the walked vertices) and
runs

    myceci -d data.graph -q <query>.graph -filter CECI -order CECI -engine CECI

for every query (at the scales --queries names, only the queries it lists),
--jobs at a time, each for at most --timeout seconds.  A
query's output already present in the work directory from an earlier run of
the same command on the same files is read instead of run again (the R-MAT 21
4-cycle and diamond take sub_ceci about an hour each).  ceci_config.npz keeps
one row per finished (scale, query): the scale, the query index in SHAPES
order, its labels, sub_ceci's #Embeddings and its "Enumerate time".
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "gpm-artifact_b200"))
import _oracle as orc  # noqa: E402
import workloads as W  # noqa: E402

OUT = os.path.join(HERE, "ceci_config.npz")
MYCECI = os.path.join(ROOT, "oracle", "_ref", "myceci")


def write_query(path, k, e, ql):
    deg = [int(((e[:, 0] == v) | (e[:, 1] == v)).sum()) for v in range(k)]
    with open(path, "w") as f:
        f.write(f"t {k} {len(e)}\n")
        f.writelines(f"v {v} {int(ql[v])} {deg[v]}\n" for v in range(k))
        f.writelines(f"e {int(a)} {int(b)}\n" for a, b in e)


def parse(out_path):
    if not os.path.exists(out_path):
        return None
    text = open(out_path).read()
    c = re.findall(r"#Embeddings: (\d+)", text)
    t = re.findall(r"Enumerate time \(seconds\): ([0-9.eE+-]+)", text)
    return (int(c[-1]), float(t[-1])) if c and t else None


def run_one(d, name, timeout):
    out = os.path.join(d, name + ".out")
    got = parse(out)
    if got:
        return got
    t0 = time.time()
    # sub_ceci prints two lines per search call (gigabytes on these graphs):
    # only the summary at the end is kept
    with open(out, "w") as f:
        p1 = subprocess.Popen(["timeout", str(int(timeout)), MYCECI, "-d", os.path.join(d, "data.graph"), "-q",
                               os.path.join(d, name + ".graph"), "-filter", "CECI", "-order", "CECI", "-engine",
                               "CECI"], stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
        p2 = subprocess.Popen(["tail", "-n", "40"], stdin=p1.stdout, stdout=f)
        p1.stdout.close()
        p2.wait()
        p1.wait()
    got = parse(out)
    print(f"{d} {name}: {time.time() - t0:.0f} s, {'done' if got else 'no result (time limit)'}", flush=True)
    return got


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scales", default="16,18,21")
    ap.add_argument("--workdir", default=os.path.join(ROOT, "_work", "ceci"))
    ap.add_argument("--timeout", type=float, default=7200)
    ap.add_argument("--jobs", type=int, default=4)
    ap.add_argument("--queries", default="21:triangle,cycle4,diamond",
                    help="scale:q1,q2;scale:... -- queries run at that scale (default: all five)")
    a = ap.parse_args()
    only = {int(t.split(":")[0]): t.split(":")[1].split(",") for t in a.queries.split(";") if t}
    names = list(W.SHAPES)
    rows = {}
    if os.path.exists(OUT):
        z = np.load(OUT)
        for r, lab in zip(z["rows"], z["labels"]):
            rows[(int(r[0]), int(r[1]))] = (r, lab)
    jobs = []
    for scale in (int(x) for x in a.scales.split(",")):
        d = os.path.join(a.workdir, f"r{scale}")
        os.makedirs(d, exist_ok=True)
        n, s, dst = orc.gen_rmat(scale, W.EDGE_FACTOR, *W.RMAT_ABC, seed=W.MATCH_SEED)
        lab = orc.gen_zipf_labels(n, W.MATCH_LABELS, W.MATCH_ZIPF, seed=W.MATCH_SEED)
        off, idx = orc.build_csr(n, s, dst)
        if not os.path.exists(os.path.join(d, "data.graph")):
            orc.write_tve(os.path.join(d, "data.graph"), off, idx, lab)
        for qi, (name, (k, e, ql)) in enumerate(W.walk_queries(off, idx, lab).items()):
            qp = os.path.join(d, name + ".graph")
            fresh = os.path.join(d, name + ".graph.new")
            write_query(fresh, k, e, ql)
            if os.path.exists(qp) and open(qp).read() != open(fresh).read():
                os.remove(os.path.join(d, name + ".out")) if os.path.exists(os.path.join(d, name + ".out")) else None
            os.replace(fresh, qp)
            if scale not in only or name in only[scale]:
                jobs.append((scale, qi, d, name, ql))
    with ThreadPoolExecutor(a.jobs) as pool:
        res = list(pool.map(lambda j: run_one(j[2], j[3], a.timeout), jobs))
    for (scale, qi, d, name, ql), got in zip(jobs, res):
        if got:
            row = np.array([scale, qi, got[0], int(round(got[1] * 1e4))], np.int64)
            rows[(scale, qi)] = (row, np.pad(ql, (0, 6 - len(ql)), constant_values=-1))
            print(scale, name, got, flush=True)
    keys = sorted(rows)
    np.savez_compressed(OUT, rows=np.array([rows[k][0] for k in keys], np.int64),
                        labels=np.array([rows[k][1] for k in keys], np.int32), shapes=np.array(names))
    print("wrote", OUT, "rows (scale, query, embeddings, enumerate time in 1e-4 s):", len(keys))


if __name__ == "__main__":
    main()
