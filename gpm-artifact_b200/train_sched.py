"""Trains the learned task scheduler's shipped parameters (sched_tc.f32).

    python gpm-artifact_b200/train_sched.py [--out PATH] [--steps 1500] [--lr 3e-3]
    python gpm-artifact_b200/train_sched.py --eval-only

Training graphs (the R-MAT scale-22 benchmark graph is not among them):
R-MAT scales 15, 16, 17, 18 (edge factor 16, seeds 11, 12, 13, 21) and two
Chung-Lu graphs (n 60000, exponent 2.2, mean degree 24, seed 14; n 120000,
exponent 2.6, mean degree 48, seed 15), each degree-oriented.  For every
graph the engine logs each owner task's cost under each of the six
configurations (instrumented count kernel, gpm_sched_collect) beside the
task's eight features; full-batch Adam fits the log2 costs.  Afterwards the
held-out R-MAT scale 20-22 graphs (seed 1) are counted under the fixed and the
learned schedule and the times printed as one JSON line each.
Needs a CUDA device.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import gpm  # noqa: E402

RMAT = [(15, 11), (16, 12), (17, 13), (18, 21)]
CHUNG_LU = [(60000, 2.2, 24.0, 14), (120000, 2.6, 48.0, 15)]


def train(steps, lr, seed=7):
    s = gpm.Sched(seed=seed)
    rows = 0
    for scale, sd in RMAT:
        rows += s.collect(gpm.Graph.rmat(scale, 16, seed=sd).orient())
    for n, gam, md, sd in CHUNG_LU:
        _, a, b = gpm.gen_chung_lu(n, gam, md, seed=sd)
        rows += s.collect(gpm.Graph.from_edges(n, a, b).orient())
    first = s.train(1, lr)
    last = s.train(steps, lr)
    return s, rows, first, last


def held_out(s, scales=(20, 21, 22), reps=5):
    import torch
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    sp = torch.cuda.current_stream().cuda_stream
    for scale in scales:
        g = gpm.Graph.rmat(scale, 16, seed=1).orient()
        s.attach(g)
        res = {}
        for name, v in (("fixed", gpm.TC_BITMAP), ("learned", gpm.TC_LEARNED)):
            g.tc_async(v, sp, out.data_ptr())
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                g.tc_async(v, sp, out.data_ptr())
            e1.record()
            torch.cuda.synchronize()
            res[name] = {"ms": e0.elapsed_time(e1) / reps, "triangles": int(out.item())}
        cfg = s.assign(g)
        hist = np.bincount(cfg[cfg != 255], minlength=6).tolist()
        print(json.dumps({"rmat_scale": scale, **res, "config_histogram": hist}), flush=True)
        g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=gpm.Sched.PRETRAINED)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--no-eval", action="store_true")
    ap.add_argument("--eval-only", action="store_true", help="evaluate the shipped parameters, no training")
    a = ap.parse_args()
    if a.eval_only:
        held_out(gpm.Sched.pretrained())
        return
    s, rows, first, last = train(a.steps, a.lr)
    s.params().astype(np.float32).tofile(a.out)
    print(json.dumps({"rows": rows, "loss_first": first, "loss_last": last, "out": a.out}), flush=True)
    if not a.no_eval:
        held_out(s)


if __name__ == "__main__":
    main()
