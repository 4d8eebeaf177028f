"""Measurements of the engine's other workloads, each beside its plain path.

    python gpm-artifact_b200/suite.py [--only er,clique,motif,motifcl,match,batch] [--quick]

Prints one JSON line per workload:
  er      triangle count, Erdos-Renyi G(16384, 131072 draws), degree-oriented
  clique  4- and 5-cliques, R-MAT scale 20 (ef 16): local-bitset kernel vs the
          edge-centric kernel shaped like the reference's clique_k_edge_warp
  motif   all 3- and 4-vertex motifs of R-MAT scale 18 (ef 16, seed 1)
  motifcl all 3- and 4-vertex motifs of a Chung-Lu graph (n 200,000, exponent
          2.18, mean degree 62): hub-dominated 4-cycles
  match   labelled matching with sub_ceci semantics, R-MAT with 8 Zipf(1.2)
          labels, five queries (triangle, 4-cycle, diamond, house, 6-vertex
          pyramid = apex over a 5-cycle) found by seeded random walks on the
          data graph with the walked vertices' labels
  batch   all 3- and 4-vertex motifs of 256 Chung-Lu graphs (n log-uniform in
          [1e3, 1e6], exponent U[2.1, 2.8], mean degree U[8, 64]): one union,
          one launch per stage, CUDA-graph replay, autotuned -- against one
          gpm_motif call per graph
Times are medians of synchronised wall times of repeated counting calls
(first calls, which include relabelling and planning, are single samples);
graph generation and host copies are outside them unless named.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import gpm  # noqa: E402

from workloads import SHAPES, batch_members, walk_query  # noqa: E402


def timed(fn, reps=1):
    """Result and median wall time of `reps` synchronised calls (medians:
    the GPUs and hosts these runs share see other users' work)."""
    import torch
    ts = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t)
    return r, float(np.median(ts))


def run_er():
    import torch
    n, s, d = gpm.gen_er(16384, 131072, seed=1)
    g = gpm.Graph.from_edges(n, s, d).orient()
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    sp = torch.cuda.current_stream().cuda_stream
    res = {}
    for name, v in (("bitmap", gpm.TC_BITMAP), ("hash", gpm.TC_HASH), ("bsearch", gpm.TC_BSEARCH)):
        g.tc_async(v, sp, out.data_ptr())

        def burst():  # 20 counts queued back to back on the stream
            for _ in range(20):
                g.tc_async(v, sp, out.data_ptr())
        _, t = timed(burst, 5)
        res[name] = t / 20 * 1e3
    m = g.info().nnz
    return {"workload": "tc_er_16384_131072", "triangles": int(out.item()), "m": m,
            "ms_per_count": res, "teps_bitmap": m / (res["bitmap"] / 1e3)}


def count_ms(g, variant, reps=5, burst=5):
    """Median over `reps` of the device milliseconds of one count in a burst
    of `burst` counts (CUDA events on the current stream), and the count."""
    import torch
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = torch.cuda.current_stream()
    g.tc_async(variant, st.cuda_stream, out.data_ptr())
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(burst):
            g.tc_async(variant, st.cuda_stream, out.data_ptr())
        e1.record(st)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / burst)
    return float(np.median(ts)), int(out.item())


def sched_eval(g):
    """Triangle-count schedules of one oriented graph, in device ms: the
    fixed rule, the shipped learned scheduler, the per-task optimum of the
    logged costs (each owner in its cheapest of the 6 configurations) and
    the reference-threshold hash kernel (plain heuristic) on the graph and
    on its degree-relabelled copy (the reference's v-centric input)."""
    res = {}
    res["fixed_ms"], want = count_ms(g, gpm.TC_BITMAP)
    gpm.Sched.pretrained().attach(g)
    res["learned_ms"], c = count_ms(g, gpm.TC_LEARNED)
    assert c == want
    cost = g.task_costs()
    task = cost.sum(axis=1) > 0
    best = np.argmin(np.where(cost > 0, cost, np.inf), axis=1).astype(np.uint8)
    best[~task] = 1
    res["logged_warp_cycles_per_task_optimum"] = float(np.min(np.where(cost > 0, cost, np.inf), axis=1)[task].sum())
    g.set_schedule(best)
    res["per_task_optimum_ms"], c = count_ms(g, gpm.TC_LEARNED)
    assert c == want
    cta = np.argmin(np.where(cost[:, 3:] > 0, cost[:, 3:], np.inf), axis=1).astype(np.uint8) + 3
    cta[~task] = 4
    g.set_schedule(cta)
    res["per_task_optimum_cta_only_ms"], c = count_ms(g, gpm.TC_LEARNED)
    assert c == want
    res["plain_hash_ms"], c = count_ms(g, gpm.TC_HASH, reps=3, burst=2)
    assert c == want
    res["triangles"] = want
    return res


def run_sched(scales=(18, 20, 22)):
    res = {"workload": "tc_schedules"}
    for sc in scales:
        g = gpm.Graph.rmat(sc, 16, seed=1).orient()
        res[f"rmat{sc}"] = sched_eval(g)
        r = gpm.Graph.rmat(sc, 16, seed=1).orient(relabel=True)
        res[f"rmat{sc}"]["plain_hash_relabelled_ms"], _ = count_ms(r, gpm.TC_HASH, reps=3, burst=2)
        print(json.dumps({sc: res[f"rmat{sc}"]}), flush=True)
    n, s, d = gpm.gen_chung_lu(1000000, 2.1, 32.0, seed=7)
    g = gpm.Graph.from_edges(n, s, d).orient()
    res["chunglu_1e6_g2.1_d32"] = sched_eval(g)
    return res


def run_clique(scale):
    g = gpm.Graph.rmat(scale, 16, seed=1).orient()
    res = {"workload": f"clique_rmat{scale}_ef16"}
    for k in (4, 5):
        _, t0 = timed(lambda: g.clique(k))  # first call: relabel (k = 4 only) and plan
        c, t = timed(lambda: g.clique(k), 5)
        c2, t2 = timed(lambda: g.clique(k, edge_centric=True), 3)
        assert c == c2, (k, c, c2)
        res[f"k{k}"] = {"cliques": c, "ms_first_call": t0 * 1e3, "ms_bitset": t * 1e3, "ms_edge_centric": t2 * 1e3,
                        "cliques_per_s": c / t, "speedup": t2 / t}
    return res


def run_motif(scale):
    """All 3- and 4-vertex motifs of one R-MAT graph (edge factor 16, seed
    1): first call (relabel and plan included) and repeated calls."""
    g = gpm.Graph.rmat(scale, 16, seed=1)
    return motif_result(g, f"motif_rmat{scale}_ef16")


def motif_result(g, name):
    m4, t_first = timed(lambda: g.motif(4))
    m4b, t = timed(lambda: g.motif(4), 7)
    assert m4.tolist() == m4b.tolist()
    m3, t3 = timed(lambda: g.motif(3), 7)
    return {"workload": name, "m": g.info().nnz // 2, "motif4": [int(x) for x in m4],
            "motif3": [int(x) for x in m3], "s_motif4_first": t_first, "s_motif4": t, "s_motif3": t3,
            "instances_per_s": float(m4.sum()) / t}


def run_motif_chung_lu():
    """All 3- and 4-vertex motifs of one heavy-tailed Chung-Lu graph
    (n = 200,000, exponent 2.18, mean degree 62, seed 11): 4-cycles are
    dominated by hub tasks with ~10^5-10^6 distinct 2-hop endpoints."""
    n, s, d = gpm.gen_chung_lu(200000, 2.18, 62.0, seed=11)
    return motif_result(gpm.Graph.from_edges(n, s, d), "motif_chunglu_200000_g2.18_d62")


def run_match(scale, seed=3):
    n, s, d = gpm.gen_rmat(scale, 16, seed=seed)
    lab = gpm.gen_zipf_labels(n, 8, 1.2, seed=seed)
    g = gpm.Graph.from_edges(n, s, d, labels=lab)
    off, idx = g.csr()
    rng = np.random.default_rng(seed)
    res = {"workload": f"match_rmat{scale}_ef16_zipf8", "queries": {}}
    for name, shape in SHAPES.items():
        ql = walk_query(off, idx, lab, shape, rng)
        e = np.array(shape[1], np.int32)
        q = gpm.Query(shape[0], e[:, 0], e[:, 1], ql)
        c, t = timed(lambda: g.match(q))
        res["queries"][name] = {"labels": ql.tolist(), "matches": c, "ms": t * 1e3, "matches_per_s": c / t}
    return res


def run_match_batch(scale, names, seed=3):
    """The labelled queries of one graph counted together (gpm_match_batch:
    one persistent launch over every query's tasks, autotuned task split,
    CUDA-graph replay) against one gpm_match call per query."""
    n, s, d = gpm.gen_rmat(scale, 16, seed=seed)
    lab = gpm.gen_zipf_labels(n, 8, 1.2, seed=seed)
    g = gpm.Graph.from_edges(n, s, d, labels=lab)
    off, idx = g.csr()
    allq = walk_queries_dict(off, idx, lab, seed)
    qs = [allq[k] for k in names]
    single, t_single = [], 0.0
    g.match(qs[0])  # label partition and bitmaps built outside the timings
    for q in qs:
        c, t = timed(lambda: g.match(q))
        single.append(c)
        t_single += t
    b = gpm.MatchBatch(g, qs)
    r, t_first = timed(lambda: b.run(use_graph=True))
    assert r[:, 0].tolist() == single
    span = b.autotune()
    b.run(use_graph=True)
    r, t = timed(lambda: b.run(use_graph=True), 3)
    assert r[:, 0].tolist() == single
    return {"workload": f"match_batch_rmat{scale}_ef16_zipf8", "queries": names, "embeddings": single,
            "s_single_calls": t_single, "s_batched_first": t_first, "s_batched_replay": t, "tuned_span": span,
            "tasks": b.info()[0], "speedup_vs_single_calls": t_single / t, "embeddings_per_s": sum(single) / t}


def walk_queries_dict(off, idx, lab, seed):
    from workloads import walk_queries
    return {k: gpm.Query(kk, e[:, 0], e[:, 1], ql) for k, (kk, e, ql) in walk_queries(off, idx, lab, seed).items()}


def run_match_scales(scales, budget_s, seed=3):
    """The labelled workload at growing R-MAT scales (same label law, queries
    walked on each graph): a query stops growing once one run took more than
    budget_s / 8 seconds (the next scale costs several times more)."""
    res = {"workload": "match_rmat_ef16_zipf8_scales", "budget_s": budget_s, "queries": {k: [] for k in SHAPES}}
    alive = set(SHAPES)
    for scale in scales:
        if not alive:
            break
        n, s, d = gpm.gen_rmat(scale, 16, seed=seed)
        lab = gpm.gen_zipf_labels(n, 8, 1.2, seed=seed)
        g = gpm.Graph.from_edges(n, s, d, labels=lab)
        off, idx = g.csr()
        rng = np.random.default_rng(seed)
        for name, shape in SHAPES.items():
            ql = walk_query(off, idx, lab, shape, rng)
            if name not in alive:
                continue
            e = np.array(shape[1], np.int32)
            q = gpm.Query(shape[0], e[:, 0], e[:, 1], ql)
            c, t = timed(lambda: g.match(q))
            res["queries"][name].append({"scale": scale, "m": g.info().nnz // 2, "labels": ql.tolist(),
                                         "matches": c, "s": t, "matches_per_s": c / t})
            print(json.dumps({"scale": scale, "query": name, "matches": c, "s": round(t, 4)}), flush=True)
            if t > budget_s / 8:
                alive.discard(name)
        g.close()
    return res



def run_batch(count, nmax):
    n, gam, md = batch_members(count, nmax)
    b = gpm.Batch.chung_lu(n, gam, md, seed=11)
    ng, ntot, nnz = b.info()
    r0, t_first = timed(lambda: b.motif(use_graph=True))
    tuned = b.autotune()
    r1, t_tuned_first = timed(lambda: b.motif(use_graph=True))
    r2, t_replay = timed(lambda: b.motif(use_graph=True), 3)
    assert (r0 == r1).all() and (r1 == r2).all()
    stages = b.stage_ms()
    # plain: one gpm_motif call per member graph (its own schedule, its syncs)
    t_plain = 0.0
    for i in range(ng):
        off, idx = b.member_csr(i)
        g = gpm.Graph.from_csr(off, idx)
        m4, t = timed(lambda: g.motif(4))
        t_plain += t
        assert m4.tolist() == r2[i, 2:].tolist(), i
        g.close()
    total = int(r2.sum())
    return {"workload": f"motif_batch_{count}_chunglu_nmax{int(nmax)}", "graphs": ng, "vertices": ntot,
            "stored_edges": nnz, "motif_instances": total, "tuned_thresholds": tuned, "stage_ms": stages,
            "s_batched_first_call": t_first, "s_batched_replay": t_replay, "s_plain_per_graph": t_plain,
            "speedup_replay_vs_plain": t_plain / t_replay, "instances_per_s": total / t_replay}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="er,clique,motif,motifcl,match,batch,sched")
    ap.add_argument("--quick", action="store_true", help="smaller sizes for a smoke run")
    ap.add_argument("--match-scales", default="", help="e.g. 16,18,20,21: the labelled workload at growing scales")
    ap.add_argument("--match-budget", type=float, default=240.0, help="seconds a query may take at its last scale x 8")
    ap.add_argument("--batch-queries", default="triangle,cycle4,diamond", help="queries of the matchbatch workload")
    a = ap.parse_args()
    todo = a.only.split(",")
    if "er" in todo:
        print(json.dumps(run_er()), flush=True)
    if "clique" in todo:
        print(json.dumps(run_clique(16 if a.quick else 20)), flush=True)
    if "motif" in todo:
        print(json.dumps(run_motif(14 if a.quick else 18)), flush=True)
    if "motifcl" in todo:
        print(json.dumps(run_motif_chung_lu()), flush=True)
    if "match" in todo:
        if a.match_scales:
            print(json.dumps(run_match_scales([int(x) for x in a.match_scales.split(",")], a.match_budget)),
                  flush=True)
        else:
            print(json.dumps(run_match(12 if a.quick else 16)), flush=True)
    if "batch" in todo:
        print(json.dumps(run_batch(32 if a.quick else 256, 3e4 if a.quick else 1e6)), flush=True)
    if "matchbatch" in todo:
        print(json.dumps(run_match_batch(14 if a.quick else 21, a.batch_queries.split(","))), flush=True)
    if "sched" in todo:
        print(json.dumps(run_sched((14, 16) if a.quick else (18, 20, 22))), flush=True)


if __name__ == "__main__":
    main()
