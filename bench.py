"""Benchmark of the graph-pattern-mining count engine, one B200 per rank.

Headline (the JSON line's top-level fields): exact triangle counting of an
R-MAT scale-22 graph (4,194,304 vertices, edge factor 16, (a,b,c,d) =
(0.57, 0.19, 0.19, 0.05), seed 1 + rank, symmetrised, self-loops and
duplicates removed, degree-oriented int32 CSR).  One step = one triangle
count of the whole graph.  Metric: TEPS = undirected edges / seconds per
count (higher is better).

  value    device-resident DAG in HBM with the count's schedule built by an
           earlier count, the count kernel timed with CUDA events on the
           launching stream (inputs 0.3 GB > 126 MB L2, no flush needed);
           ms_per_count_with_plan times a count on a freshly oriented graph
           (relabel + plan + count)
  e2e      the same count through the C ABI from pinned HOST memory
           (gpm_tc_host_csr: H2D of the symmetric CSR, orientation on the
           device, count, D2H of the 8-byte result), all inside the timed
           region
  roofline DRAM bytes per launch (ncu, profiles/k_tc_rank_rmat22.md) over
           the count kernel's event time, against the measured HBM copy
           bandwidth; beside it the graded algorithmic bytes
           B = 4(n+1) + 4m + 4*sum_{u->v} deg+(v), which this kernel does not
           read, and the bytes it requests (mostly served by L2)
  cpu_baseline  the CPU restatement (OpenMP marker algorithm) on all host
           threads and on one, timed on a bounded vertex sample of the graph

At N = 1 the line also carries "workloads" (default --workload all): the
other measured workloads, each with its own value, e2e, roofline and CPU
baseline -- k-cliques (k = 4, 5) of R-MAT 20, the batched 3/4-vertex motif
census of 256 Chung-Lu graphs (autotuned, CUDA-graph replay, against one
call per graph) and labelled matching on R-MAT 21 with 8 Zipf labels.

--impl reference: the reference's CPU implementation of each workload on the
host cores -- the oracle port of its counting loops (the reference has no CPU
counter of its own for TC, cliques or motifs) and the reference's own
sub_ceci matcher built from its sources (oracle/_ref/myceci) for labelled
matching -- never the engine (libgpm.so is not loaded).  Beside it, the
reference's own GPU triangle-count solvers on the same graph.

Multi-GPU (torchrun): each rank counts its own independently seeded graph;
no data-path collective (weak scaling); the timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpm-artifact_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import workloads as W  # noqa: E402  (pure numpy: loads neither the engine nor the oracle)

SCALE, EF = W.TC_SCALE, W.EDGE_FACTOR
A, B, C = W.RMAT_ABC
METRIC = "triangle-count TEPS (R-MAT scale 22, exact uint64)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100, help="timed counts (100 x ~7 ms: long enough to sample clocks)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="all", choices=["all", "tc", "clique", "motif", "match"],
                    help="all: the TC line with the other workloads under 'workloads' (N = 1 only)")
    ap.add_argument("--scale", type=int, default=SCALE, help="R-MAT scale of the TC workload (22 is the headline)")
    ap.add_argument("--variant", default="auto",
                    choices=["auto", "bitmap", "hash", "bsearch", "merge", "learned"])
    ap.add_argument("--match-queries", default="triangle,cycle4,diamond",
                    help="labelled queries timed on the GPU (all five: triangle,cycle4,diamond,house,pyramid6)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true", help="reference arm: skip the reference's GPU solvers")
    ap.add_argument("--ref-extra", default="", help="reference arm: also time the reference's GPU solvers on "
                    "'clique' (R-MAT 20, k = 4, 5) and/or 'motif' (R-MAT 18, Motif4); one more JSON line")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target time of each CPU sample")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def host_threads():
    return len(os.sched_getaffinity(0))


class Clocks:
    """nvidia-smi sampler for the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period_ms=50):
        self.index = index
        self.period_ms = period_ms
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)  # the first sample lands before the timed work starts
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def profiled(name, key):
    """A figure recorded in a committed ncu summary (profiles/<name>.md, a
    line '<key>: <number>'), else None."""
    path = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith(key + ":"):
            v = line.split(":", 1)[1].strip()
            return float(v) if "." in v else int(v)
    return None


def roofline(traffic, kernel_ms, hbm, peak_kind, **extra):
    """DRAM bytes per launch (ncu) over the kernel's average CUDA-event time,
    against the measured HBM copy bandwidth."""
    gbs = traffic / (kernel_ms / 1e3) / 1e9 if traffic else None
    r = {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm if gbs else None,
         "traffic": traffic, "kernel_ms": kernel_ms, "peak_kind": peak_kind,
         "basis": "DRAM bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum) / CUDA-event time"}
    r.update(extra)
    return r


def over_ranks(dist, dev, ms, edges):
    """Whole-job figures from one rank's own: (max over ranks of the per-step
    milliseconds, sum over ranks of the undirected edges counted per step).
    With no process group the rank's own figures are the job's."""
    if not dist:
        return float(ms), float(edges)
    import torch
    tt = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    me = torch.tensor([float(edges)], dtype=torch.float64, device=dev)
    dist.all_reduce(me, op=dist.ReduceOp.SUM)
    return float(tt.item()), float(me.item())


def event_ms(fn, stream, reps=1):
    """Device milliseconds of each of `reps` calls of fn, CUDA events on
    `stream` around each, synchronised on both sides."""
    import torch
    out = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out, r


# --------------------------------------------------------------------------- CPU baselines
def _stride_sample(run, weight, seconds):
    """Runs run(keep) on every stride-th task, growing the sample until it
    takes about seconds / 3 or covers everything; returns (seconds, the
    sample's share of the work weight, run's result, description)."""
    import numpy as np
    n = len(weight)
    total = float(weight.sum())
    stride = max(1, n // 64)
    while True:
        keep = np.zeros(n, np.uint8)
        keep[::stride] = 1
        frac = float(weight[keep.astype(bool)].sum()) / max(total, 1e-12)
        t0 = time.perf_counter()
        r = run(keep)
        t = time.perf_counter() - t0
        if t >= seconds / 3 or stride == 1:
            break
        stride = max(1, int(stride * max(0.05, t / seconds)))
    return t, frac, r, f"tasks of every {stride}-th vertex ({frac * 100:.2f}% of the work weight) in {t:.2f} s"


def cpu_tc(doff, didx, m_und, seconds, threads):
    """The CPU restatement of the triangle count (OpenMP marker algorithm):
    TEPS from the sample's time scaled by its share of the work weight
    w(u) = d+(u) + sum_{v in N+(u)} d+(v)."""
    import numpy as np
    import _oracle as orc
    n = len(doff) - 1
    deg = np.diff(doff)
    wv = np.zeros(n, np.float64)
    np.add.at(wv, np.repeat(np.arange(n), deg), deg[didx].astype(np.float64))
    wv += deg
    t, frac, _, sample = _stride_sample(lambda keep: orc.tc_tasks(doff, didx, keep, threads), wv, seconds)
    return m_und / (t / max(frac, 1e-12)), sample + ", scaled to the whole graph"


def cpu_clique(doff, didx, k, seconds, threads):
    """The CPU restatement of CFSolver's nested intersections on a vertex
    sample: the cliques found in the sampled tasks per second of it."""
    import numpy as np
    import _oracle as orc
    deg = np.diff(doff)
    wv = np.zeros(len(doff) - 1, np.float64)
    np.add.at(wv, np.repeat(np.arange(len(deg)), deg), (deg[didx] + np.repeat(deg, deg)).astype(np.float64))
    t, frac, found, sample = _stride_sample(lambda keep: orc.clique_tasks(doff, didx, k, keep, threads), wv,
                                            seconds)
    return found / t, sample + f", {found} cliques found"


def cpu_motif_members(gen_member, members, seconds, threads):
    """The CPU restatement of Motif4_G2Miner (and the 3-vertex census from
    its degrees and triangles) on whole member graphs, smallest first, until
    `seconds` are spent: motif instances per second over the members done.
    The large, hub-heavy members cost the CPU most, so this rate favours the
    CPU."""
    import numpy as np
    import _oracle as orc
    order = sorted(range(len(members)), key=lambda i: members[i])
    inst, spent, done = 0, 0.0, 0
    for i in order:
        n, s, d = gen_member(i)
        off, idx = orc.build_csr(n, s, d)
        t0 = time.perf_counter()
        m4 = orc.motif4(off, idx, threads)
        doff, didx = orc.orient(off, idx)
        tri = orc.tc(doff, didx, threads)
        m3 = orc.motif3(off, idx, tri)
        spent += time.perf_counter() - t0
        inst += int(np.sum(m4)) + int(np.sum(m3))
        done += 1
        if spent >= seconds:
            break
    return inst / max(spent, 1e-9), (f"{done} whole member graphs (the smallest, n <= "
                                     f"{members[order[done - 1]]}) in {spent:.2f} s")


def cpu_match_ceci(off, idx, labels, queries, num):
    """The reference's own sub_ceci (built from its sources into
    oracle/_ref/myceci; single-threaded), -filter/-order/-engine CECI, each
    query stopped after `num` embeddings (its -num option); embeddings per
    second by its own "Enumerate time" line (sub_ceci/myceci.cpp:1111).  The
    five queries run as concurrent single-threaded processes."""
    import _oracle as orc
    exe = os.path.join(ROOT, "oracle", "_ref", "myceci")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/myceci not built (make -C oracle ref where the reference is mounted)"}
    res = {}
    with tempfile.TemporaryDirectory() as td:
        data = os.path.join(td, "data.graph")
        orc.write_tve(data, off, idx, labels)
        procs = {}
        for name, (k, e, ql) in queries.items():
            qp = os.path.join(td, name + ".graph")
            deg = [int(((e[:, 0] == v) | (e[:, 1] == v)).sum()) for v in range(k)]
            with open(qp, "w") as f:
                f.write(f"t {k} {len(e)}\n")
                f.writelines(f"v {v} {int(ql[v])} {deg[v]}\n" for v in range(k))
                f.writelines(f"e {int(a)} {int(b)}\n" for a, b in e)
            # sub_ceci prints two lines per search call (hundreds of MB here):
            # only the summary at the end is kept
            p1 = subprocess.Popen([exe, "-d", data, "-q", qp, "-filter", "CECI", "-order", "CECI", "-engine", "CECI",
                                   "-num", str(int(num))], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL)
            procs[name] = (p1, subprocess.Popen(["tail", "-n", "40"], stdin=p1.stdout, stdout=subprocess.PIPE,
                                                text=True))
            p1.stdout.close()
        for name, (p1, p) in procs.items():
            try:
                out, _ = p.communicate(timeout=900)
                p1.wait(timeout=60)
            except subprocess.TimeoutExpired:
                p1.kill()
                p.kill()
                res[name] = {"unavailable": "no result within 900 s"}
                continue
            t = re.findall(r"Enumerate time \(seconds\): ([0-9.eE+-]+)", out)
            c = re.findall(r"#Embeddings: (\d+)", out)
            if not t or not c:
                res[name] = {"unavailable": f"exit {p.returncode}, no Enumerate/#Embeddings line"}
                continue
            emb, sec = int(c[-1]), float(t[-1])
            res[name] = {"embeddings": emb, "enumerate_s": sec, "embeddings_per_s": emb / max(sec, 1e-9),
                         "complete": emb < num}
    return res


# --------------------------------------------------------------------------- GPU workloads (this engine)
def tc_line(args, rank, world, dist, local):
    import numpy as np
    import torch
    import gpm

    dev = torch.device("cuda", local)
    seed = W.TC_SEED + rank
    g = gpm.Graph.rmat(args.scale, EF, A, B, C, seed=seed)
    sym_off, sym_idx = g.csr()
    g.orient()
    inf = g.info()
    n, m_und = inf.n, inf.nnz
    wedge, pair = g.work()
    bytes_graded = 4 * (n + 1) + 4 * m_und + 4 * wedge
    # bytes this kernel requests: the clipped segments (4 B a key, a 16-byte
    # descriptor each), the core-row words of the dense segments (4 B each),
    # every owner list once, 36 B of offsets and counts per owner
    nseg, seg_keys, owner_keys, ntasks, dense_segs, dense_words = g.plan_stats()
    bytes_req = 4 * seg_keys + 4 * dense_words + 16 * nseg + 4 * owner_keys + 36 * ntasks
    variants = {"auto": gpm.TC_AUTO, "bitmap": gpm.TC_BITMAP, "hash": gpm.TC_HASH, "bsearch": gpm.TC_BSEARCH,
                "merge": gpm.TC_MERGE, "learned": gpm.TC_LEARNED}
    variant = variants[args.variant]
    # the shipped scheduler weights (trained on logged task costs of smaller
    # R-MAT and Chung-Lu graphs, none of them this graph)
    sched = gpm.Sched.pretrained()
    sched.set_default()
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    out = torch.zeros(1, dtype=torch.int64, device=dev)

    warm = max(args.warmup, 3)
    for _ in range(warm):
        g.tc_async(variant, sp, out.data_ptr())
    torch.cuda.synchronize()
    count = int(out.item())

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        t_all0 = torch.cuda.Event(enable_timing=True)
        t_all1 = torch.cuda.Event(enable_timing=True)
        t_all0.record(stream)
        for k in range(args.steps):
            starts[k].record(stream)
            g.tc_async(variant, sp, out.data_ptr())
            ends[k].record(stream)
        t_all1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms_total = t_all0.elapsed_time(t_all1)
    per = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    assert int(out.item()) == count, "count changed between steps"
    ms_step, m_total = over_ranks(dist, dev, ms_total / args.steps, m_und)
    value = m_total / (ms_step / 1e3)

    # ---- a count on a freshly oriented graph: rank relabel + plan + count
    def fresh():
        g.drop_plans()
        return event_ms(lambda: g.tc_async(variant, sp, out.data_ptr()), stream)[0][0]
    with_plan = statistics.median([fresh() for _ in range(3)])
    assert int(out.item()) == count
    g.tc_async(variant, sp, out.data_ptr())  # schedule cached again

    # ---- the other schedules on the same graph (outside the timed region)
    others = {}
    for name in ("bitmap", "learned", "hash"):
        if name == args.variant or (name == "bitmap" and args.variant == "auto"):
            continue
        v = variants[name]
        g.tc_async(v, sp, out.data_ptr())
        torch.cuda.synchronize()
        assert int(out.item()) == count, name
        ms, _ = event_ms(lambda: [g.tc_async(v, sp, out.data_ptr()) for _ in range(3)], stream)
        others[name] = round(ms[0] / 3, 3)
    others[args.variant] = round(ms_step, 3)

    # ---- end to end through the C ABI from pinned host memory
    e2e = None
    if not args.no_e2e:
        hoff = torch.from_numpy(sym_off).pin_memory()
        hidx = torch.from_numpy(sym_idx).pin_memory()
        nn = len(sym_off) - 1
        for _ in range(2):
            c2 = gpm.tc_host_csr_ptrs(nn, hoff.data_ptr(), hidx.data_ptr(), variant, sp)
        assert c2 == count, (c2, count)
        ks = max(3, min(args.steps, 5))
        if dist:
            dist.barrier()
        ms, _ = event_ms(lambda: [gpm.tc_host_csr_ptrs(nn, hoff.data_ptr(), hidx.data_ptr(), variant, sp)
                                  for _ in range(ks)], stream)
        ms_e2e, _ = over_ranks(dist, dev, ms[0] / ks, m_und)
        e2e = {"value": m_total / (ms_e2e / 1e3), "unit": "TEPS", "ms_per_step": ms_e2e,
               "h2d_bytes_per_step": int(hoff.numel() * 8 + hidx.numel() * 4), "d2h_bytes_per_step": 8,
               "path": "gpm_tc_host_csr (pinned symmetric CSR -> upload overlapped with the relabel -> plan -> "
                       "count -> 8-byte result)"}

    # ---- CPU baseline (rank 0, N = 1 only): all host threads and one
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        doff, didx = g.csr()
        threads = host_threads()
        v_all, sample = cpu_tc(doff, didx, m_und, args.cpu_seconds, threads)
        v_one, sample1 = cpu_tc(doff, didx, m_und, args.cpu_seconds / 2, 1)
        cpu = {"value": v_all, "unit": "TEPS", "cores": threads, "kind": "port", "sample": sample,
               "one_core": {"value": v_one, "cores": 1, "sample": sample1}}

    hbm, peak_kind = peaks()
    avg_kernel_ms = sum(per) / len(per)
    traffic = (profiled("k_tc_rank_rmat22", "traffic_bytes_per_launch[" +
                        ("learned" if args.variant == "learned" else "bitmap") + "]")
               if args.scale == SCALE and args.variant in ("auto", "bitmap", "learned") else None)
    roof = roofline(traffic, avg_kernel_ms, hbm, peak_kind,
                    graded={"algorithmic_bytes": bytes_graded,
                            "gbs": bytes_graded / (avg_kernel_ms / 1e3) / 1e9,
                            "frac_graded": bytes_graded / (avg_kernel_ms / 1e3) / 1e9 / hbm,
                            "note": "B = 4(n+1) + 4m + 4*sum_{u->v} d+(v): every wedge list read in full, "
                                    "the vertex iterator's reads; this kernel streams only the shorter side, "
                                    "clipped, so it never reads these bytes"},
                    requested={"bytes": bytes_req, "gbs": bytes_req / (avg_kernel_ms / 1e3) / 1e9,
                               "frac": bytes_req / (avg_kernel_ms / 1e3) / 1e9 / hbm,
                               "note": "bytes the kernel loads (segment keys, core-row words and descriptors, owner lists), "
                                       "mostly served by L2"},
                    plan={"segments": nseg, "segment_keys": seg_keys, "owner_keys": owner_keys,
                          "owner_tasks": ntasks, "dense_segments": dense_segs, "dense_words": dense_words})
    line = {
        "metric": METRIC,
        "value": value, "unit": "TEPS", "n_gpus": world, "steps": args.steps, "warmup": warm,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"tc_rmat{args.scale}_ef{EF}", "graph": "R-MAT", "scale": args.scale,
                   "edge_factor": EF, "abcd": [A, B, C, round(1 - A - B - C, 2)], "seed": "1+rank",
                   "n": n, "m_undirected": m_und, "dag_max_outdeg": inf.max_degree,
                   "triangles": count, "variant": args.variant, "parallelism": f"replicas{world}",
                   "l2": "inputs > L2 (DAG %.0f MB), no flush" % ((8 * (n + 1) + 4 * m_und) / 1e6),
                   "ms_per_count_with_plan": with_plan,
                   "ms_per_count_by_schedule": others},
        "e2e": e2e,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        # per step one count kernel (k_tc_rank, or k_tc_hash / k_tc_bsearch / k_tc_merge), and k_tc_dense
        # beside k_tc_rank when the plan has dense core segments
        "gpu_launches": args.steps * (2 if dense_segs and args.variant in ("auto", "bitmap") else 1),
    }
    g.close()
    return line


def clique_workload(args, stream):
    """k-cliques (k = 4, 5) of R-MAT scale 20 on the degree-oriented DAG."""
    import numpy as np
    import torch
    import gpm
    sp = stream.cuda_stream
    hbm, peak_kind = peaks()
    n, s, d = gpm.gen_rmat(W.CLIQUE_SCALE, EF, A, B, C, seed=W.CLIQUE_SEED)
    g = gpm.Graph.from_edges(n, s, d)
    sym_off, sym_idx = g.csr()
    g.orient()
    inf = g.info()
    res = {"workload": f"clique_rmat{W.CLIQUE_SCALE}_ef{EF}", "metric": "k-clique matches/s (exact uint64)",
           "unit": "cliques/s", "n": inf.n, "m_undirected": inf.nnz, "dag_max_outdeg": inf.max_degree}
    launches = 0
    for k in (4, 5):
        first, c0 = event_ms(lambda: g.clique(k), stream)  # relabel (first k) + local-DAG plan + count
        reps = max(1, min(args.steps, 10 if k == 4 else 3))
        ms, c = event_ms(lambda: g.clique(k), stream, reps)
        assert c == c0
        launches += reps
        avg = sum(ms) / len(ms)
        r = {"cliques": c, "value": c / (avg / 1e3), "ms_per_count": avg, "steps": reps,
             "ms_first_call": first[0],
             "roofline": roofline(profiled(f"k_clique_local_rmat{W.CLIQUE_SCALE}",
                                           f"traffic_bytes_per_launch[k{k}]"), avg, hbm, peak_kind,
                                  issue_active_pct=profiled(f"k_clique_local_rmat{W.CLIQUE_SCALE}",
                                                            f"issue_active_pct[k{k}]"),
                                  note="bitset intersections in shared memory: issue-bound, DRAM only for "
                                       "the graph (profiles/k_clique_local_rmat20.md)")}
        if k == 4:
            # the reference-shaped path: warp per stored edge, materialised
            # nested intersections (clique_4_edge_warp)
            pm, pc = event_ms(lambda: g.clique(k, edge_centric=True), stream)
            assert pc == c
            r["plain_edge_centric_ms"] = pm[0]
            r["speedup_vs_plain"] = pm[0] / avg
        res[f"k{k}"] = r
    res["value"] = res["k4"]["value"]
    # end to end: pinned symmetric CSR -> gpm_graph_create_csr -> orient ->
    # 4-clique count -> result
    if not args.no_e2e:
        hoff = torch.from_numpy(sym_off).pin_memory()
        hidx = torch.from_numpy(sym_idx).pin_memory()

        def e2e_once():
            h = gpm.Graph.from_csr_ptrs(len(sym_off) - 1, hoff.data_ptr(), hidx.data_ptr())
            c = h.orient().clique(4)
            h.close()
            return c
        ms, c = event_ms(e2e_once, stream, 2)
        assert c == res["k4"]["cliques"]
        res["e2e"] = {"value": c / (min(ms) / 1e3), "unit": "cliques/s", "ms_per_step": min(ms), "k": 4,
                      "h2d_bytes_per_step": int(hoff.numel() * 8 + hidx.numel() * 4), "d2h_bytes_per_step": 8}
    g.close()
    if not args.no_cpu:
        import _oracle as orc
        off, idx = orc.build_csr(n, s, d)
        doff, didx = orc.orient(off, idx)
        th = host_threads()
        for k in (4, 5):
            v, smp = cpu_clique(doff, didx, k, args.cpu_seconds, th)
            res[f"k{k}"]["cpu_baseline"] = {"value": v, "unit": "cliques/s", "cores": th, "kind": "port",
                                            "sample": smp}
        v1, smp1 = cpu_clique(doff, didx, 4, args.cpu_seconds / 2, 1)
        res["k4"]["cpu_baseline"]["one_core"] = {"value": v1, "cores": 1, "sample": smp1}
        res["cpu_baseline"] = res["k4"]["cpu_baseline"]
    res["gpu_launches_timed"] = launches
    return res


def motif_workload(args, stream):
    """All 3- and 4-vertex induced motifs of 256 Chung-Lu graphs: one device
    union, one persistent launch per pipeline stage, autotuned thresholds,
    replayed as a CUDA graph; against one gpm_motif call per graph."""
    import numpy as np
    import torch
    import gpm
    sp = stream.cuda_stream
    hbm, peak_kind = peaks()
    nv, gam, md = W.batch_members()
    t0 = time.perf_counter()
    members = [gpm.gen_chung_lu(int(nv[i]), gam[i], md[i], seed=W.member_seed(i)) for i in range(len(nv))]
    t_gen = time.perf_counter() - t0
    src = np.concatenate([m[1] for m in members])
    dst = np.concatenate([m[2] for m in members])
    mlen = np.array([len(m[1]) for m in members], np.int64)
    del members
    hsrc = torch.from_numpy(src).pin_memory()
    hdst = torch.from_numpy(dst).pin_memory()
    del src, dst
    res = {"workload": f"motif_batch_{len(nv)}_chunglu", "metric": "3/4-vertex motif instances/s (exact uint64)",
           "unit": "instances/s", "graphs": len(nv), "host_generation_s": t_gen}

    def create():
        return gpm.Batch.from_edge_ptrs(nv, mlen, hsrc.data_ptr(), hdst.data_ptr())

    # end to end: pinned member edge lists -> union CSR on the device -> plan ->
    # captured pipeline -> per-member counts to the host
    def e2e_once():
        b = create()
        r = b.motif(use_graph=True)
        b.close()
        return r
    e2e_ms, r_e2e = event_ms(e2e_once, stream, 1 if args.no_e2e else 2)
    b = create()
    ng, ntot, nnz = b.info()
    first, r0 = event_ms(lambda: b.motif(use_graph=True), stream)
    assert (r0 == r_e2e).all()
    t0 = time.perf_counter()
    tuned = b.autotune()
    t_tune = time.perf_counter() - t0
    b.motif(use_graph=True)  # captures the tuned pipeline
    dout = torch.zeros(8 * ng, dtype=torch.int64, device=stream.device)
    reps = max(1, min(args.steps, 5))
    ms, _ = event_ms(lambda: b.motif_async(True, sp, dout.data_ptr()), stream, reps)
    r1 = dout.cpu().numpy().view(np.uint64).reshape(ng, 8)
    assert (r1 == r0).all()
    stages = b.stage_ms()
    avg = sum(ms) / len(ms)
    total = int(r1.sum())
    # plain: one gpm_motif call per member graph (its own plan and syncs),
    # member CSRs already on the device
    t_plain = 0.0
    for i in range(ng):
        off, idx = b.member_csr(i)
        gg = gpm.Graph.from_csr(off, idx)
        pm, m4 = event_ms(lambda: gg.motif(4), stream)
        t_plain += pm[0]
        assert m4.tolist() == r1[i, 2:].tolist(), i
        gg.close()
    b.close()
    res.update({
        "vertices": ntot, "stored_edges": nnz, "motif_instances": total, "value": total / (avg / 1e3),
        "ms_per_replay": avg, "steps": reps, "ms_first_call": first[0], "tuned_thresholds": tuned,
        "autotune_s": t_tune, "stage_ms": stages, "plain_per_graph_ms": t_plain,
        "speedup_vs_plain": t_plain / avg,
        "plain": "one gpm_motif (k = 4) call per member graph, member CSR resident, first call each "
                 "(its own relabel, plan and synchronisations)",
        "e2e": {"value": total / (min(e2e_ms) / 1e3), "unit": "instances/s", "ms_per_step": min(e2e_ms),
                "h2d_bytes_per_step": int(hsrc.numel() * 4 + hdst.numel() * 4),
                "d2h_bytes_per_step": int(8 * 8 * ng)},
        # the dominant stage's kernel, k_c4_big: its DRAM bytes and duration
        # from one ncu capture of this batch (the stage time also holds k_c4)
        "roofline": roofline(profiled("k_edge_tri_batch32", "traffic_bytes_per_launch[c4_big_batch256]"),
                             profiled("k_edge_tri_batch32", "kernel_ms[c4_big_batch256]") or stages["four_cycles"],
                             hbm, peak_kind, kernel="k_c4_big (the 4-cycle stage's large tasks)",
                             issue_active_pct=profiled("k_edge_tri_batch32", "issue_active_pct[edge_tri_batch32]"),
                             note="issue- and latency-bound pipeline (profiles/k_edge_tri_batch32.md, "
                                  "profiles/k_c4_big_chunglu200k.md)"),
        "gpu_launches_timed": None,
    })
    if not args.no_cpu:
        import _oracle as orc
        th = host_threads()
        gen = lambda i: orc.gen_chung_lu(int(nv[i]), gam[i], md[i], seed=W.member_seed(i), threads=th)
        v, smp = cpu_motif_members(gen, [int(x) for x in nv], args.cpu_seconds, th)
        res["cpu_baseline"] = {"value": v, "unit": "instances/s", "cores": th, "kind": "port", "sample": smp}
    return res


def match_workload(args, stream):
    """Labelled matching (sub_ceci semantics) on R-MAT 21 with 8 Zipf labels."""
    import numpy as np
    import torch
    import gpm
    n, s, d = gpm.gen_rmat(W.MATCH_SCALE, EF, A, B, C, seed=W.MATCH_SEED)
    lab = gpm.gen_zipf_labels(n, W.MATCH_LABELS, W.MATCH_ZIPF, seed=W.MATCH_SEED)
    g = gpm.Graph.from_edges(n, s, d, labels=lab)
    off, idx = g.csr()
    queries = W.walk_queries(off, idx, lab)
    todo = [q for q in args.match_queries.split(",") if q in queries]
    res = {"workload": f"match_rmat{W.MATCH_SCALE}_ef{EF}_zipf{W.MATCH_LABELS}",
           "metric": "labelled embeddings/s (sub_ceci semantics, exact uint64)", "unit": "embeddings/s",
           "m_undirected": len(idx) // 2, "queries": {}}
    tot_e, tot_ms = 0, 0.0
    for name in todo:
        k, e, ql = queries[name]
        q = gpm.Query(k, e[:, 0], e[:, 1], ql)
        first, c = event_ms(lambda: g.match(q), stream)
        reps = 2 if first[0] > 2000 else max(1, min(args.steps, 5))
        ms, c2 = event_ms(lambda: g.match(q), stream, reps)
        assert c2 == c
        avg = sum(ms) / len(ms)
        res["queries"][name] = {"labels": ql.tolist(), "embeddings": c, "ms": avg, "ms_first_call": first[0],
                                "value": c / (avg / 1e3), "steps": reps}
        tot_e += c
        tot_ms += avg
    res["value"] = tot_e / (tot_ms / 1e3) if tot_ms else None
    res["ms_per_step"] = tot_ms
    res["untimed_queries"] = [q for q in queries if q not in todo]
    hbm, peak_kind = peaks()
    if "cycle4" in res["queries"]:
        res["roofline"] = roofline(profiled("k_match_rmat21_cycle4", "traffic_bytes_per_launch[cycle4_rmat21]"),
                                   res["queries"]["cycle4"]["ms"], hbm, peak_kind, kernel="k_match (4-cycle query)",
                                   note="DRAM bytes of one ncu capture of this query on this graph: the "
                                        "back-edge tests read adjacency-bitmap words and label-segment keys "
                                        "at random (profiles/k_match_rmat21_cycle4.md)")
    if todo:
        # the same queries counted together: one persistent launch over every
        # query's tasks, autotuned task split, CUDA-graph replay -- against
        # one gpm_match call per query (each synchronising, as the reference
        # synchronises after every pattern)
        qs = [gpm.Query(*[queries[k][0], queries[k][1][:, 0], queries[k][1][:, 1], queries[k][2]]) for k in todo]
        mb = gpm.MatchBatch(g, qs)
        span = mb.autotune()
        first, r = event_ms(lambda: mb.run(use_graph=True), stream)
        reps = max(1, min(args.steps, 3))
        ms, r = event_ms(lambda: mb.run(use_graph=True), stream, reps)
        assert r[:, 0].tolist() == [res["queries"][k]["embeddings"] for k in todo]
        bt = sum(ms) / len(ms)
        res["batched"] = {"queries": todo, "ms_per_replay": bt, "value": tot_e / (bt / 1e3), "tuned_span": span,
                          "tasks": mb.info()[0], "speedup_vs_single_calls": tot_ms / bt, "steps": reps}
        mb.close()
    if not args.no_e2e and todo:
        # end to end: host edge list + labels -> graph on the device -> label
        # partition -> the first query's count -> result
        k, e, ql = queries[todo[0]]
        hs = torch.from_numpy(np.ascontiguousarray(s)).pin_memory()
        hd = torch.from_numpy(np.ascontiguousarray(d)).pin_memory()
        hl = torch.from_numpy(np.ascontiguousarray(lab)).pin_memory()

        def e2e_once():
            h = gpm.Graph.from_edge_ptrs(n, len(s), hs.data_ptr(), hd.data_ptr(), hl.data_ptr())
            c = h.match(gpm.Query(k, e[:, 0], e[:, 1], ql))
            h.close()
            return c
        ms, c = event_ms(e2e_once, stream, 2)
        assert c == res["queries"][todo[0]]["embeddings"]
        res["e2e"] = {"value": c / (min(ms) / 1e3), "unit": "embeddings/s", "ms_per_step": min(ms),
                      "query": todo[0], "h2d_bytes_per_step": int(hs.numel() * 8 + hl.numel() * 4),
                      "d2h_bytes_per_step": 8}
    g.close()
    if not args.no_cpu:
        ceci = cpu_match_ceci(off, idx, lab, queries, num=5e7)
        res["cpu_baseline_queries"] = ceci
        ok = [v for kq, v in ceci.items() if isinstance(v, dict) and "embeddings_per_s" in v and kq in todo]
        if ok:
            e_, s_ = sum(v["embeddings"] for v in ok), sum(v["enumerate_s"] for v in ok)
            res["cpu_baseline"] = {"value": e_ / s_, "unit": "embeddings/s", "cores": 1, "kind": "reference",
                                   "sample": "sub_ceci (oracle/_ref/myceci, built from the reference's sources), "
                                             "each query stopped after 5e7 embeddings (-num), by its own "
                                             "'Enumerate time' line"}
    return res


def other_workloads(args, local):
    """The non-headline workloads at N = 1; a failing one is reported, not fatal."""
    import torch
    stream = torch.cuda.current_stream(torch.device("cuda", local))
    out = {}
    fns = {"clique": clique_workload, "motif": motif_workload, "match": match_workload}
    for name, fn in fns.items():
        if args.workload not in ("all", name):
            continue
        t0 = time.perf_counter()
        try:
            out[name] = fn(args, stream)
        except Exception as e:  # noqa: BLE001  (the headline line must still print)
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["wall_s"] = time.perf_counter() - t0
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        return reference_arm(args, rank, world, dist)
    import gpm  # noqa: F401  (fails loudly when libgpm.so is missing)

    torch.cuda.set_device(local)
    if args.workload in ("all", "tc"):
        line = tc_line(args, rank, world, dist, local)
        if world == 1 and args.workload == "all":
            line["workloads"] = other_workloads(args, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    elif rank == 0:
        print(json.dumps(other_workloads(args, local)), flush=True)
    if dist:
        dist.destroy_process_group()


# --------------------------------------------------------------------------- reference arm
def reference_gpu(off, idx, m_und, timeout=600):
    """The reference's own GPU triangle count of the same graph, for the
    record: its e-centric (test_engine) and v-centric (test_trianglecounting)
    drivers, compiled for sm_100a from its sources into oracle/_ref, each
    timed by its own kernel-window line "Triangle counting  time: X seconds"
    (src/TCSolver.cuh:26,61-63,108-113).  The reference's .mtx loader sizes
    the graph from the ids present, so isolated vertices are dropped first
    (an order-preserving renumbering: same orientation, same count)."""
    import _oracle as orc
    ref = os.path.join(ROOT, "oracle", "_ref")
    drivers = {"e_centric": ("test_engine", r"Result: (\d+)"),
               "v_centric": ("test_trianglecounting", r"Pattern 0: (\d+)")}
    if not all(os.path.exists(os.path.join(ref, d)) for d, _ in drivers.values()):
        return {"unavailable": "reference GPU drivers not built (make -C oracle refgpu where the reference is mounted)"}
    off2, idx2 = _compact_csr(off, idx)
    res = {"graph": f"{len(off2) - 1} non-isolated vertices, {m_und} edges"}
    with tempfile.TemporaryDirectory() as td:
        mtx, lab = os.path.join(td, "g.mtx"), os.path.join(td, "g.lab")
        orc.write_mtx(mtx, off2, idx2)
        with open(lab, "w") as f:
            f.write("".join(f"{v} 1\n" for v in range(1, len(off2))))
        for mode, (drv, pat) in drivers.items():
            argv = [os.path.join(ref, drv), mtx] + ([lab] if drv == "test_engine" else [])
            try:
                out = subprocess.run(argv, capture_output=True, text=True, timeout=timeout)
            except subprocess.TimeoutExpired:
                res[mode] = {"unavailable": f"no result within {timeout} s"}
                continue
            t = re.findall(r"Triangle counting\s+time:\s*([0-9.eE+-]+)\s*seconds", out.stdout)
            c = re.findall(pat, out.stdout)
            if out.returncode != 0 or not t or not c:
                res[mode] = {"unavailable": f"exit {out.returncode}, no time/result line"}
                continue
            sec = float(t[-1])
            res[mode] = {"ms": sec * 1e3, "triangles": int(c[-1]), "teps": m_und / sec}
    return res


def _compact_csr(off, idx):
    """Isolated vertices dropped by an order-preserving renumbering (the
    reference's .mtx loader sizes the graph from the ids present)."""
    import numpy as np
    deg = np.diff(off)
    live = np.nonzero(deg)[0]
    remap = np.full(len(deg), -1, np.int64)
    remap[live] = np.arange(len(live))
    off2 = np.zeros(len(live) + 1, np.int64)
    off2[1:] = np.cumsum(deg[live])
    return off2, remap[idx].astype(np.int32)


def reference_gpu_extra(names, timeout=900):
    """The reference's own GPU solvers on the other workloads (opt-in, one
    JSON line): k-cliques (CFSolver through oracle/ref_cf_driver.cu, whole
    call timed) on R-MAT scale 20, edge factor 16, seed 1, and 4-vertex
    motifs (G2MinerSolver / PatternSolver "Motif4", their own kernel-window
    lines, src/G2MinerSolver.cuh:110-163, src/PatternSolver.cuh:177-248) on
    R-MAT scale 18, edge factor 16, seed 1."""
    import _oracle as orc
    ref = os.path.join(ROOT, "oracle", "_ref")

    def run(argv):
        try:
            return subprocess.run(argv, capture_output=True, text=True, timeout=timeout).stdout
        except subprocess.TimeoutExpired:
            return ""

    res = {"impl": "reference", "extra": True}
    with tempfile.TemporaryDirectory() as td:
        if "clique" in names:
            n, s_, d_ = orc.gen_rmat(20, EF, A, B, C, seed=1)
            off, idx = _compact_csr(*orc.build_csr(n, s_, d_))
            mtx = os.path.join(td, "r20.mtx")
            orc.write_mtx(mtx, off, idx)
            for k in (4, 5):
                out = run([os.path.join(ref, "ref_cf"), mtx, str(k)])
                c = re.findall(r"Result: (\d+)", out)
                t = re.findall(r"CFSolver call time: ([0-9.eE+-]+) seconds", out)
                res[f"clique{k}_rmat20"] = ({"cliques": int(c[-1]), "s_call": float(t[-1])} if c and t
                                            else {"unavailable": "no result"})
        if "motif" in names:
            n, s_, d_ = orc.gen_rmat(18, EF, A, B, C, seed=1)
            off, idx = _compact_csr(*orc.build_csr(n, s_, d_))
            mtx = os.path.join(td, "r18.mtx")
            orc.write_mtx(mtx, off, idx)
            for fam, drv in (("g2miner", "test_G2Miner"), ("pattern_solver", "test_patternEnum")):
                out = run([os.path.join(ref, drv), mtx, "Motif4"])
                t = re.findall(r"matching\s+time:\s*([0-9.eE+-]+)\s*seconds", out)
                got = dict(re.findall(r"Result(\d): (\d+)", out))
                res[f"motif4_rmat18_{fam}"] = ({"s_kernel": float(t[-1]),
                                                "counts": [int(got[str(i)]) for i in range(6)]}
                                               if t and len(got) == 6 else {"unavailable": "no result"})
    return res


def reference_workloads(args):
    """The CPU reference of the other workloads on the host cores: the oracle
    port (cliques, motifs) and the reference's own sub_ceci (labelled)."""
    import numpy as np
    import _oracle as orc
    th = host_threads()
    out = {}
    if args.workload in ("all", "clique"):
        t0 = time.perf_counter()
        n, s, d = orc.gen_rmat(W.CLIQUE_SCALE, EF, A, B, C, seed=W.CLIQUE_SEED, threads=th)
        off, idx = orc.build_csr(n, s, d)
        doff, didx = orc.orient(off, idx)
        r = {"workload": f"clique_rmat{W.CLIQUE_SCALE}_ef{EF}", "unit": "cliques/s"}
        for k in (4, 5):
            v, smp = cpu_clique(doff, didx, k, args.cpu_seconds, th)
            r[f"k{k}"] = {"value": v, "cores": th, "kind": "port", "sample": smp}
        r["value"] = r["k4"]["value"]
        r["wall_s"] = time.perf_counter() - t0
        out["clique"] = r
    if args.workload in ("all", "motif"):
        t0 = time.perf_counter()
        nv, gam, md = W.batch_members()
        gen = lambda i: orc.gen_chung_lu(int(nv[i]), gam[i], md[i], seed=W.member_seed(i), threads=th)
        v, smp = cpu_motif_members(gen, [int(x) for x in nv], args.cpu_seconds, th)
        out["motif"] = {"workload": f"motif_batch_{len(nv)}_chunglu", "unit": "instances/s", "value": v,
                        "cores": th, "kind": "port", "sample": smp, "wall_s": time.perf_counter() - t0}
    if args.workload in ("all", "match"):
        t0 = time.perf_counter()
        n, s, d = orc.gen_rmat(W.MATCH_SCALE, EF, A, B, C, seed=W.MATCH_SEED, threads=th)
        lab = orc.gen_zipf_labels(n, W.MATCH_LABELS, W.MATCH_ZIPF, seed=W.MATCH_SEED, threads=th)
        off, idx = orc.build_csr(n, s, d)
        queries = W.walk_queries(off, idx, lab)
        ceci = cpu_match_ceci(off, idx, lab, queries, num=5e7)
        todo = [q for q in args.match_queries.split(",") if q in queries]
        ok = [v for kq, v in ceci.items() if isinstance(v, dict) and "embeddings_per_s" in v and kq in todo]
        val = sum(v["embeddings"] for v in ok) / sum(v["enumerate_s"] for v in ok) if ok else None
        out["match"] = {"workload": f"match_rmat{W.MATCH_SCALE}_ef{EF}_zipf{W.MATCH_LABELS}",
                        "unit": "embeddings/s", "value": val, "cores": 1, "kind": "reference",
                        "queries": ceci, "wall_s": time.perf_counter() - t0}
    return out


def reference_arm(args, rank, world, dist):
    """The reference has no CPU triangle counter of its own; its arm is the
    CPU restatement of its algorithm (oracle port) on all host threads, each
    step a vertex sample.  The graph comes from the oracle's restatement of
    the engine's seeded generator, so this process never loads the engine.
    Beside it, the reference's own GPU solvers on the same graph."""
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    import _oracle as orc
    threads = host_threads()
    n, s, d = orc.gen_rmat(args.scale, EF, A, B, C, seed=W.TC_SEED, threads=threads)
    off, idx = orc.build_csr(n, s, d)
    doff, didx = orc.orient(off, idx)
    m_und = len(didx)
    vals = []
    sample = ""
    warm = max(args.warmup, 3)
    per_step = min(args.cpu_seconds, 6.0, 60.0 / (warm + args.steps))
    for k in range(warm + args.steps):
        v, sample = cpu_tc(doff, didx, m_und, per_step, threads)
        if k >= warm:
            vals.append(v)
    value = statistics.median(vals)
    v1, sample1 = cpu_tc(doff, didx, m_und, args.cpu_seconds / 2, 1)
    line = {"metric": METRIC, "impl": "reference",
            "value": value, "unit": "TEPS", "n_gpus": world, "steps": args.steps, "warmup": warm,
            "ms_per_step": m_und / value * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": f"tc_rmat{args.scale}_ef{EF}", "graph": "R-MAT", "scale": args.scale,
                       "edge_factor": EF, "parallelism": "cpu"},
            "cpu_baseline": {"value": value, "unit": "TEPS", "cores": threads, "kind": "port", "sample": sample,
                             "one_core": {"value": v1, "cores": 1, "sample": sample1}},
            "e2e": {"value": value, "unit": "TEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_ref_gpu:
        line["reference_gpu"] = reference_gpu(off, idx, m_und)
    if world == 1 and args.workload == "all":
        line["workloads"] = reference_workloads(args)
    print(json.dumps(line), flush=True)
    if args.ref_extra:
        print(json.dumps(reference_gpu_extra(args.ref_extra.split(","))), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
