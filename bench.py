"""Headline benchmark: exact triangle counting on an R-MAT scale-22 graph.

Workload (one step = one triangle count of the whole graph):
  R-MAT scale 22 (4,194,304 vertices), edge factor 16, (a,b,c,d) =
  (0.57, 0.19, 0.19, 0.05), seeded (seed = 1 + rank), symmetrised, self-loops
  and duplicates removed, int32 CSR with sorted lists, degree-oriented DAG
  (ties by id).  Output: exact uint64 triangle count.
Metric: TEPS = undirected edges / seconds per count (higher is better).

  value    device-resident DAG in HBM, the count kernel(s) timed with CUDA
           events on the launching stream (inputs 0.3 GB > 126 MB L2, so no
           flush is needed between steps).
  e2e      the same count through the C ABI from pinned HOST memory
           (gpm_tc_host_csr: H2D of the symmetric CSR, orientation on the
           device, count, D2H of the 8-byte result) -- all inside the timed
           region.
  roofline the count kernel against the measured HBM copy bandwidth, with
           the algorithmic bytes B = 4(n+1) + 4m + 4*sum_{u->v} deg+(v).
  cpu_baseline / --impl reference: the CPU restatement (OpenMP, all host
           threads) timed on a bounded vertex sample of the same graph.

Multi-GPU (torchrun): each rank counts its own independently seeded graph;
no data-path collective (weak scaling); the timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpm-artifact_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

SCALE, EF = 22, 16
A, B, C = 0.57, 0.19, 0.19


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100, help="timed counts (100 x ~7 ms: long enough to sample clocks)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=SCALE, help="R-MAT scale (22 is the headline workload)")
    ap.add_argument("--variant", default="auto",
                    choices=["auto", "bitmap", "hash", "bsearch", "merge", "learned"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true", help="reference arm: skip the reference's GPU solvers")
    ap.add_argument("--ref-extra", default="", help="reference arm: also time the reference's GPU solvers on "
                    "'clique' (R-MAT 20, k = 4, 5) and/or 'motif' (R-MAT 18, Motif4); one more JSON line")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU sample time")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler for the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
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


def cpu_sample(doff, didx, m_und, seconds, threads):
    """Times the CPU restatement (OpenMP marker algorithm) on the tasks of a
    vertex sample sized for about `seconds`, and scales to the whole graph by
    the sample's share of the algorithmic work."""
    import numpy as np
    import _oracle as orc
    n = len(doff) - 1
    deg = np.diff(doff)
    wv = np.zeros(n, np.float64)  # w(u) = d+(u) + sum_{v in N+(u)} d+(v)
    np.add.at(wv, np.repeat(np.arange(n), deg), deg[didx].astype(np.float64))
    wv += deg
    total = wv.sum()

    def run(stride):
        keep = np.zeros(n, np.uint8)
        keep[::stride] = 1
        frac = wv[keep.astype(bool)].sum() / total
        t0 = time.perf_counter()
        orc.tc_tasks(doff, didx, keep, threads)
        return time.perf_counter() - t0, frac

    stride = 256
    t, frac = run(stride)
    while t < seconds / 3 and stride > 1:
        stride = max(1, int(stride * max(0.05, t / seconds)))
        t, frac = run(stride)
    est_full = t / max(frac, 1e-12)
    return m_und / est_full, (f"tasks of every {stride}-th vertex ({frac * 100:.2f}% of the wedge work) "
                              f"in {t:.2f} s, scaled to the whole graph")


def profiled_traffic(scale, variant):
    """DRAM bytes per launch of the count kernel from the committed ncu
    summary of this workload (profiles/k_tc_rank_rmat22.md), else None."""
    if scale != SCALE or variant not in ("learned", "bitmap", "auto"):
        return None
    path = os.path.join(ROOT, "profiles", "k_tc_rank_rmat22.md")
    if not os.path.exists(path):
        return None
    key = f"traffic_bytes_per_launch[{'learned' if variant == 'learned' else 'bitmap'}]:"
    for line in open(path):
        if line.strip().startswith(key):
            return int(line.split(":")[1].strip())
    return None


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


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import numpy as np
    import torch

    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        return reference_arm(args, rank, world, dist)
    import gpm

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    seed = 1 + rank
    g = gpm.Graph.rmat(args.scale, EF, A, B, C, seed=seed)
    sym_off, sym_idx = g.csr()
    g.orient()
    inf = g.info()
    n, m_und = inf.n, inf.nnz
    wedge, pair = g.work()
    bytes_alg = 4 * (n + 1) + 4 * m_und + 4 * wedge
    # what this kernel streams: the clipped segments (4 B a key, a 16-byte
    # descriptor each) and every owner list once, plus per owner 36 B of
    # offsets and counts
    nseg, seg_keys, owner_keys, ntasks = g.plan_stats()
    bytes_kernel = 4 * seg_keys + 16 * nseg + 4 * owner_keys + 36 * ntasks
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

    for _ in range(max(args.warmup, 3)):
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

    # ---- the other schedules on the same graph (outside the timed region)
    others = {}
    for name in ("bitmap", "learned", "hash"):
        if name == args.variant or (name == "bitmap" and args.variant == "auto"):
            continue
        v = variants[name]
        g.tc_async(v, sp, out.data_ptr())
        torch.cuda.synchronize()
        assert int(out.item()) == count, name
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            g.tc_async(v, sp, out.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        others[name] = round(e0.elapsed_time(e1) / 3, 3)
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
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(ks):
            gpm.tc_host_csr_ptrs(nn, hoff.data_ptr(), hidx.data_ptr(), variant, sp)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_e2e, _ = over_ranks(dist, dev, e0.elapsed_time(e1) / ks, m_und)
        e2e = {"value": m_total / (ms_e2e / 1e3), "unit": "TEPS", "ms_per_step": ms_e2e,
               "h2d_bytes_per_step": int(hoff.numel() * 8 + hidx.numel() * 4), "d2h_bytes_per_step": 8}

    # ---- CPU baseline (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        doff, didx = g.csr()
        threads = len(os.sched_getaffinity(0))
        v_cpu, sample = cpu_sample(doff, didx, m_und, args.cpu_seconds, threads)
        cpu = {"value": v_cpu, "unit": "TEPS", "cores": threads, "kind": "port", "sample": sample}

    hbm, peak_kind = peaks()
    avg_kernel_ms = sum(per) / len(per)
    achieved = bytes_alg / (avg_kernel_ms / 1e3) / 1e9
    traffic = profiled_traffic(args.scale, args.variant)
    if rank == 0:
        line = {
            "metric": "triangle-count TEPS (R-MAT scale 22, exact uint64)",
            "value": value, "unit": "TEPS", "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic",
            "config": {"workload": f"tc_rmat{args.scale}_ef{EF}", "graph": "R-MAT", "scale": args.scale,
                       "edge_factor": EF, "abcd": [A, B, C, round(1 - A - B - C, 2)], "seed": "1+rank",
                       "n": n, "m_undirected": m_und, "dag_max_outdeg": inf.max_degree,
                       "triangles": count, "variant": args.variant, "parallelism": f"replicas{world}",
                       "l2": "inputs > L2 (DAG %.0f MB), no flush" % ((8 * (n + 1) + 4 * m_und) / 1e6),
                       "ms_per_count_by_schedule": others},
            "e2e": e2e,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes": bytes_alg, "kernel_ms": avg_kernel_ms,
                         # B_TC counts the vertex-iterator's reads (every wedge list in
                         # full); this kernel streams only the clipped smaller side:
                         "kernel_bytes": bytes_kernel,
                         "kernel_bytes_gbs": bytes_kernel / (avg_kernel_ms / 1e3) / 1e9,
                         "kernel_bytes_frac": bytes_kernel / (avg_kernel_ms / 1e3) / 1e9 / hbm,
                         "dram_gbs": traffic / (avg_kernel_ms / 1e3) / 1e9 if traffic else None,
                         "plan": {"segments": nseg, "segment_keys": seg_keys, "owner_keys": owner_keys,
                                  "owner_tasks": ntasks}},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            # one count kernel per step (k_tc_rank, or k_tc_hash / k_tc_bsearch / k_tc_merge)
            "gpu_launches": args.steps,
        }
        print(json.dumps(line), flush=True)
    g.close()
    if dist:
        dist.destroy_process_group()


def reference_gpu(off, idx, m_und, timeout=600):
    """The reference's own GPU triangle count of the same graph, for the
    record: its e-centric (test_engine) and v-centric (test_trianglecounting)
    drivers, compiled for sm_100a from its sources into oracle/_ref, each
    timed by its own kernel-window line "Triangle counting  time: X seconds"
    (src/TCSolver.cuh:26,61-63,108-113).  The reference's .mtx loader sizes
    the graph from the ids present, so isolated vertices are dropped first
    (an order-preserving renumbering: same orientation, same count)."""
    import re
    import tempfile
    import numpy as np
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
    import re
    import tempfile
    import gpm
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
            n, s_, d_ = gpm.gen_rmat(20, EF, A, B, C, seed=1)
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
            n, s_, d_ = gpm.gen_rmat(18, EF, A, B, C, seed=1)
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


def reference_arm(args, rank, world, dist):
    """The reference has no CPU triangle counter of its own; its arm is the
    CPU restatement of its algorithm (oracle port) on all host threads.  Each
    step is a vertex sample sized so that all steps take about 90 s.  Beside
    it, the reference's own GPU solvers on the same graph (reference_gpu)."""
    import numpy as np
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    import gpm
    import _oracle as orc
    n, s, d = gpm.gen_rmat(args.scale, EF, A, B, C, seed=1)
    off, idx = orc.build_csr(n, s, d)
    doff, didx = orc.orient(off, idx)
    m_und = len(didx)
    threads = len(os.sched_getaffinity(0))
    vals = []
    sample = ""
    per_step = min(args.cpu_seconds, 8.0, 90.0 / (max(args.warmup, 3) + args.steps))
    for k in range(max(args.warmup, 3) + args.steps):
        v, sample = cpu_sample(doff, didx, m_und, per_step, threads)
        if k >= max(args.warmup, 3):
            vals.append(v)
    value = statistics.median(vals)
    line = {"metric": "triangle-count TEPS (R-MAT scale 22, exact uint64)", "impl": "reference",
            "value": value, "unit": "TEPS", "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": m_und / value * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": f"tc_rmat{args.scale}_ef{EF}", "graph": "R-MAT", "scale": args.scale,
                       "edge_factor": EF, "parallelism": "cpu"},
            "cpu_baseline": {"value": value, "unit": "TEPS", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "TEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_ref_gpu:
        line["reference_gpu"] = reference_gpu(off, idx, m_und)
    print(json.dumps(line), flush=True)
    if args.ref_extra:
        print(json.dumps(reference_gpu_extra(args.ref_extra.split(","))), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
