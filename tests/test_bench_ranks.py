"""The benchmark's multi-rank path on CPU: two gloo ranks, each with its own
per-step time and edge count, must agree on the whole-job figures (the slowest
rank's time, the sum of the edges), and a non-zero rank of the reference arm
must leave without work or output."""
import json
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, outdir):
    import datetime
    import io
    import contextlib
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [10.0, 12.5, 7.0, 11.0][rank]
    edges = [100, 300, 50, 7][rank]
    ms_max, e_sum = bench.over_ranks(dist, torch.device("cpu"), ms, edges)
    ms_e2e, _ = bench.over_ranks(dist, torch.device("cpu"), 2 * ms, edges)
    printed = io.StringIO()
    if rank != 0:
        with contextlib.redirect_stdout(printed):
            bench.reference_arm(None, rank, world, dist)
    else:
        dist.destroy_process_group()
    with open(os.path.join(outdir, f"r{rank}.json"), "w") as f:
        json.dump({"ms": ms_max, "edges": e_sum, "ms_e2e": ms_e2e, "printed": printed.getvalue()}, f)


@pytest.mark.parametrize("world", [2, 4])
def test_over_ranks_gloo(tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    ms = [10.0, 12.5, 7.0, 11.0][:world]
    edges = [100, 300, 50, 7][:world]
    for r in res:
        assert r["ms"] == max(ms)
        assert r["edges"] == sum(edges)
        assert r["ms_e2e"] == 2 * max(ms)
    assert all(r["printed"] == "" for r in res[1:])


def test_over_ranks_single():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.over_ranks(None, None, 3.5, 42) == (3.5, 42.0)


def test_reference_arm_never_loads_the_engine():
    # the reference arm times the reference's CPU implementation (the oracle
    # port, sub_ceci); its process must not map libgpm.so at all
    import subprocess
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'tc', '--scale', '12', "
            "'--steps', '1', '--warmup', '1', '--cpu-seconds', '0.2', '--no-ref-gpu']; sys.path.insert(0, '.'); "
            "import bench; bench.main(); "
            "print('MAPS', sum('libgpm' in l for l in open('/proc/self/maps')))")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["one_core"]["cores"] == 1
    assert lines[-1] == "MAPS 0"
