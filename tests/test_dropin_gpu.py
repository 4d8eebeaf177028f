"""The C++ drop-in layer (antirf/antirf.h) through drivers that mirror the
reference's test/*.cu command lines."""
import os
import re
import subprocess

import numpy as np
import pytest

import _oracle as orc

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRV = os.path.join(ROOT, "gpm-artifact_b200", "drivers")
GOLD = os.path.join(ROOT, "tests", "golden")


def run(*args):
    out = subprocess.run([os.path.join(DRV, args[0]), *map(str, args[1:])], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    return out.stdout


def write_mtx(path, n, src, dst):
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern general\n")
        f.write(f"{n} {n} {len(src)}\n")
        for a, b in zip(src, dst):
            f.write(f"{a + 1} {b + 1}\n")


@pytest.fixture(scope="module")
def rmat_mtx(tmp_path_factory):
    import gpm
    n, s, d = gpm.gen_rmat(11, 8, seed=4)
    off, idx = orc.build_csr(n, s, d)
    src = np.repeat(np.arange(n), np.diff(off))
    p = tmp_path_factory.mktemp("g") / "rmat.mtx"
    write_mtx(p, n, src, idx)  # both directions, as datasets/simple.mtx lists them
    # vertex ids in the file start at 1; the loader shifts by the smallest id seen
    used = np.unique(np.concatenate([src, idx]))
    return str(p), off, idx, used


def test_simple_mtx_drivers(tmp_path):
    z = np.load(os.path.join(GOLD, "ref_small.npz"))
    e = z["simple_mtx"]
    p = tmp_path / "simple.mtx"
    write_mtx(p, 4, e[:, 0], e[:, 1])
    lab = tmp_path / "vlabel.txt"
    lab.write_text("1 1\n2 1\n3 1\n4 1\n")
    assert "Pattern 0: 0" in run("test_trianglecounting", p)
    assert "Result: 0" in run("test_engine", p, lab)
    out = run("test_G2Miner", p, "Motif4")
    assert [int(x) for x in re.findall(r"Result\d: (\d+)", out)] == [0, 1, 0, 0, 0, 0]
    assert "Result: 1" in run("test_G2Miner", p, "P4")


def test_rmat_drivers_against_oracle(rmat_mtx):
    path, off, idx, used = rmat_mtx
    assert used.min() == 0  # vertex 0 present, so no id shift
    doff, didx = orc.orient(off, idx)
    tri = orc.tc(doff, didx)
    assert f"Pattern 0: {tri}" in run("test_trianglecounting", path)
    assert f"Result: {orc.clique(doff, didx, 4)}" in run("test_cf", path, 4)
    m4 = orc.motif4(off, idx)
    for drv in ("test_G2Miner", "test_patternEnum"):
        out = run(drv, path, "Motif4")
        assert [int(x) for x in re.findall(r"Result\d: (\d+)", out)] == m4.tolist()
    assert f"Result: {orc.pattern_g2miner(off, idx, 7)}" in run("test_patternEnum", path, "P7")


def test_match_driver_hprd(tmp_path):
    z = np.load(os.path.join(GOLD, "hprd_kat.npz"))
    off, idx, lab = z["off"], z["idx"], z["labels"]
    n = len(off) - 1
    deg = np.diff(off)
    dpath = tmp_path / "hprd.graph"
    src = np.repeat(np.arange(n), deg)
    with open(dpath, "w") as f:
        f.write(f"t {n} {len(idx) // 2}\n")
        f.writelines(f"v {v} {lab[v]} {deg[v]}\n" for v in range(n))
        f.writelines(f"e {a} {b}\n" for a, b in zip(src, idx) if a < b)
    po = pi = pl = 0
    for i, m in enumerate(z["qn"][:20]):
        qo = z["qoff"][po: po + m + 1]
        po += m + 1
        qi = z["qidx"][pi: pi + qo[-1]]
        pi += qo[-1]
        ql = z["qlab"][pl: pl + m]
        pl += m
        qpath = tmp_path / f"q{i}.graph"
        qs = np.repeat(np.arange(m), np.diff(qo))
        with open(qpath, "w") as f:
            f.write(f"t {m} {len(qi) // 2}\n")
            f.writelines(f"v {v} {ql[v]} {qo[v + 1] - qo[v]}\n" for v in range(m))
            f.writelines(f"e {a} {b}\n" for a, b in zip(qs, qi) if a < b)
        assert f"#Embeddings: {int(z['expected'][i])}" in run("test_match", "-d", dpath, "-q", qpath)


def test_engine_driver_reads_binary_csr(rmat_mtx, tmp_path):
    """Loader::Load(path, "bin"): the graph written as a binary CSR (the
    gbin_reader layout) gives the same count as the .mtx of the same graph."""
    import gpm
    path, off, idx, used = rmat_mtx
    lab = "random2"  # labels are loaded and unused; the two loads size the graph differently
    pre = str(tmp_path / "bin")
    gpm.write_gbin(pre, off, idx)
    tri = orc.tc(*orc.orient(off, idx))
    assert f"Result: {tri}" in run("test_engine", path, lab)
    assert f"Result: {tri}" in run("test_engine", pre, lab)
