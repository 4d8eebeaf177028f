"""libgpm.so without a GPU: it loads, exports every declared entry point, its
host-only parts (readers, generators) work, and device entry points report an
error status instead of aborting when no device is present."""
import os
import re
import subprocess

import numpy as np
import pytest

import gpm
import _oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def declared_symbols():
    syms = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            syms |= set(re.findall(r"\b(gpm_[a-z0-9_]+)\s*\(", text))
    return syms


def test_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", gpm.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (gpm_[a-z0-9_]+)", out))
    missing = declared_symbols() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    assert len(declared_symbols()) >= 25


def test_abi_version():
    assert gpm.lib.gpm_abi_version() == 1


def test_read_mtx_follows_reference_loader(tmp_path):
    # comment lines skipped, header read, self-loop dropped, ids shifted by vmin
    p = tmp_path / "g.mtx"
    p.write_text("%%MatrixMarket\n% comment\n5 5 5\n3 4\n4 4\n5 3\n3 5\n6 7\n")
    n, src, dst, vmin = gpm.read_mtx(str(p))
    assert vmin == 3 and n == 5
    assert src.tolist() == [0, 2, 0, 3] and dst.tolist() == [1, 0, 2, 4]


def test_read_mtx_unterminated_last_line(tmp_path):
    p = tmp_path / "g.mtx"
    p.write_text("3 3 2\n1 2\n2 3")  # the reference's stream loop stops before "2 3"
    n, src, dst, _ = gpm.read_mtx(str(p))
    assert src.tolist() == [0]


def test_read_mtx_missing_file():
    with pytest.raises(gpm.GpmError) as e:
        gpm.read_mtx("/nonexistent/x.mtx")
    assert e.value.status == 6


def test_read_labels(tmp_path):
    p = tmp_path / "l.txt"
    p.write_text("1 5\n2 6\n3 7\n")
    assert gpm.read_labels(str(p), 3, 1).tolist() == [5, 6, 7]
    with pytest.raises(gpm.GpmError):
        gpm.read_labels(str(p), 4, 1)  # "vertex size not match"
    lab = gpm.read_labels("random4", 100, 0)
    assert lab.min() >= 0 and lab.max() < 4


def test_read_tve(tmp_path):
    p = tmp_path / "q.graph"
    p.write_text("t # 0\nv 0 3\nv 1 4\nv 2 5\ne 0 1 0\ne 1 2 0\n")
    n, src, dst, lab = gpm.read_tve(str(p))
    assert n == 3 and lab.tolist() == [3, 4, 5] and src.tolist() == [0, 1] and dst.tolist() == [1, 2]


def test_generators_deterministic():
    n, s1, d1 = gpm.gen_rmat(10, 4, seed=5)
    _, s2, d2 = gpm.gen_rmat(10, 4, seed=5)
    _, s3, _ = gpm.gen_rmat(10, 4, seed=6)
    assert (s1 == s2).all() and (d1 == d2).all() and not (s1 == s3).all()
    assert s1.min() >= 0 and s1.max() < n
    # R-MAT skew: vertex 0 quadrant gets the largest share
    assert np.bincount(s1, minlength=n)[0] == np.bincount(s1, minlength=n).max()
    n, s, d = gpm.gen_er(1000, 5000, seed=3)
    assert s.max() < 1000 and d.max() < 1000
    n, s, d = gpm.gen_chung_lu(5000, 2.3, 16.0, seed=2)
    off, idx = orc.build_csr(n, s, d)
    deg = np.diff(off)
    assert 10 < deg.mean() < 20 and deg.max() > 10 * deg.mean()
    lab = gpm.gen_zipf_labels(20000, 8, 1.2, seed=1)
    cnt = np.bincount(lab, minlength=8)
    assert (np.diff(cnt) < 0).all()


def test_device_calls_fail_cleanly_without_gpu():
    if gpm.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(gpm.GpmError) as e:
        gpm.Graph.from_edges(3, [0, 1], [1, 2])
    assert e.value.status == 7


def test_query_size_limit():
    """Query graphs of up to 64 vertices are accepted (sub_ceci's
    MAX_QUERY_VERTEX, sub_ceci/configuration/config.h:12); 65 is refused."""
    path = np.arange(63, dtype=np.int32)
    q = gpm.Query(64, path, path + 1, np.zeros(64, np.int32))
    q.close()
    with pytest.raises(gpm.GpmError) as e:
        gpm.Query(65, path, path + 1, np.zeros(65, np.int32))
    assert "64" in str(e.value)


def test_oracle_generators_match_the_engine():
    # bench.py's reference arm and the fixture scripts build their graphs with
    # the oracle's restated generators so that they never load the engine;
    # the edges must be the engine's own, draw for draw
    for scale, ef, seed in ((10, 16, 7), (15, 4, 1)):
        a, b = orc.gen_rmat(scale, ef, seed=seed), gpm.gen_rmat(scale, ef, seed=seed)
        assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    a, b = orc.gen_rmat(12, 8, 0.45, 0.15, 0.15, seed=3), gpm.gen_rmat(12, 8, 0.45, 0.15, 0.15, seed=3)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    a, b = orc.gen_er(5000, 40000, seed=3), gpm.gen_er(5000, 40000, seed=3)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    import workloads
    n, gam, md = workloads.batch_members()
    for m in (0, 111, 222):
        a = orc.gen_chung_lu(int(n[m]), gam[m], md[m], seed=workloads.member_seed(m))
        b = gpm.gen_chung_lu(int(n[m]), gam[m], md[m], seed=workloads.member_seed(m))
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    for s in (1.2, 0.7):
        assert np.array_equal(orc.gen_zipf_labels(100000, 8, s, seed=3), gpm.gen_zipf_labels(100000, 8, s, seed=3))


def test_oracle_tve_writer(tmp_path):
    n, s, d = orc.gen_rmat(8, 4, seed=2)
    off, idx = orc.build_csr(n, s, d)
    lab = orc.gen_zipf_labels(n, 3, 1.2, seed=2)
    path = tmp_path / "g.graph"
    orc.write_tve(path, off, idx, lab)
    n2, s2, d2, lab2 = gpm.read_tve(str(path))
    off2, idx2 = orc.build_csr(n2, s2, d2)
    assert n2 == n and np.array_equal(off2, off) and np.array_equal(idx2, idx) and np.array_equal(lab2, lab)
