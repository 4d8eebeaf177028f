"""File formats on the host: the .mtx reader against a plain-Python
restatement of the reference loader's token stream (src/graph/io.h:84-139),
on crafted files that exercise every rule and on a large file (the parallel
line path), and the binary CSR layout of scripts/gbin_reader (reader, writer,
converter) against golden output of the reference's own converter."""
import os

import numpy as np
import pytest

import gpm
import _oracle as orc

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def mtx_reference(text):
    """Loader::_load_mtx restated: comment lines skipped until one starts
    with a digit; three header integers; then integers read in pairs with
    any whitespace between them, the rest of the second one's line ignored,
    a pair whose line has no newline dropped, self-loops dropped; reading
    stops at a token that is not an int32; ids shifted by the minimum."""
    lines = text.split("\n")
    pos = 0
    while pos < len(text) and not text[pos].isdigit():
        nl = text.find("\n", pos)
        pos = len(text) if nl < 0 else nl + 1
    ws = " \t\n\r\v\f"

    def token(p):
        while p < len(text) and text[p] in ws:
            p += 1
        q = p
        if q < len(text) and text[q] in "+-":
            q += 1
        r = q
        while r < len(text) and text[r].isdigit():
            r += 1
        if r == q:
            return None, p
        v = int(text[p:r])
        if not -2**31 <= v < 2**31:
            return None, p
        return v, r

    for _ in range(3):
        v, pos = token(pos)
        assert v is not None, "bad header"
    edges = []
    while True:
        a, pos = token(pos)
        if a is None:
            break
        b, pos = token(pos)
        if b is None:
            break
        nl = text.find("\n", pos)
        if nl < 0:
            break
        pos = nl + 1
        if a != b:
            edges.append((a, b))
    if not edges:
        return 0, np.zeros(0, np.int32), np.zeros(0, np.int32), 0
    e = np.array(edges, np.int64)
    vmin, vmax = e.min(), e.max()
    return int(vmax - vmin + 1), (e[:, 0] - vmin).astype(np.int32), (e[:, 1] - vmin).astype(np.int32), int(vmin)


CASES = {
    "plain": "4 4 3\n1 2\n2 3\n3 4\n",
    "comments": "%%MatrixMarket matrix coordinate pattern general\n% a comment\n%\n5 5 4\n1 2\n2 3\n3 1\n4 5\n",
    "weighted": "3 3 3\n1 2 0.5\n2 3 7\n3 1 -1e3\n",
    "self_loops": "3 3 4\n1 1\n1 2\n2 2\n2 3\n",
    "unterminated": "3 3 2\n1 2\n2 3",
    "blank_lines": "3 3 2\n1 2\n\n\n2 3\n",
    "pair_across_lines": "4 4 2\n1\n2 9 9\n3 4\n",
    "after_header": "4 4 2 1 2\n3 4\n",
    "stops_at_text": "5 5 3\n1 2\nfoo bar\n3 4\n",
    "signs_and_zero": "4 4 3\n0 +2\n-1 3\n2 -1\n",
    "tabs_crlf": "3 3 2\r\n1\t2\r\n2 3\r\n",
    "empty": "0 0 0\n",
    "too_big": "3 3 2\n1 2\n1 99999999999\n2 3\n",
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_mtx_reader_follows_the_loader(tmp_path, case):
    p = tmp_path / f"{case}.mtx"
    p.write_text(CASES[case])
    n, s, d, vmin = gpm.read_mtx(str(p))
    rn, rs, rd, rvmin = mtx_reference(CASES[case])
    assert n == rn and vmin == rvmin
    assert s.tolist() == rs.tolist() and d.tolist() == rd.tolist()


def test_mtx_reader_large_file_parallel_path(tmp_path):
    """A multi-megabyte file goes through the line-parallel path; it must
    give exactly the sequential restatement's edges, in file order."""
    rng = np.random.default_rng(4)
    e = rng.integers(1, 50000, size=(300000, 2))
    body = "".join(f"{a} {b}\n" for a, b in e)
    text = "% big\n50000 50000 300000\n" + body + "7 8"  # unterminated tail
    p = tmp_path / "big.mtx"
    p.write_text(text)
    n, s, d, vmin = gpm.read_mtx(str(p))
    rn, rs, rd, rvmin = mtx_reference(text)
    assert (n, vmin) == (rn, rvmin)
    assert np.array_equal(s, rs) and np.array_equal(d, rd)


def test_mtx_round_trip_through_the_oracle_writer(tmp_path):
    n, s, d = gpm.gen_rmat(12, 8, seed=3)
    off, idx = orc.build_csr(n, s, d)
    p = tmp_path / "g.mtx"
    orc.write_mtx(str(p), off, idx)
    n2, s2, d2, vmin = gpm.read_mtx(str(p))
    deg = np.diff(off)
    live = np.nonzero(deg)[0]
    lo = live.min()  # 1-indexed in the file: the reader shifts by lo + 1
    assert vmin == lo + 1 and n2 == live.max() - lo + 1
    assert np.array_equal(s2, np.repeat(np.arange(n), deg) - lo) and np.array_equal(d2, idx - lo)


def test_gbin_round_trip(tmp_path):
    n, s, d = gpm.gen_rmat(11, 8, seed=5)
    off, idx = orc.build_csr(n, s, d)
    pre = str(tmp_path / "bin")
    gpm.write_gbin(pre, off, idx)
    off2, idx2, md = gpm.read_gbin(pre)
    assert np.array_equal(off, off2) and np.array_equal(idx, idx2) and md == np.diff(off).max()
    meta = open(os.path.join(pre, "graph.meta.txt")).read().split()
    assert meta == [str(n), str(len(idx)), "4", str(int(np.diff(off).max()))]


def test_gbin_rejects_inconsistent_files(tmp_path):
    pre = str(tmp_path / "bad")
    gpm.write_gbin(pre, np.array([0, 1, 2], np.int64), np.array([1, 0], np.int32))
    with open(os.path.join(pre, "graph.edge.bin"), "ab") as f:
        f.write(b"\0\0\0\0")
    with pytest.raises(gpm.GpmError):
        gpm.read_gbin(pre)
    gpm.write_gbin(pre, np.array([0, 1, 2], np.int64), np.array([1, 7], np.int32))
    with pytest.raises(gpm.GpmError):
        gpm.read_gbin(pre)


def test_converter_matches_the_reference_converter(tmp_path):
    """Golden files written by the reference's own converter (built from
    scripts/gbin_reader/greader.cpp, see golden/make_gbin_golden.py)."""
    g = np.load(os.path.join(GOLD, "gbin_golden.npz"))
    for i, text in enumerate(g["inputs"]):
        p = tmp_path / f"c{i}.mtx"
        p.write_text(str(text))
        pre = str(tmp_path / f"c{i}")
        gpm.convert_mtx_gbin(str(p), pre)
        off, idx, md = gpm.read_gbin(pre)
        assert off.tolist() == g[f"off{i}"].tolist(), i
        assert idx.tolist() == g[f"idx{i}"].tolist(), i
        assert open(os.path.join(pre, "graph.meta.txt")).read() == str(g["meta"][i]), i
