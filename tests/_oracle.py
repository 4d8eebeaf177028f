"""ctypes binding of oracle/liboracle.so -- the CPU checker (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use it.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_int, c_int64, c_uint64, c_void_p

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise ImportError(f"{ORACLE_SO} missing: run `make -C {os.path.dirname(ORACLE_SO)}`")
        L = ctypes.CDLL(ORACLE_SO)
        for f in ("orc_tc", "orc_tc_tasks", "orc_tc_merge", "orc_clique", "orc_clique_tasks", "orc_pattern_g2miner", "orc_pattern_solver", "orc_match"):
            getattr(L, f).restype = c_uint64
        L.orc_build_csr.restype = c_int64
        L.orc_orient.restype = c_int64
        L.orc_write_mtx.restype = c_int64
        L.orc_tc_weighted.restype = c_uint64
        L.orc_write_tve.restype = c_int64
        L.orc_gen_chung_lu.restype = c_int64
        for f in ("orc_gen_rmat", "orc_gen_er", "orc_gen_zipf_labels"):
            getattr(L, f).restype = None
        _lib = L
    return _lib


def _p(a):
    return c_void_p(a.ctypes.data)


def build_csr(n, src, dst, symmetrize=True):
    s0 = np.ascontiguousarray(src, np.int32)
    s1 = np.ascontiguousarray(dst, np.int32)
    off = np.zeros(n + 1, np.int64)
    idx = np.zeros(2 * len(s0) + 1, np.int32)
    m = lib().orc_build_csr(c_int64(n), c_int64(len(s0)), _p(s0), _p(s1), 1 if symmetrize else 0, _p(off),
                            _p(idx), c_int64(len(idx)))
    assert m >= 0
    return off, idx[:m].copy()


def orient(off, idx):
    n = len(off) - 1
    off = np.ascontiguousarray(off, np.int64)
    idx = np.ascontiguousarray(idx, np.int32)
    doff = np.zeros(n + 1, np.int64)
    didx = np.zeros(len(idx) + 1, np.int32)
    m = lib().orc_orient(c_int64(n), _p(off), _p(idx), _p(doff), _p(didx))
    return doff, didx[:m].copy()


def tc(doff, didx, threads=0):
    return lib().orc_tc(c_int64(len(doff) - 1), _p(doff), _p(didx), c_int(threads))


def tc_tasks(doff, didx, keep, threads=0):
    keep = np.ascontiguousarray(keep, np.uint8)
    return lib().orc_tc_tasks(c_int64(len(doff) - 1), _p(doff), _p(didx), _p(keep), c_int(threads))


def tc_merge(doff, didx):
    return lib().orc_tc_merge(c_int64(len(doff) - 1), _p(doff), _p(didx))


def clique(doff, didx, k, threads=0):
    return lib().orc_clique(c_int64(len(doff) - 1), _p(doff), _p(didx), c_int(k), c_int(threads))


def clique_tasks(doff, didx, k, keep, threads=0):
    keep = np.ascontiguousarray(keep, np.uint8)
    return lib().orc_clique_tasks(c_int64(len(doff) - 1), _p(doff), _p(didx), c_int(k), _p(keep), c_int(threads))


def motif4_tasks(off, idx, keep, threads=0):
    keep = np.ascontiguousarray(keep, np.uint8)
    out = (c_uint64 * 6)()
    lib().orc_motif4_tasks(c_int64(len(off) - 1), _p(off), _p(idx), _p(keep), out, c_int(threads))
    return np.array(list(out), np.uint64)


def motif4(off, idx, threads=0):
    out = (c_uint64 * 6)()
    lib().orc_motif4_g2miner(c_int64(len(off) - 1), _p(off), _p(idx), out, c_int(threads))
    return np.array(list(out), np.uint64)


def bruteforce(off, idx):
    out = (c_uint64 * 8)()
    lib().orc_motif_bruteforce(c_int64(len(off) - 1), _p(off), _p(idx), out)
    return np.array(list(out), np.uint64)


def pattern_g2miner(off, idx, p, threads=0):
    return lib().orc_pattern_g2miner(c_int64(len(off) - 1), _p(off), _p(idx), c_int(p), c_int(threads))


def pattern_solver(off, idx, p, threads=0):
    out = (c_uint64 * 6)()
    r = lib().orc_pattern_solver(c_int64(len(off) - 1), _p(off), _p(idx), c_int(p), out, c_int(threads))
    return r, np.array(list(out), np.uint64)


def match(off, idx, labels, qoff, qidx, qlabels, threads=0):
    labels = np.ascontiguousarray(labels, np.int32)
    qlabels = np.ascontiguousarray(qlabels, np.int32)
    return lib().orc_match(c_int64(len(off) - 1), _p(off), _p(idx), _p(labels), c_int64(len(qoff) - 1), _p(qoff),
                           _p(qidx), _p(qlabels), c_int(threads))


def motif3(off, idx, tri):
    """3-vertex motifs: induced 2-paths = sum C(d,2) - 3T, triangles."""
    d = np.diff(off).astype(np.uint64)
    wedges = int(np.sum(d * (d - np.uint64(1)) // np.uint64(2))) if len(d) else 0
    return np.array([wedges - 3 * tri, tri], np.uint64)


def write_mtx(path, off, idx):
    """The CSR as 1-indexed Matrix Market text for the reference's loader."""
    off = np.ascontiguousarray(off, np.int64)
    idx = np.ascontiguousarray(idx, np.int32)
    r = lib().orc_write_mtx(str(path).encode(), c_int64(len(off) - 1), _p(off), _p(idx))
    if r < 0:
        raise OSError(f"writing {path} failed")
    return r


def tc_weighted(doff, didx, wt, threads=0):
    """Sum over DAG triangles u -> v -> w of wt[w]."""
    wt = np.ascontiguousarray(wt, np.int64)
    return lib().orc_tc_weighted(c_int64(len(doff) - 1), _p(doff), _p(didx), _p(wt), c_int(threads))


def c4_two_hubs(off, idx, h0, h1):
    """Non-induced 4-cycles of a graph whose only high-degree vertices are two
    non-adjacent hubs h0, h1, without enumerating the hubs' neighbour pairs:
    cycles avoiding both hubs (sum over vertex pairs of C(common, 2) / 2 from
    the sparse square of the rest), cycles through one hub h (its opposite
    vertex y has C(|N(y) & N(h)|, 2) of them) and cycles through both (pairs
    of their common neighbours).  Test infrastructure only."""
    import scipy.sparse as sp
    n = len(off) - 1
    src = np.repeat(np.arange(n), np.diff(off))
    assert not np.any((src == h0) & (idx == h1)), "hubs must not be adjacent"
    rest = (src != h0) & (src != h1) & (idx != h0) & (idx != h1)
    A = sp.csr_matrix((np.ones(int(rest.sum()), np.int64), (src[rest], idx[rest])), shape=(n, n))
    P = sp.triu(A @ A, k=1).tocoo()
    c = P.data.astype(np.int64)
    total = int((c * (c - 1) // 2).sum()) // 2
    sets = []
    for h in (h0, h1):
        nb = idx[off[h]:off[h + 1]]
        ind = np.zeros(n, np.int64)
        ind[nb] = 1
        t = A @ ind
        total += int((t * (t - 1) // 2).sum())
        sets.append(nb)
    k = len(np.intersect1d(sets[0], sets[1]))
    return total + k * (k - 1) // 2


def two_hub_graph(n, m_rand, d0, d1, mids, seed):
    """Random sparse graph on [2, n) with `mids` medium hubs (list of degrees,
    vertices 2, 3, ...) and two non-adjacent hubs 0 and 1 of degrees d0, d1."""
    rng = np.random.default_rng(seed)
    e = rng.integers(2, n, size=(m_rand, 2))
    parts = [e]
    for i, dm in enumerate(mids):
        parts.append(np.stack([np.full(dm, 2 + i), rng.integers(2, n, size=dm)], 1))
    for h, dh in ((0, d0), (1, d1)):
        nb = rng.choice(np.arange(2, n), size=dh, replace=False)
        parts.append(np.stack([np.full(dh, h), nb], 1))
    e = np.concatenate(parts).astype(np.int32)
    return build_csr(n, e[:, 0], e[:, 1])


def gen_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, threads=0):
    """The engine's seeded R-MAT draws, restated in the oracle (same edges as
    gpm.gen_rmat without loading the engine)."""
    m = (1 << scale) * edge_factor
    src = np.empty(m, np.int32)
    dst = np.empty(m, np.int32)
    lib().orc_gen_rmat(c_int(scale), c_int64(m), ctypes.c_double(a), ctypes.c_double(b), ctypes.c_double(c),
                       c_uint64(seed), _p(src), _p(dst), c_int(threads))
    return 1 << scale, src, dst


def gen_er(n, m, seed=1, threads=0):
    src = np.empty(m, np.int32)
    dst = np.empty(m, np.int32)
    lib().orc_gen_er(c_int64(n), c_int64(m), c_uint64(seed), _p(src), _p(dst), c_int(threads))
    return n, src, dst


def gen_chung_lu(n, gamma, mean_deg, seed=1, threads=0):
    m = lib().orc_gen_chung_lu(c_int64(n), ctypes.c_double(gamma), ctypes.c_double(mean_deg), c_uint64(seed), None,
                               None, c_int(threads))
    src = np.empty(m, np.int32)
    dst = np.empty(m, np.int32)
    lib().orc_gen_chung_lu(c_int64(n), ctypes.c_double(gamma), ctypes.c_double(mean_deg), c_uint64(seed), _p(src),
                           _p(dst), c_int(threads))
    return n, src, dst


def gen_zipf_labels(n, nlabels, s=1.2, seed=1, threads=0):
    lab = np.empty(n, np.int32)
    lib().orc_gen_zipf_labels(c_int64(n), c_int(nlabels), ctypes.c_double(s), c_uint64(seed), _p(lab),
                              c_int(threads))
    return lab


def write_tve(path, off, idx, labels):
    """Symmetric labelled CSR as sub_ceci's t/v/e text."""
    off = np.ascontiguousarray(off, np.int64)
    idx = np.ascontiguousarray(idx, np.int32)
    labels = np.ascontiguousarray(labels, np.int32)
    r = lib().orc_write_tve(str(path).encode(), c_int64(len(off) - 1), _p(off), _p(idx), _p(labels))
    if r < 0:
        raise OSError(f"writing {path} failed")
    return r
