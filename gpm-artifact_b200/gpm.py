"""ctypes binding of libgpm.so (the C ABI declared in include/gpm.h).

Tests and bench.py call the engine through this module, i.e. through the
same extern "C" boundary a C, C++ or FFI caller uses.  Loading fails loudly
when libgpm.so has not been built: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GPM_LIB") or os.path.join(HERE, "libgpm.so")  # GPM_LIB: another build of it

GPM_OK = 0
STATUS = {0: "GPM_OK", 1: "GPM_EINVAL", 2: "GPM_ECUDA", 3: "GPM_ENOMEM", 4: "GPM_EUNSUPPORTED",
          5: "GPM_ETIMEOUT", 6: "GPM_EIO", 7: "GPM_ENODEV"}
V_CENTRIC, E_CENTRIC = 0, 1
TC_AUTO, TC_BSEARCH, TC_HASH, TC_MERGE, TC_LEARNED, TC_BITMAP = 0, 1, 2, 3, 4, 5
G2MINER, PATTERN_SOLVER = 0, 1
SYMMETRIZE = 1


class GpmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` "
                          "(or __graft_entry__.build()); the engine has no CPU fallback")
    return ctypes.CDLL(LIB_PATH)


lib = _load()
_P = c_void_p
_SIGS = {
    "gpm_last_error": ([], c_char_p),
    "gpm_abi_version": ([], c_int),
    "gpm_device_count": ([POINTER(c_int)], c_int),
    "gpm_read_mtx": ([c_char_p, POINTER(c_int64), POINTER(c_int64), _P, _P, c_int64, POINTER(c_int32)], c_int),
    "gpm_read_labels": ([c_char_p, c_int64, c_int32, _P], c_int),
    "gpm_read_tve": ([c_char_p, POINTER(c_int64), POINTER(c_int64), _P, _P, _P, c_int64], c_int),
    "gpm_read_gbin": ([c_char_p, POINTER(c_int64), POINTER(c_int64), _P, _P, POINTER(c_int32)], c_int),
    "gpm_write_gbin": ([c_char_p, c_int64, _P, _P], c_int),
    "gpm_convert_mtx_gbin": ([c_char_p, c_char_p], c_int),
    "gpm_gen_rmat": ([c_int, c_int, c_double, c_double, c_double, c_uint64, _P, _P], c_int),
    "gpm_gen_er": ([c_int64, c_int64, c_uint64, _P, _P], c_int),
    "gpm_gen_chung_lu": ([c_int64, c_double, c_double, c_uint64, POINTER(c_int64), _P, _P], c_int),
    "gpm_gen_zipf_labels": ([c_int64, c_int, c_double, c_uint64, _P], c_int),
    "gpm_graph_create": ([c_int64, c_int64, _P, _P, _P, c_int, POINTER(c_void_p)], c_int),
    "gpm_graph_create_csr": ([c_int64, _P, _P, _P, POINTER(c_void_p)], c_int),
    "gpm_graph_create_device": ([c_int64, c_int64, _P, _P, c_int, POINTER(c_void_p)], c_int),
    "gpm_graph_generate": ([c_int, c_int64, c_int64, c_double, c_double, c_double, c_uint64,
                            POINTER(c_void_p)], c_int),
    "gpm_graph_destroy": ([_P], c_int),
    "gpm_graph_get_info": ([_P, _P], c_int),
    "gpm_graph_copy_csr": ([_P, _P, _P], c_int),
    "gpm_graph_set_labels": ([_P, _P], c_int),
    "gpm_graph_orient": ([_P, c_int], c_int),
    "gpm_graph_work": ([_P, POINTER(c_uint64), POINTER(c_uint64)], c_int),
    "gpm_graph_drop_plans": ([_P], c_int),
    "gpm_tc": ([_P, c_int, POINTER(c_uint64)], c_int),
    "gpm_tc_async": ([_P, c_int, _P, _P], c_int),
    "gpm_tc_host_csr": ([c_int64, _P, _P, c_int, _P, POINTER(c_uint64)], c_int),
    "gpm_tc_plan_stats": ([_P, _P], c_int),
    "gpm_tc_csr_noalloc": ([c_int64, _P, _P, _P, _P], c_int),
    "gpm_clique": ([_P, c_int, POINTER(c_uint64)], c_int),
    "gpm_clique_ex": ([_P, c_int, c_int, POINTER(c_uint64)], c_int),
    "gpm_motif": ([_P, c_int, _P], c_int),
    "gpm_pattern": ([_P, c_char_p, c_int, _P, POINTER(c_uint64)], c_int),
    "gpm_sched_create": ([c_uint64, POINTER(c_void_p)], c_int),
    "gpm_sched_destroy": ([_P], c_int),
    "gpm_sched_param_count": ([], c_int),
    "gpm_sched_get_params": ([_P, _P], c_int),
    "gpm_sched_set_params": ([_P, _P], c_int),
    "gpm_sched_collect": ([_P, _P, POINTER(c_int64)], c_int),
    "gpm_sched_dataset": ([_P, POINTER(c_int64), _P, _P], c_int),
    "gpm_sched_grad": ([_P, c_int64, _P, _P, _P, POINTER(c_double)], c_int),
    "gpm_sched_predict": ([_P, c_int64, _P, _P], c_int),
    "gpm_sched_train": ([_P, c_int, ctypes.c_float, POINTER(c_double)], c_int),
    "gpm_sched_attach": ([_P, _P], c_int),
    "gpm_sched_set_default": ([_P], c_int),
    "gpm_sched_assign": ([_P, _P, _P], c_int),
    "gpm_tc_task_costs": ([_P, _P], c_int),
    "gpm_tc_set_schedule": ([_P, _P], c_int),
    "gpm_batch_create": ([c_int, _P, _P, _P, _P, POINTER(c_void_p)], c_int),
    "gpm_batch_generate_chung_lu": ([c_int, _P, _P, _P, c_uint64, POINTER(c_void_p)], c_int),
    "gpm_batch_info": ([_P, POINTER(c_int), POINTER(c_int64), POINTER(c_int64)], c_int),
    "gpm_batch_member_csr": ([_P, c_int, _P, _P, POINTER(c_int64), POINTER(c_int64)], c_int),
    "gpm_batch_autotune": ([_P, _P], c_int),
    "gpm_batch_stage_ms": ([_P, _P], c_int),
    "gpm_batch_motif": ([_P, c_int, _P, _P], c_int),
    "gpm_batch_motif_async": ([_P, c_int, _P, _P], c_int),
    "gpm_batch_destroy": ([_P], c_int),
    "gpm_query_create": ([c_int64, c_int64, _P, _P, _P, POINTER(c_void_p)], c_int),
    "gpm_query_destroy": ([_P], c_int),
    "gpm_match": ([_P, _P, POINTER(c_uint64)], c_int),
    "gpm_match_limit": ([_P, _P, c_uint64, POINTER(c_uint64)], c_int),
    "gpm_match_list": ([_P, _P, c_uint64, _P, POINTER(c_uint64)], c_int),
    "gpm_match_batch_create": ([_P, c_int, _P, _P, c_int, POINTER(c_void_p)], c_int),
    "gpm_match_batch_autotune": ([_P, POINTER(c_int64)], c_int),
    "gpm_match_batch_run": ([_P, c_int, _P, _P], c_int),
    "gpm_match_batch_run_async": ([_P, c_int, _P, _P], c_int),
    "gpm_match_batch_info": ([_P, POINTER(c_int64), POINTER(c_int64)], c_int),
    "gpm_match_batch_destroy": ([_P], c_int),
}
for _name, (_args, _res) in _SIGS.items():
    if hasattr(lib, _name):
        _f = getattr(lib, _name)
        _f.argtypes = _args
        _f.restype = _res


def check(status: int):
    if status != GPM_OK:
        raise GpmError(status, lib.gpm_last_error().decode(errors="replace"))


def _ptr(a):
    return None if a is None else c_void_p(a.ctypes.data)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class GraphInfo(ctypes.Structure):
    _fields_ = [("n", c_int64), ("nnz", c_int64), ("max_degree", c_int32), ("oriented", c_int32),
                ("relabeled", c_int32), ("has_labels", c_int32)]


def device_count() -> int:
    n = c_int(0)
    check(lib.gpm_device_count(ctypes.byref(n)))
    return n.value


# ---------------------------------------------------------------- host helpers
def read_mtx(path: str):
    n, m, vmin = c_int64(), c_int64(), c_int32()
    check(lib.gpm_read_mtx(path.encode(), ctypes.byref(n), ctypes.byref(m), None, None, 0, ctypes.byref(vmin)))
    src = np.empty(m.value, np.int32)
    dst = np.empty(m.value, np.int32)
    check(lib.gpm_read_mtx(path.encode(), ctypes.byref(n), ctypes.byref(m), _ptr(src), _ptr(dst), m.value,
                           ctypes.byref(vmin)))
    return n.value, src, dst, vmin.value


def read_gbin(prefix: str):
    """Binary CSR (graph.vertex.bin / graph.edge.bin / graph.meta.txt):
    (offsets int64[n+1], indices int32[nnz], max_degree)."""
    n, m, md = c_int64(), c_int64(), c_int32()
    check(lib.gpm_read_gbin(prefix.encode(), ctypes.byref(n), ctypes.byref(m), None, None, ctypes.byref(md)))
    off = np.empty(n.value + 1, np.int64)
    idx = np.empty(max(m.value, 1), np.int32)
    check(lib.gpm_read_gbin(prefix.encode(), ctypes.byref(n), ctypes.byref(m), _ptr(off), _ptr(idx),
                            ctypes.byref(md)))
    return off, idx[: m.value], md.value


def write_gbin(prefix: str, offsets, indices):
    off = np.ascontiguousarray(offsets, np.int64)
    idx = np.ascontiguousarray(indices, np.int32)
    check(lib.gpm_write_gbin(prefix.encode(), len(off) - 1, _ptr(off), _ptr(idx) if len(idx) else None))


def convert_mtx_gbin(mtx_path: str, prefix: str):
    check(lib.gpm_convert_mtx_gbin(mtx_path.encode(), prefix.encode()))


def read_labels(path: str, n: int, vmin: int = 0):
    lab = np.empty(n, np.int32)
    check(lib.gpm_read_labels(path.encode(), n, vmin, _ptr(lab)))
    return lab


def read_tve(path: str):
    n, m = c_int64(), c_int64()
    check(lib.gpm_read_tve(path.encode(), ctypes.byref(n), ctypes.byref(m), None, None, None, 0))
    lab = np.empty(max(n.value, 1), np.int32)
    src = np.empty(m.value, np.int32)
    dst = np.empty(m.value, np.int32)
    check(lib.gpm_read_tve(path.encode(), ctypes.byref(n), ctypes.byref(m), _ptr(lab), _ptr(src), _ptr(dst),
                           m.value))
    return n.value, src, dst, lab[: n.value]


def gen_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1):
    m = (1 << scale) * edge_factor
    src = np.empty(m, np.int32)
    dst = np.empty(m, np.int32)
    check(lib.gpm_gen_rmat(scale, edge_factor, a, b, c, seed, _ptr(src), _ptr(dst)))
    return 1 << scale, src, dst


def gen_er(n, m, seed=1):
    src = np.empty(m, np.int32)
    dst = np.empty(m, np.int32)
    check(lib.gpm_gen_er(n, m, seed, _ptr(src), _ptr(dst)))
    return n, src, dst


def gen_chung_lu(n, gamma, mean_deg, seed=1):
    m = c_int64()
    check(lib.gpm_gen_chung_lu(n, gamma, mean_deg, seed, ctypes.byref(m), None, None))
    src = np.empty(m.value, np.int32)
    dst = np.empty(m.value, np.int32)
    check(lib.gpm_gen_chung_lu(n, gamma, mean_deg, seed, ctypes.byref(m), _ptr(src), _ptr(dst)))
    return n, src, dst


def gen_zipf_labels(n, nlabels, s=1.2, seed=1):
    lab = np.empty(n, np.int32)
    check(lib.gpm_gen_zipf_labels(n, nlabels, s, seed, _ptr(lab)))
    return lab


# ---------------------------------------------------------------- device objects
class Graph:
    """Owning wrapper of a gpm_graph handle."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def from_edges(cls, n, src, dst, labels=None, symmetrize=True):
        src, dst = _i32(src), _i32(dst)
        lab = None if labels is None else _i32(labels)
        h = c_void_p()
        check(lib.gpm_graph_create(n, len(src), _ptr(src), _ptr(dst), _ptr(lab), SYMMETRIZE if symmetrize else 0,
                                   ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_csr(cls, offsets, indices, labels=None):
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        idx = _i32(indices)
        lab = None if labels is None else _i32(labels)
        h = c_void_p()
        check(lib.gpm_graph_create_csr(len(off) - 1, _ptr(off), _ptr(idx), _ptr(lab), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_csr_ptrs(cls, n, off_ptr, idx_ptr, labels_ptr=None):
        """from_csr on raw host pointers (e.g. pinned buffers)."""
        h = c_void_p()
        check(lib.gpm_graph_create_csr(n, c_void_p(off_ptr), c_void_p(idx_ptr),
                                       c_void_p(labels_ptr) if labels_ptr else None, ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_edge_ptrs(cls, n, m, src_ptr, dst_ptr, labels_ptr=None, symmetrize=True):
        """from_edges on raw host pointers (e.g. pinned buffers)."""
        h = c_void_p()
        check(lib.gpm_graph_create(n, m, c_void_p(src_ptr), c_void_p(dst_ptr),
                                   c_void_p(labels_ptr) if labels_ptr else None, SYMMETRIZE if symmetrize else 0,
                                   ctypes.byref(h)))
        return cls(h)

    @classmethod
    def generate(cls, kind, p0, p1=0, a=0.0, b=0.0, c=0.0, seed=1):
        h = c_void_p()
        check(lib.gpm_graph_generate(kind, p0, p1, a, b, c, seed, ctypes.byref(h)))
        return cls(h)

    @classmethod
    def rmat(cls, scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1):
        return cls.generate(0, scale, edge_factor, a, b, c, seed)

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.gpm_graph_destroy(self.h)
        self.h = None

    __del__ = close

    def info(self) -> GraphInfo:
        inf = GraphInfo()
        check(lib.gpm_graph_get_info(self.h, ctypes.byref(inf)))
        return inf

    def csr(self):
        inf = self.info()
        off = np.empty(inf.n + 1, np.int64)
        idx = np.empty(max(inf.nnz, 1), np.int32)
        check(lib.gpm_graph_copy_csr(self.h, _ptr(off), _ptr(idx)))
        return off, idx[: inf.nnz]

    def set_labels(self, labels):
        lab = _i32(labels)
        check(lib.gpm_graph_set_labels(self.h, _ptr(lab)))

    def orient(self, relabel=False):
        check(lib.gpm_graph_orient(self.h, 1 if relabel else 0))
        return self

    def drop_plans(self):
        """Frees the schedules earlier counts cached with this graph."""
        check(lib.gpm_graph_drop_plans(self.h))
        return self

    def work(self):
        w, p = c_uint64(), c_uint64()
        check(lib.gpm_graph_work(self.h, ctypes.byref(w), ctypes.byref(p)))
        return w.value, p.value

    def plan_stats(self):
        """(segments, streamed keys, owner keys, owner tasks, dense segments,
        bitmap words ANDed for them) of the fixed GPM_TC_BITMAP plan."""
        st = np.zeros(6, np.uint64)
        check(lib.gpm_tc_plan_stats(self.h, _ptr(st)))
        return tuple(int(x) for x in st)

    def task_costs(self):
        """Logged active warp-cycles of every owner task under each of the 6
        scheduler configurations: float32[n, 6] (0 where v owns no task)."""
        c = np.zeros((self.info().n, 6), np.float32)
        check(lib.gpm_tc_task_costs(self.h, _ptr(c)))
        return c

    def set_schedule(self, cfg):
        """Explicit per-owner configuration (uint8[n], 0..5) for TC_LEARNED."""
        cfg = np.ascontiguousarray(cfg, np.uint8)
        check(lib.gpm_tc_set_schedule(self.h, _ptr(cfg)))
        return self

    def tc(self, mode=V_CENTRIC) -> int:
        out = c_uint64()
        check(lib.gpm_tc(self.h, mode, ctypes.byref(out)))
        return out.value

    def tc_async(self, variant, stream_ptr, d_out_ptr):
        check(lib.gpm_tc_async(self.h, variant, c_void_p(stream_ptr), c_void_p(d_out_ptr)))

    def clique(self, k, edge_centric=False) -> int:
        out = c_uint64()
        check(lib.gpm_clique_ex(self.h, k, 1 if edge_centric else 0, ctypes.byref(out)))
        return out.value

    def motif(self, k):
        out = np.zeros(2 if k == 3 else 6, np.uint64)
        check(lib.gpm_motif(self.h, k, _ptr(out)))
        return out

    def pattern(self, name, family=G2MINER):
        counters = np.zeros(6, np.uint64)
        res = c_uint64()
        check(lib.gpm_pattern(self.h, name.encode(), family, _ptr(counters), ctypes.byref(res)))
        return res.value, counters

    def match(self, q: "Query", limit=None) -> int:
        """Embeddings of q (sub_ceci semantics); with limit, min(total, limit)."""
        out = c_uint64()
        if limit is None:
            check(lib.gpm_match(self.h, q.h, ctypes.byref(out)))
        else:
            check(lib.gpm_match_limit(self.h, q.h, int(limit), ctypes.byref(out)))
        return out.value

    def match_list(self, q: "Query", limit):
        """Up to `limit` embeddings, one row of q.n data-vertex ids each."""
        emb = np.empty((max(int(limit), 1), q.n), np.int32)
        out = c_uint64()
        check(lib.gpm_match_list(self.h, q.h, int(limit), _ptr(emb), ctypes.byref(out)))
        return emb[: out.value]


class Sched:
    """Owning wrapper of the learned task scheduler (gpm_sched)."""

    # Parameters trained on logged task costs of R-MAT (scales 15-18) and
    # Chung-Lu graphs; written by train_sched.py beside this file.
    PRETRAINED = os.path.join(HERE, "sched_tc.f32")

    def __init__(self, seed=1):
        h = c_void_p()
        check(lib.gpm_sched_create(seed, ctypes.byref(h)))
        self.h = h
        self.nparams = lib.gpm_sched_param_count()

    @classmethod
    def pretrained(cls):
        s = cls()
        s.set_params(np.fromfile(cls.PRETRAINED, dtype=np.float32))
        return s

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.gpm_sched_destroy(self.h)
        self.h = None

    __del__ = close

    def params(self):
        p = np.empty(self.nparams, np.float32)
        check(lib.gpm_sched_get_params(self.h, _ptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        check(lib.gpm_sched_set_params(self.h, _ptr(p)))

    def collect(self, g: "Graph") -> int:
        r = c_int64()
        check(lib.gpm_sched_collect(self.h, g.h, ctypes.byref(r)))
        return r.value

    def dataset(self):
        r = c_int64()
        check(lib.gpm_sched_dataset(self.h, ctypes.byref(r), None, None))
        X = np.empty((r.value, 8), np.float32)
        Y = np.empty((r.value, 6), np.float32)
        check(lib.gpm_sched_dataset(self.h, ctypes.byref(r), _ptr(X), _ptr(Y)))
        return X, Y

    def grad(self, X, T):
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        gr = np.empty(self.nparams, np.float32)
        loss = c_double()
        check(lib.gpm_sched_grad(self.h, len(X), _ptr(X), _ptr(T), _ptr(gr), ctypes.byref(loss)))
        return loss.value, gr

    def predict(self, X):
        X = np.ascontiguousarray(X, np.float32)
        Y = np.empty((len(X), 6), np.float32)
        check(lib.gpm_sched_predict(self.h, len(X), _ptr(X), _ptr(Y)))
        return Y

    def train(self, steps, lr=1e-2):
        loss = c_double()
        check(lib.gpm_sched_train(self.h, steps, lr, ctypes.byref(loss)))
        return loss.value

    def attach(self, g: "Graph"):
        check(lib.gpm_sched_attach(g.h, self.h))
        g._sched = self  # the graph keeps its scheduler alive

    _default = None  # the process default, kept alive while it is the default

    def set_default(self):
        """Use this scheduler for every graph without an attached one."""
        check(lib.gpm_sched_set_default(self.h))
        Sched._default = self
        return self

    def assign(self, g: "Graph"):
        n = g.info().n
        cfg = np.empty(n, np.uint8)
        check(lib.gpm_sched_assign(self.h, g.h, _ptr(cfg)))
        return cfg


class Batch:
    """Owning wrapper of a gpm_batch (many graphs as one device union)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def from_edges(cls, members):
        """members: list of (n, src, dst) with member-local ids."""
        n = np.array([m[0] for m in members], np.int64)
        m = np.array([len(x[1]) for x in members], np.int64)
        src = _i32(np.concatenate([x[1] for x in members]) if len(members) else [])
        dst = _i32(np.concatenate([x[2] for x in members]) if len(members) else [])
        h = c_void_p()
        check(lib.gpm_batch_create(len(members), _ptr(n), _ptr(m), _ptr(src), _ptr(dst), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_edge_ptrs(cls, n, m, src_ptr, dst_ptr):
        """from_edges with member sizes n[], m[] and all members' edges back
        to back behind raw host pointers (e.g. pinned buffers)."""
        n = np.ascontiguousarray(n, np.int64)
        m = np.ascontiguousarray(m, np.int64)
        h = c_void_p()
        check(lib.gpm_batch_create(len(n), _ptr(n), _ptr(m), c_void_p(src_ptr), c_void_p(dst_ptr), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def chung_lu(cls, n, gamma, mean_deg, seed=1):
        n = np.ascontiguousarray(n, np.int64)
        gm = np.ascontiguousarray(gamma, np.float64)
        md = np.ascontiguousarray(mean_deg, np.float64)
        h = c_void_p()
        check(lib.gpm_batch_generate_chung_lu(len(n), _ptr(n), _ptr(gm), _ptr(md), seed, ctypes.byref(h)))
        return cls(h)

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.gpm_batch_destroy(self.h)
        self.h = None

    __del__ = close

    def info(self):
        g, n, e = c_int(), c_int64(), c_int64()
        check(lib.gpm_batch_info(self.h, ctypes.byref(g), ctypes.byref(n), ctypes.byref(e)))
        return g.value, n.value, e.value

    def member_csr(self, g):
        n, e = c_int64(), c_int64()
        check(lib.gpm_batch_member_csr(self.h, g, None, None, ctypes.byref(n), ctypes.byref(e)))
        off = np.empty(n.value + 1, np.int64)
        idx = np.empty(max(e.value, 1), np.int32)
        check(lib.gpm_batch_member_csr(self.h, g, _ptr(off), _ptr(idx), ctypes.byref(n), ctypes.byref(e)))
        return off, idx[: e.value]

    def autotune(self):
        t = np.zeros(3, np.int32)
        check(lib.gpm_batch_autotune(self.h, _ptr(t)))
        return t.tolist()

    def stage_ms(self):
        ms = np.zeros(3, np.float32)
        check(lib.gpm_batch_stage_ms(self.h, _ptr(ms)))
        return {"triangles_per_edge": float(ms[0]), "four_cycles": float(ms[1]), "four_cliques": float(ms[2])}

    def motif(self, use_graph=True, stream_ptr=0):
        ng = self.info()[0]
        out = np.zeros(8 * ng, np.uint64)
        check(lib.gpm_batch_motif(self.h, 1 if use_graph else 0, c_void_p(stream_ptr), _ptr(out)))
        return out.reshape(ng, 8)

    def motif_async(self, use_graph, stream_ptr, d_out_ptr):
        check(lib.gpm_batch_motif_async(self.h, 1 if use_graph else 0, c_void_p(stream_ptr), c_void_p(d_out_ptr)))


class Query:
    def __init__(self, n, src, dst, labels):
        self.n = int(n)
        src, dst, lab = _i32(src), _i32(dst), _i32(labels)
        h = c_void_p()
        check(lib.gpm_query_create(n, len(src), _ptr(src), _ptr(dst), _ptr(lab), ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.gpm_query_destroy(self.h)
        self.h = None

    __del__ = close


class MatchBatch:
    """Many labelled queries on one data graph in one launch (gpm_match_batch)."""

    def __init__(self, g: "Graph", queries, member=None, nmembers=1):
        self.g, self.queries = g, list(queries)  # kept alive with the batch
        arr = (c_void_p * len(self.queries))(*[q.h.value for q in self.queries])
        mem = None if member is None else _i32(member)
        self.nm = int(nmembers) if member is not None else 1
        h = c_void_p()
        check(lib.gpm_match_batch_create(g.h, len(self.queries), arr, _ptr(mem), self.nm, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) and lib is not None:
            lib.gpm_match_batch_destroy(self.h)
        self.h = None

    __del__ = close

    def autotune(self) -> int:
        sp = c_int64()
        check(lib.gpm_match_batch_autotune(self.h, ctypes.byref(sp)))
        return sp.value

    def info(self):
        t, sp = c_int64(), c_int64()
        check(lib.gpm_match_batch_info(self.h, ctypes.byref(t), ctypes.byref(sp)))
        return t.value, sp.value

    def run(self, use_graph=True, stream_ptr=0):
        """Counts as uint64[nq, nmembers]."""
        out = np.zeros(len(self.queries) * self.nm, np.uint64)
        check(lib.gpm_match_batch_run(self.h, 1 if use_graph else 0, c_void_p(stream_ptr), _ptr(out)))
        return out.reshape(len(self.queries), self.nm)

    def run_async(self, use_graph, stream_ptr, d_out_ptr):
        check(lib.gpm_match_batch_run_async(self.h, 1 if use_graph else 0, c_void_p(stream_ptr), c_void_p(d_out_ptr)))


def tc_host_csr(offsets, indices, variant=TC_AUTO, stream_ptr=0) -> int:
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    idx = _i32(indices)
    out = c_uint64()
    check(lib.gpm_tc_host_csr(len(off) - 1, _ptr(off), _ptr(idx), variant, c_void_p(stream_ptr),
                              ctypes.byref(out)))
    return out.value


def tc_host_csr_ptrs(n, off_ptr, idx_ptr, variant, stream_ptr) -> int:
    """Same as tc_host_csr on raw (pinned) host pointers."""
    out = c_uint64()
    check(lib.gpm_tc_host_csr(n, c_void_p(off_ptr), c_void_p(idx_ptr), variant, c_void_p(stream_ptr),
                              ctypes.byref(out)))
    return out.value
