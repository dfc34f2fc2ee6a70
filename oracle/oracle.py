"""Test infrastructure only (the oracle).

ctypes bindings for
  * ``lib/libnkoracle.so`` - the plain-C restatement of the reference paths
    (``pagerank_oracle.c``: PageRank, its adjoint, EigenvectorCentrality,
    KatzCentrality, ApproximatePageRank and PageRankNibble's sweep), and
  * ``_ref/libnkref.so`` - the reference's own implementations compiled from
    the reference sources (``Makefile``, ``ref/nkref_capi.cpp``), present only
    where it was built.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` (the reference arm, and the reference's own runs timed beside
each companion form) import this module, and only as the checker or the
baseline. The product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "lib", "libnkoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libnkref.so")

_u64p = C.POINTER(C.c_uint64)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
_f64p = C.POINTER(C.c_double)


class _Params(C.Structure):
    _fields_ = [
        ("damp", C.c_double),
        ("tol", C.c_double),
        ("norm", C.c_int32),
        ("normalized", C.c_int32),
        ("distribute_sinks", C.c_int32),
        ("nthreads", C.c_int32),
        ("max_iterations", C.c_uint64),
    ]


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference sources are present, the
    reference library)."""
    target = "all" if ref else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def _ptr(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        lib = C.CDLL(ORACLE_SO)
        lib.nko_pagerank.restype = C.c_int
        lib.nko_pagerank.argtypes = [C.c_uint64, _u64p, _u32p, _f64p, _f64p, _u32p, _u8p, _f64p,
                                     C.POINTER(_Params), _f64p, _u64p, _f64p, _f64p, C.c_uint64]
        lib.nko_ranking.restype = C.c_int
        lib.nko_ranking.argtypes = [C.c_uint64, _f64p, _u8p, _u64p, _f64p]
        lib.nko_pagerank_adjoint.restype = C.c_int64
        lib.nko_pagerank_adjoint.argtypes = [C.c_uint64, _u64p, _u32p, _f64p, _f64p, _u32p, _f64p,
                                             C.c_double, C.c_int, _f64p, _f64p, C.c_double,
                                             C.c_uint64, _f64p, _f64p, _f64p, C.c_int]
        lib.nko_eigenvector.restype = C.c_int64
        lib.nko_eigenvector.argtypes = [C.c_uint64, _u64p, _u32p, _f64p, _u8p, C.c_double,
                                        C.c_uint64, _f64p]
        lib.nko_katz.restype = C.c_int64
        lib.nko_katz.argtypes = [C.c_uint64, _u64p, _u32p, _f64p, _u8p, C.c_double, C.c_double,
                                 C.c_double, C.c_uint64, _f64p]
        lib.nko_volumes.restype = C.c_int
        lib.nko_volumes.argtypes = [C.c_uint64, _u64p, _u32p, _f64p, _f64p]
        lib.nko_apr.restype = C.c_int64
        lib.nko_apr.argtypes = [C.c_uint64, _u64p, _u32p, _f64p, _f64p, C.c_double, C.c_double,
                                _u32p, C.c_uint64, C.c_uint64, _u32p, _f64p, _u64p]
        lib.nko_finish.restype = None
        lib.nko_finish.argtypes = [C.c_uint64, _u8p, _u32p, C.c_double, C.c_int, C.c_uint64,
                                   _f64p, _f64p]
        lib.nko_sweep_rows.restype = C.c_int
        lib.nko_sweep_rows.argtypes = [C.c_uint64, _u64p, _u32p, _f64p, _f64p, _f64p, _u32p,
                                       C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_int,
                                       C.c_int, _f64p, _f64p, _f64p]
        lib.nko_sweep_set.restype = C.c_int64
        lib.nko_sweep_set.argtypes = [C.c_uint64, _u64p, _u32p, _f64p, _f64p, C.c_double,
                                      C.c_uint64, C.c_uint64, _u32p, _f64p, _u32p]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("reference library not built: " + REF_SO)
        lib = C.CDLL(REF_SO)
        lib.nkref_last_error.restype = C.c_char_p
        lib.nkref_graph_create.restype = C.c_int
        lib.nkref_graph_create.argtypes = [C.POINTER(C.c_void_p), C.c_uint64, C.c_int, C.c_int,
                                           C.c_uint64, _u32p, _u32p, _f64p, _u8p]
        lib.nkref_graph_read.restype = C.c_int
        lib.nkref_graph_read.argtypes = [C.POINTER(C.c_void_p), C.c_char_p, C.c_int, C.c_int]
        lib.nkref_graph_destroy.argtypes = [C.c_void_p]
        for f in ("nkref_graph_num_nodes", "nkref_graph_upper_node_id", "nkref_graph_num_edges"):
            getattr(lib, f).restype = C.c_uint64
            getattr(lib, f).argtypes = [C.c_void_p]
        lib.nkref_graph_is_directed.argtypes = [C.c_void_p]
        lib.nkref_graph_is_weighted.argtypes = [C.c_void_p]
        lib.nkref_graph_arc_counts.argtypes = [C.c_void_p, _u64p, _u64p]
        lib.nkref_graph_export.restype = C.c_int
        lib.nkref_graph_export.argtypes = [C.c_void_p, _u64p, _u32p, _f64p, _u64p, _u32p, _f64p,
                                           _u8p]
        lib.nkref_write_nkbg.restype = C.c_int
        lib.nkref_write_nkbg.argtypes = [C.c_void_p, C.c_char_p, C.c_uint64, C.c_int]
        lib.nkref_read_nkbg.restype = C.c_int
        lib.nkref_read_nkbg.argtypes = [C.POINTER(C.c_void_p), C.c_char_p]
        lib.nkref_barabasi_albert.restype = C.c_int
        lib.nkref_barabasi_albert.argtypes = [C.POINTER(C.c_void_p), C.c_uint64, C.c_uint64,
                                              C.c_uint64, C.c_uint64]
        lib.nkref_hyperbolic.restype = C.c_int
        lib.nkref_hyperbolic.argtypes = [C.POINTER(C.c_void_p), C.c_uint64, C.c_double,
                                         C.c_double, C.c_uint64, C.c_int]
        lib.nkref_erdos_renyi.restype = C.c_int
        lib.nkref_erdos_renyi.argtypes = [C.POINTER(C.c_void_p), C.c_uint64, C.c_double,
                                          C.c_uint64, C.c_int, C.c_int]
        lib.nkref_eigenvector.restype = C.c_int
        lib.nkref_eigenvector.argtypes = [C.c_void_p, C.c_double, C.c_int, _f64p, _f64p]
        lib.nkref_katz.restype = C.c_int
        lib.nkref_katz.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int,
                                   C.c_int, _f64p, _u64p, _f64p]
        lib.nkref_pagerank.restype = C.c_int
        lib.nkref_pagerank.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int,
                                       C.c_uint64, C.c_int, _f64p, _u64p, _f64p, _u64p, _f64p,
                                       _f64p]
        lib.nkref_apr.restype = C.c_int
        lib.nkref_apr.argtypes = [C.c_void_p, C.c_double, C.c_double, _u32p, C.c_uint64,
                                  C.c_uint64, _u32p, _f64p, _u64p, _f64p]
        lib.nkref_prn.restype = C.c_int
        lib.nkref_prn.argtypes = [C.c_void_p, C.c_double, C.c_double, _u32p, C.c_uint64, C.c_int,
                                  C.c_uint64, _u64p, _u32p, _u64p, _f64p]
        _ref = lib
    return _ref


@dataclass
class OracleResult:
    scores: np.ndarray
    iterations: int
    maximum: float
    trace: np.ndarray


def pagerank(csr, damp=0.85, tol=1e-8, norm=1, normalized=False, distribute_sinks=False,
             max_iterations=2**64 - 1, teleport=None, nthreads=1, trace_cap=100000) -> OracleResult:
    """Run the C restatement on an in-CSR (any object with the attributes
    z, in_ptr, in_col, in_w, wdeg, outdeg, exists)."""
    lib = oracle_lib()
    z = int(csr.z)
    scores = np.empty(z, np.float64)
    iters = C.c_uint64(0)
    mx = C.c_double(0.0)
    trace = np.zeros(trace_cap, np.float64)
    p = _Params(damp, tol, int(norm), int(bool(normalized)), int(bool(distribute_sinks)),
                int(nthreads), int(max_iterations))
    tele = None if teleport is None else np.ascontiguousarray(teleport, np.float64)
    rc = lib.nko_pagerank(z, _ptr(csr.in_ptr, _u64p), _ptr(csr.in_col, _u32p),
                          _ptr(csr.in_w, _f64p), _ptr(csr.wdeg, _f64p), _ptr(csr.outdeg, _u32p),
                          _ptr(csr.exists, _u8p), _ptr(tele, _f64p), C.byref(p),
                          _ptr(scores, _f64p), C.byref(iters), C.byref(mx), _ptr(trace, _f64p),
                          trace_cap)
    if rc != 0:
        raise RuntimeError("oracle nko_pagerank failed")
    it = int(iters.value)
    return OracleResult(scores, it, float(mx.value), trace[:min(it, trace_cap)].copy())


def finish(scores, outdeg, damp, normalized, n=None, exists=None):
    """PageRank.cpp:75-102 on a final iterate (a copy): (scores, maximum)."""
    lib = oracle_lib()
    x = np.array(scores, np.float64, copy=True)
    z = x.shape[0]
    n = z if n is None else int(n)
    mx = C.c_double(0.0)
    lib.nko_finish(z, _ptr(exists, _u8p), _ptr(np.ascontiguousarray(outdeg, np.uint32), _u32p),
                   float(damp), int(bool(normalized)), n, _ptr(x, _f64p), C.byref(mx))
    return x, float(mx.value)


def sweep_rows(ptr, col, w, x, wdeg, outdeg_rows, base, damp, teleport_prob, share, distribute,
               l2, x_out):
    """One sweep of a row slice (nko_sweep_rows): writes x_out, returns
    (residual partial sum, sink-mass partial sum)."""
    lib = oracle_lib()
    res, sink = C.c_double(0.0), C.c_double(0.0)
    rows = int(np.asarray(ptr).shape[0]) - 1
    rc = lib.nko_sweep_rows(rows, _ptr(ptr, _u64p), _ptr(col, _u32p), _ptr(w, _f64p),
                            _ptr(x, _f64p), _ptr(wdeg, _f64p), _ptr(outdeg_rows, _u32p), int(base),
                            float(damp), float(teleport_prob), float(share), int(bool(distribute)),
                            int(bool(l2)), _ptr(x_out, _f64p), C.byref(res), C.byref(sink))
    if rc != 0:
        raise RuntimeError("oracle nko_sweep_rows failed")
    return float(res.value), float(sink.value)


def ranking(scores, exists=None):
    lib = oracle_lib()
    z = scores.shape[0]
    n = z if exists is None else int(np.count_nonzero(exists))
    ids = np.empty(n, np.uint64)
    vals = np.empty(n, np.float64)
    sc = np.ascontiguousarray(scores, np.float64)
    ex = None if exists is None else np.ascontiguousarray(exists, np.uint8)
    lib.nko_ranking(z, _ptr(sc, _f64p), _ptr(ex, _u8p), _ptr(ids, _u64p), _ptr(vals, _f64p))
    return ids, vals


def eigenvector(csr, tol=1e-9, max_iterations=100000):
    """EigenvectorCentrality (C restatement); returns (scores, iterations)."""
    lib = oracle_lib()
    z = int(csr.z)
    scores = np.empty(z, np.float64)
    ex = None if csr.exists is None else np.ascontiguousarray(csr.exists, np.uint8)
    it = lib.nko_eigenvector(z, _ptr(np.ascontiguousarray(csr.in_ptr, np.uint64), _u64p),
                             _ptr(np.ascontiguousarray(csr.in_col, np.uint32), _u32p),
                             _ptr(csr.in_w, _f64p), _ptr(ex, _u8p), tol, max_iterations,
                             _ptr(scores, _f64p))
    if it < 0:
        raise RuntimeError("oracle eigenvector failed")
    return scores, int(it)


def katz(z, ptr, col, w=None, exists=None, alpha=0.0, beta=0.1, tol=1e-8, max_degree=None,
         max_iterations=100000):
    """KatzCentrality (C restatement) over the adjacency (ptr, col, w): the
    in-CSR for InEdges, the out-CSR for OutEdges. alpha 0 = 1/(1 + max_degree)
    (KatzCentrality.cpp:15-17). Returns (scores, iterations)."""
    lib = oracle_lib()
    if alpha == 0:
        alpha = 1.0 / (1.0 + max_degree)
    scores = np.empty(int(z), np.float64)
    ex = None if exists is None else np.ascontiguousarray(exists, np.uint8)
    ww = None if w is None else np.ascontiguousarray(w, np.float64)
    it = lib.nko_katz(int(z), _ptr(np.ascontiguousarray(ptr, np.uint64), _u64p),
                      _ptr(np.ascontiguousarray(col, np.uint32), _u32p), _ptr(ww, _f64p),
                      _ptr(ex, _u8p), alpha, beta, tol, max_iterations, _ptr(scores, _f64p))
    if it < 0:
        raise RuntimeError("oracle katz failed")
    return scores, int(it)


def adjoint(csr, x, g, damp=0.85, distribute_sinks=True, teleport=None, tol=1e-14,
            max_iter=100000, nthreads=1):
    """FP64 host adjoint solve; returns (lam, grad_w, grad_t, sweeps). The
    result does not depend on nthreads."""
    lib = oracle_lib()
    z = int(csr.z)
    lam = np.empty(z, np.float64)
    gw = np.empty(csr.in_col.shape[0], np.float64)
    gt = np.empty(z, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    g = np.ascontiguousarray(g, np.float64)
    tele = None if teleport is None else np.ascontiguousarray(teleport, np.float64)
    sweeps = lib.nko_pagerank_adjoint(z, _ptr(csr.in_ptr, _u64p), _ptr(csr.in_col, _u32p),
                                      _ptr(csr.in_w, _f64p), _ptr(csr.wdeg, _f64p),
                                      _ptr(csr.outdeg, _u32p), _ptr(tele, _f64p), damp,
                                      int(bool(distribute_sinks)), _ptr(x, _f64p),
                                      _ptr(g, _f64p), tol, max_iter, _ptr(lam, _f64p),
                                      _ptr(gw, _f64p), _ptr(gt, _f64p), int(nthreads))
    if sweeps < 0:
        raise RuntimeError("oracle adjoint failed")
    return lam, gw, gt, int(sweeps)


# ---------------------------------------------------------------------------
# The reference library (oracle/_ref)


def volumes(z, ptr, col, w=None):
    """weightedDegree(u, true) of every node of a neighbour CSR."""
    vol = np.empty(int(z), np.float64)
    oracle_lib().nko_volumes(int(z), _ptr(np.ascontiguousarray(ptr, np.uint64), _u64p),
                             _ptr(np.ascontiguousarray(col, np.uint32), _u32p),
                             _ptr(None if w is None else np.ascontiguousarray(w, np.float64),
                                  _f64p), _ptr(vol, _f64p))
    return vol


@dataclass
class AprResult:
    nodes: np.ndarray   # support, ascending ids
    values: np.ndarray  # p of each support node
    pushes: int


def apr(z, ptr, col, w, seeds, alpha, eps, vol=None):
    """ApproximatePageRank(G, alpha, eps).run(seeds) over the neighbour CSR
    (forNeighborsOf order); seeds: any iterable (made a sorted set)."""
    ptr = np.ascontiguousarray(ptr, np.uint64)
    col = np.ascontiguousarray(col, np.uint32)
    w = None if w is None else np.ascontiguousarray(w, np.float64)
    if vol is None:
        vol = volumes(z, ptr, col, w)
    sd = np.unique(np.asarray(list(seeds) if not np.isscalar(seeds) else [seeds],
                              np.int64)).astype(np.uint32)
    cap = 1 << 16
    pushes = C.c_uint64(0)
    while True:
        nodes = np.empty(cap, np.uint32)
        vals = np.empty(cap, np.float64)
        cnt = oracle_lib().nko_apr(int(z), _ptr(ptr, _u64p), _ptr(col, _u32p), _ptr(w, _f64p),
                                   _ptr(vol, _f64p), float(alpha), float(eps), _ptr(sd, _u32p),
                                   sd.shape[0], cap, _ptr(nodes, _u32p), _ptr(vals, _f64p),
                                   C.byref(pushes))
        if cnt < 0:
            raise ValueError("bad APR input")
        if cnt <= cap:
            return AprResult(nodes[:cnt].copy(), vals[:cnt].copy(), int(pushes.value))
        cap = int(cnt)


def sweep_set(z, ptr, col, w, vol, total_volume, n_nodes, nodes, values):
    """PageRankNibble::bestSweepSet over an APR support; ascending ids."""
    nodes = np.ascontiguousarray(nodes, np.uint32)
    values = np.ascontiguousarray(values, np.float64)
    out = np.empty(max(1, nodes.shape[0]), np.uint32)
    k = oracle_lib().nko_sweep_set(
        int(z), _ptr(np.ascontiguousarray(ptr, np.uint64), _u64p),
        _ptr(np.ascontiguousarray(col, np.uint32), _u32p),
        _ptr(None if w is None else np.ascontiguousarray(w, np.float64), _f64p),
        _ptr(np.ascontiguousarray(vol, np.float64), _f64p), float(total_volume), int(n_nodes),
        nodes.shape[0], _ptr(nodes, _u32p), _ptr(values, _f64p), _ptr(out, _u32p))
    if k < 0:
        raise ValueError("bad sweep input")
    return out[:k].copy()


class RefGraph:
    """A NetworKit::Graph owned by the reference library."""

    def __init__(self, handle):
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.nkref_graph_destroy(self.h)
            self.h = None

    @classmethod
    def from_edges(cls, n, src, dst, w=None, directed=False, weighted=False, exists=None):
        lib = ref_lib()
        h = C.c_void_p()
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        w = None if w is None else np.ascontiguousarray(w, np.float64)
        ex = None if exists is None else np.ascontiguousarray(exists, np.uint8)
        rc = lib.nkref_graph_create(C.byref(h), int(n), int(bool(weighted)), int(bool(directed)),
                                    src.shape[0], _ptr(src, _u32p), _ptr(dst, _u32p),
                                    _ptr(w, _f64p), _ptr(ex, _u8p))
        if rc != 0:
            raise RuntimeError(lib.nkref_last_error().decode())
        return cls(h)

    @classmethod
    def read(cls, path, kind, directed=False):
        """kind: 0 = SNAP, 1 = METIS, 2 = GML (the reference readers)."""
        lib = ref_lib()
        h = C.c_void_p()
        rc = lib.nkref_graph_read(C.byref(h), path.encode(), int(kind), int(bool(directed)))
        if rc != 0:
            raise RuntimeError(lib.nkref_last_error().decode())
        return cls(h)

    @property
    def z(self):
        return int(ref_lib().nkref_graph_upper_node_id(self.h))

    @property
    def n(self):
        return int(ref_lib().nkref_graph_num_nodes(self.h))

    @property
    def m(self):
        return int(ref_lib().nkref_graph_num_edges(self.h))

    @property
    def directed(self):
        return bool(ref_lib().nkref_graph_is_directed(self.h))

    @property
    def weighted(self):
        return bool(ref_lib().nkref_graph_is_weighted(self.h))

    def export(self):
        """Adjacency in storage order: dict with out_ptr, out_adj, out_w, in_ptr,
        in_adj, in_w (directed only), exists."""
        lib = ref_lib()
        oa, ia = C.c_uint64(0), C.c_uint64(0)
        lib.nkref_graph_arc_counts(self.h, C.byref(oa), C.byref(ia))
        z = self.z
        out_ptr = np.zeros(z + 1, np.uint64)
        out_adj = np.zeros(oa.value, np.uint32)
        out_w = np.zeros(oa.value, np.float64)
        directed = self.directed
        in_ptr = np.zeros(z + 1, np.uint64) if directed else None
        in_adj = np.zeros(ia.value, np.uint32) if directed else None
        in_w = np.zeros(ia.value, np.float64) if directed else None
        exists = np.zeros(z, np.uint8)
        rc = lib.nkref_graph_export(self.h, _ptr(out_ptr, _u64p), _ptr(out_adj, _u32p),
                                    _ptr(out_w, _f64p), _ptr(in_ptr, _u64p), _ptr(in_adj, _u32p),
                                    _ptr(in_w, _f64p), _ptr(exists, _u8p))
        if rc != 0:
            raise RuntimeError(lib.nkref_last_error().decode())
        return dict(out_ptr=out_ptr, out_adj=out_adj, out_w=out_w, in_ptr=in_ptr, in_adj=in_adj,
                    in_w=in_w, exists=exists, directed=directed, weighted=self.weighted)

    def write_nkbg(self, path, chunks=32, weights=5):
        """weights: 0 none, 1 unsigned varint, 2 signed varint, 3 double,
        4 float, 5 auto-detect (NetworkitBinaryWriter.hpp:17-24)."""
        lib = ref_lib()
        if lib.nkref_write_nkbg(self.h, path.encode(), int(chunks), int(weights)) != 0:
            raise RuntimeError(lib.nkref_last_error().decode())

    @classmethod
    def read_nkbg(cls, path):
        lib = ref_lib()
        h = C.c_void_p()
        if lib.nkref_read_nkbg(C.byref(h), path.encode()) != 0:
            raise RuntimeError(lib.nkref_last_error().decode())
        return cls(h)

    @classmethod
    def erdos_renyi(cls, n, p, seed=42, directed=False, threads=1):
        """The reference's ErdosRenyiGenerator(n, p, directed).generate() on
        `threads` OpenMP threads after Aux::Random::setSeed(seed, False)."""
        lib = ref_lib()
        h = C.c_void_p()
        if lib.nkref_erdos_renyi(C.byref(h), int(n), float(p), int(seed), int(bool(directed)),
                                 int(threads)) != 0:
            raise RuntimeError(lib.nkref_last_error().decode())
        return cls(h)

    @classmethod
    def barabasi_albert(cls, k, n, seed=42, n0=0):
        """The reference's BarabasiAlbertGenerator(k, n, n0).generate() after
        Aux::Random::setSeed(seed, False)."""
        lib = ref_lib()
        h = C.c_void_p()
        if lib.nkref_barabasi_albert(C.byref(h), int(k), int(n), int(n0), int(seed)) != 0:
            raise RuntimeError(lib.nkref_last_error().decode())
        return cls(h)

    @classmethod
    def hyperbolic(cls, n, avg_deg=16.0, exponent=3.0, seed=42, threads=1):
        """The reference's HyperbolicGenerator(n, avg_deg, exponent).generate()
        on `threads` OpenMP threads after Aux::Random::setSeed(seed, False)."""
        lib = ref_lib()
        h = C.c_void_p()
        if lib.nkref_hyperbolic(C.byref(h), int(n), float(avg_deg), float(exponent), int(seed),
                                int(threads)) != 0:
            raise RuntimeError(lib.nkref_last_error().decode())
        return cls(h)

    def apr(self, alpha, eps, seeds):
        """The reference's ApproximatePageRank(G, alpha, eps).run(seeds):
        (nodes ascending, values, seconds)."""
        lib = ref_lib()
        sd = np.ascontiguousarray(np.atleast_1d(np.asarray(seeds, np.int64)), np.uint32)
        cap = 1 << 16
        while True:
            nodes = np.empty(cap, np.uint32)
            vals = np.empty(cap, np.float64)
            cnt = C.c_uint64(0)
            secs = C.c_double(0.0)
            if lib.nkref_apr(self.h, float(alpha), float(eps), _ptr(sd, _u32p), sd.shape[0], cap,
                             _ptr(nodes, _u32p), _ptr(vals, _f64p), C.byref(cnt),
                             C.byref(secs)) != 0:
                raise RuntimeError(lib.nkref_last_error().decode())
            if cnt.value <= cap:
                k = int(cnt.value)
                return nodes[:k].copy(), vals[:k].copy(), secs.value
            cap = int(cnt.value)

    def prn(self, alpha, eps, seeds, joint=False):
        """The reference's PageRankNibble(G, alpha, eps): one community per
        seed (run(seeds), seeds ascending) or, with joint, one community of
        the seed set. Returns (list of ascending id arrays, seconds)."""
        lib = ref_lib()
        sd = np.ascontiguousarray(np.atleast_1d(np.asarray(seeds, np.int64)), np.uint32)
        k = 1 if joint else np.unique(sd).shape[0]
        cap = 1 << 16
        while True:
            offs = np.zeros(k + 1, np.uint64)
            sets = np.empty(cap, np.uint32)
            tot = C.c_uint64(0)
            secs = C.c_double(0.0)
            if lib.nkref_prn(self.h, float(alpha), float(eps), _ptr(sd, _u32p), sd.shape[0],
                             int(bool(joint)), cap, _ptr(offs, _u64p), _ptr(sets, _u32p),
                             C.byref(tot), C.byref(secs)) != 0:
                raise RuntimeError(lib.nkref_last_error().decode())
            if tot.value <= cap:
                return [sets[int(offs[i]):int(offs[i + 1])].copy() for i in range(k)], secs.value
            cap = int(tot.value)

    def eigenvector(self, tol=1e-9, nthreads=0, timed=False):
        """scores (and, with timed, the seconds of run())."""
        lib = ref_lib()
        scores = np.empty(self.z, np.float64)
        secs = C.c_double(0.0)
        if lib.nkref_eigenvector(self.h, tol, int(nthreads), _ptr(scores, _f64p),
                                 C.byref(secs)) != 0:
            raise RuntimeError(lib.nkref_last_error().decode())
        return (scores, secs.value) if timed else scores

    def katz(self, alpha=0.0, beta=0.1, tol=1e-8, out_edges=False, nthreads=0, timed=False):
        """(scores, ranking ids) (and, with timed, the seconds of run())."""
        lib = ref_lib()
        scores = np.empty(self.z, np.float64)
        ids = np.empty(self.n, np.uint64)
        secs = C.c_double(0.0)
        if lib.nkref_katz(self.h, alpha, beta, tol, int(bool(out_edges)), int(nthreads),
                          _ptr(scores, _f64p), _ptr(ids, _u64p), C.byref(secs)) != 0:
            raise RuntimeError(lib.nkref_last_error().decode())
        return (scores, ids, secs.value) if timed else (scores, ids)

    def pagerank(self, damp=0.85, tol=1e-8, normalized=False, norm=1, max_iterations=2**64 - 1,
                 nthreads=0, want_ranking=True):
        lib = ref_lib()
        z, n = self.z, self.n
        scores = np.empty(z, np.float64)
        iters = C.c_uint64(0)
        mx = C.c_double(0.0)
        secs = C.c_double(0.0)
        ids = np.empty(n, np.uint64) if want_ranking else None
        vals = np.empty(n, np.float64) if want_ranking else None
        rc = lib.nkref_pagerank(self.h, damp, tol, int(bool(normalized)), int(norm),
                                int(max_iterations), int(nthreads), _ptr(scores, _f64p),
                                C.byref(iters), C.byref(mx), _ptr(ids, _u64p), _ptr(vals, _f64p),
                                C.byref(secs))
        if rc != 0:
            raise RuntimeError(lib.nkref_last_error().decode())
        return dict(scores=scores, iterations=int(iters.value), maximum=float(mx.value),
                    ranking_ids=ids, ranking_vals=vals, seconds=float(secs.value))
