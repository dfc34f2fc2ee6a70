"""Synthetic graph workloads (host C++/OpenMP, ``_lib/libnkgen.so``).

Each generator returns an :class:`~networkit_b200.graph.InCSR` in canonical
form (edges taken in lexicographic insertion order, so every in-row is
ascending). Draws come from a counter-based hash, so a seed gives the same
graph on any machine and thread count.

* :func:`rmat_directed` - the quadrant recursion of RmatGenerator.cpp:37-65,
  directed, duplicates and self-loops removed.
* :func:`erdos_renyi` - undirected G(n, p) (ErdosRenyiGenerator shape).
* :func:`barabasi_albert` - undirected preferential attachment
  (BarabasiAlbertGenerator shape, Batagelj variant).
* :func:`hyperbolic`, :func:`hyperbolic_batch` - undirected threshold random
  hyperbolic graphs (HyperbolicGenerator shape at temperature 0: average
  degree and power-law exponent given).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build
from .graph import InCSR

_lib = None


class _Csr(C.Structure):
    _fields_ = [
        ("z", C.c_uint64),
        ("arcs", C.c_uint64),
        ("in_ptr", C.POINTER(C.c_uint64)),
        ("in_col", C.POINTER(C.c_uint32)),
        ("outdeg", C.POINTER(C.c_uint32)),
        ("w", C.POINTER(C.c_double)),
    ]


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_build.GEN_LIB):
            _build.build_gen()
        L = C.CDLL(_build.GEN_LIB)
        L.nkgen_last_error.restype = C.c_char_p
        L.nkgen_free.argtypes = [C.POINTER(_Csr)]
        L.nkgen_rmat.argtypes = [C.c_int, C.c_uint64, C.c_double, C.c_double, C.c_double,
                                 C.c_uint64, C.c_int, C.POINTER(_Csr)]
        L.nkgen_erdos_renyi.argtypes = [C.c_uint64, C.c_double, C.c_uint64, C.c_int,
                                        C.POINTER(_Csr)]
        L.nkgen_erdos_renyi_stream.argtypes = [C.c_uint64, C.c_double, C.c_uint64, C.c_int,
                                               C.c_int, C.POINTER(_Csr)]
        L.nkgen_barabasi_albert_stream.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64,
                                                   C.c_uint64, C.POINTER(_Csr)]
        L.nkgen_hyperbolic_stream.argtypes = [C.c_uint64, C.c_double, C.c_double, C.c_uint64,
                                              C.POINTER(_Csr)]
        L.nkgen_hyperbolic_stream_batch.argtypes = [C.c_uint64, C.POINTER(C.c_uint64),
                                                    C.c_double, C.c_double, C.c_uint64,
                                                    C.POINTER(_Csr), C.POINTER(C.c_uint64)]
        L.nkgen_barabasi_albert.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(_Csr)]
        L.nkgen_hyperbolic.argtypes = [C.c_uint64, C.c_double, C.c_double, C.c_uint64,
                                       C.POINTER(_Csr)]
        L.nkgen_hyperbolic_batch.argtypes = [C.c_uint64, C.POINTER(C.c_uint64), C.c_double,
                                             C.c_double, C.c_uint64, C.c_int, C.POINTER(_Csr),
                                             C.POINTER(C.c_uint64)]
        _lib = L
    return _lib


def _take(c: _Csr, directed: bool) -> InCSR:
    z, m = int(c.z), int(c.arcs)
    in_ptr = np.ctypeslib.as_array(c.in_ptr, shape=(z + 1,)).copy()
    in_col = (np.ctypeslib.as_array(c.in_col, shape=(m,)).copy() if m
              else np.zeros(0, np.uint32))
    outdeg = np.ctypeslib.as_array(c.outdeg, shape=(z,)).copy()
    _load().nkgen_free(C.byref(c))
    return InCSR(z, z, in_ptr, in_col, None, outdeg.astype(np.float64), outdeg, None, directed)


def _check(rc):
    if rc != 0:
        raise RuntimeError(_load().nkgen_last_error().decode())


def rmat_directed(scale: int, edgefactor: int = 16, a: float = 0.57, b: float = 0.19,
                  c: float = 0.19, seed: int = 42, nthreads: int = 0) -> InCSR:
    """Directed R-MAT with edgefactor * 2^scale draws (d = 1 - a - b - c),
    duplicates and self-loops removed, unweighted."""
    out = _Csr()
    _check(_load().nkgen_rmat(int(scale), int(edgefactor), float(a), float(b), float(c),
                              int(seed), int(nthreads), C.byref(out)))
    return _take(out, True)


def erdos_renyi(n: int, p: float, seed: int = 42, nthreads: int = 0) -> InCSR:
    """Undirected G(n, p) without self-loops."""
    out = _Csr()
    _check(_load().nkgen_erdos_renyi(int(n), float(p), int(seed), int(nthreads), C.byref(out)))
    return _take(out, False)


def erdos_renyi_stream(n: int, p: float, seed: int = 42, directed: bool = False,
                       threads: int = 1) -> InCSR:
    """G(n, p) drawn as NetworKit's ErdosRenyiGenerator(n, p, directed) draws
    it with `threads` OpenMP threads after ``setSeed(seed, False)``: the same
    graph, with the adjacency order of the Graph it builds. The reference's
    graph depends on its thread count (every thread restarts the seed's
    stream on its own range of rows), so the count is part of the input."""
    out = _Csr()
    _check(_load().nkgen_erdos_renyi_stream(int(n), float(p), int(seed), int(bool(directed)),
                                            int(threads), C.byref(out)))
    return _take(out, bool(directed))


def barabasi_albert(k: int, n: int, seed: int = 42) -> InCSR:
    """Undirected Barabasi-Albert graph: a ring of k nodes, then every new node
    attaches to k distinct earlier nodes chosen proportionally to degree."""
    out = _Csr()
    _check(_load().nkgen_barabasi_albert(int(k), int(n), int(seed), C.byref(out)))
    return _take(out, False)


def barabasi_albert_stream(k: int, n: int, seed: int = 42, n0: int = 0) -> InCSR:
    """Undirected Barabasi-Albert graph as NetworKit's
    BarabasiAlbertGenerator(k, n, n0) draws it (its default Batagelj-Brandes
    method) after ``setSeed(seed, False)``: the same graph, with the
    adjacency order of the Graph it builds."""
    out = _Csr()
    _check(_load().nkgen_barabasi_albert_stream(int(k), int(n), int(n0), int(seed),
                                                C.byref(out)))
    return _take(out, False)


def hyperbolic(n: int, avg_deg: float = 16.0, exponent: float = 3.0, seed: int = 42) -> InCSR:
    """Undirected random hyperbolic graph, threshold model: n points in a
    hyperbolic disc whose radius gives expected average degree avg_deg,
    radial density exponent-dependent (alpha = (exponent - 1) / 2), edges
    between points at distance <= the radius."""
    out = _Csr()
    _check(_load().nkgen_hyperbolic(int(n), float(avg_deg), float(exponent), int(seed),
                                    C.byref(out)))
    return _take(out, False)


def hyperbolic_stream(n: int, avg_deg: float = 16.0, exponent: float = 3.0,
                      seed: int = 42) -> InCSR:
    """Undirected threshold random hyperbolic graph as NetworKit's
    HyperbolicGenerator(n, avg_deg, exponent).generate() draws it after
    ``setSeed(seed, False)``: the same graph (nodes numbered by angle), with
    the adjacency order of the Graph it builds on one thread."""
    out = _Csr()
    _check(_load().nkgen_hyperbolic_stream(int(n), float(avg_deg), float(exponent), int(seed),
                                           C.byref(out)))
    return _take(out, False)


def hyperbolic_stream_batch(ns, avg_deg: float = 16.0, exponent: float = 3.0, seed: int = 42):
    """len(ns) graphs of `hyperbolic_stream` (graph i with ns[i] nodes and
    seed + i) as one block-diagonal InCSR plus node_offsets."""
    ns = np.ascontiguousarray(ns, np.uint64)
    offs = np.zeros(ns.shape[0] + 1, np.uint64)
    out = _Csr()
    _check(_load().nkgen_hyperbolic_stream_batch(
        int(ns.shape[0]), ns.ctypes.data_as(C.POINTER(C.c_uint64)), float(avg_deg),
        float(exponent), int(seed), C.byref(out), offs.ctypes.data_as(C.POINTER(C.c_uint64))))
    return _take(out, False), offs


def hyperbolic_batch(ns, avg_deg: float = 16.0, exponent: float = 3.0, seed: int = 42,
                     nthreads: int = 0):
    """len(ns) hyperbolic graphs (graph i with ns[i] nodes and seed + i) as one
    block-diagonal InCSR plus node_offsets (graph i = nodes
    [node_offsets[i], node_offsets[i+1]))."""
    ns = np.ascontiguousarray(ns, np.uint64)
    offs = np.zeros(ns.shape[0] + 1, np.uint64)
    out = _Csr()
    _check(_load().nkgen_hyperbolic_batch(
        int(ns.shape[0]), ns.ctypes.data_as(C.POINTER(C.c_uint64)), float(avg_deg),
        float(exponent), int(seed), int(nthreads), C.byref(out),
        offs.ctypes.data_as(C.POINTER(C.c_uint64))))
    return _take(out, False), offs


def with_uniform_weights(csr: InCSR, seed: int = 43, low: float = 0.1, high: float = 1.0) -> InCSR:
    """Copy of ``csr`` with arc weights uniform in (low, high] and the matching
    weighted out-degrees. Undirected graphs get one weight per edge (both arcs
    of an edge share it)."""
    rng = np.random.default_rng(seed)
    m = csr.arcs
    if csr.directed:
        w = high - (high - low) * rng.random(m)
    else:
        rows = np.repeat(np.arange(csr.z, dtype=np.int64), np.diff(csr.in_ptr).astype(np.int64))
        cols = csr.in_col.astype(np.int64)
        lo = np.minimum(rows, cols)
        hi = np.maximum(rows, cols)
        key = lo * csr.z + hi
        uk, inv = np.unique(key, return_inverse=True)
        we = high - (high - low) * rng.random(uk.shape[0])
        w = we[inv]
    wdeg = np.bincount(csr.in_col, weights=w, minlength=csr.z)
    return InCSR(csr.z, csr.n, csr.in_ptr, csr.in_col, np.ascontiguousarray(w), wdeg,
                 csr.outdeg, csr.exists, csr.directed)
