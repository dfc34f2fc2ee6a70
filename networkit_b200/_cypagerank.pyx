# cython: language_level=3, boundscheck=False, wraparound=False
"""``PageRank`` as a compiled Cython class over include/nkgpu.h.

This is the binding a NetworKit build would carry in place of its own
``cdef class PageRank(Centrality)`` (networkit/centrality.pyx:1989-2037): the
same constructor arguments and defaults, the ``norm`` / ``maxIterations``
properties (:2021-2037), ``run()`` with the GIL released around the library
call (networkit/base.pyx:17-30), and the inherited ``scores`` / ``score`` /
``ranking`` / ``maximum`` / ``centralization`` / ``hasFinished``
(networkit/centrality.pyx:46-100). Errors from the library come back as
``RuntimeError(nkg_last_error())``, the form ``except +`` gives the reference's
``std::runtime_error``.

The graph is a ``networkit_b200.Graph``; its in-adjacency is uploaded on the
first ``run()`` and kept while the graph is unchanged.
"""
from libc.stdint cimport uint8_t, uint32_t, uint64_t, UINT64_MAX

from networkit_b200._nkgpu cimport (
    nkg_graph, nkg_pr_params, nkg_stats, nkg_graph_create, nkg_graph_destroy, nkg_pagerank_run,
    nkg_ranking, nkg_cancel, nkg_sigint_cancels, nkg_last_error, NKG_PREC_FP64, NKG_NORM_L2,
    NKG_ERR_CANCELLED)
from libc.string cimport memset

import numpy as np

from networkit_b200.graph import Graph


cdef _raise_last():
    raise RuntimeError(nkg_last_error().decode("utf-8", "replace"))


cdef class PageRank:
    """PageRank(G, damp=0.85, tol=1e-8, normalized=False, distributeSinks=False)

    Compute PageRank as node centrality measure (networkit/centrality.pyx:1989-2008)."""

    cdef nkg_graph *_g
    cdef nkg_pr_params _p
    cdef object _G, _csr, _scores, _exists
    cdef uint64_t _iters
    cdef double _max
    cdef bint _hasRun
    cdef readonly dict lastStats

    def __cinit__(self, G, double damp=0.85, double tol=1e-8, bint normalized=False,
                  bint distributeSinks=False):
        if not isinstance(G, Graph):
            raise TypeError("G must be a networkit_b200.Graph")
        self._g = NULL
        self._G = G
        self._csr = None
        self._p.damp = damp
        self._p.tol = tol
        self._p.norm = NKG_NORM_L2            # PageRank.hpp:67
        self._p.normalized = normalized
        self._p.distribute_sinks = distributeSinks
        self._p.precision = NKG_PREC_FP64
        self._p.max_iterations = UINT64_MAX   # PageRank.hpp:64
        self._hasRun = False
        self._max = 1.0
        self.lastStats = {}

    def __dealloc__(self):
        if self._g != NULL:
            nkg_graph_destroy(self._g)
            self._g = NULL

    cdef _upload(self, csr):
        cdef const uint64_t[::1] ptr = np.ascontiguousarray(csr.in_ptr, np.uint64)
        cdef const uint32_t[::1] col = np.ascontiguousarray(csr.in_col, np.uint32)
        cdef const double[::1] wdeg = np.ascontiguousarray(csr.wdeg, np.float64)
        cdef const double[::1] w
        cdef const uint8_t[::1] ex
        cdef const uint32_t *colp = NULL
        cdef const double *wp = NULL
        cdef const uint8_t *exp_ = NULL
        cdef uint64_t arcs = col.shape[0]
        cdef nkg_graph *g = NULL
        if arcs:
            colp = &col[0]
        if csr.in_w is not None and arcs:
            w = np.ascontiguousarray(csr.in_w, np.float64)
            wp = &w[0]
        if csr.exists is not None:
            ex = np.ascontiguousarray(csr.exists, np.uint8)
            exp_ = &ex[0]
        if self._g != NULL:
            nkg_graph_destroy(self._g)
            self._g = NULL
        if nkg_graph_create(&g, csr.z, arcs, &ptr[0], colp, wp, &wdeg[0], exp_,
                            1 if csr.directed else 0) != 0:
            _raise_last()
        self._g = g
        self._csr = csr

    def run(self):
        """Executes the algorithm (PageRank::run, PageRank.cpp:20-104); returns self."""
        csr = self._G.inCSR()
        self._exists = csr.exists
        if csr.n == 0:
            # No nodes: nothing is iterated, as in the reference.
            self._scores = np.full(csr.z, np.inf)
            self._iters = 1
            self._max = 1.0
            self._hasRun = True
            return self
        if self._g == NULL or self._csr is not csr:
            self._upload(csr)
        scores = np.empty(csr.z, np.float64)
        cdef double[::1] s = scores
        cdef nkg_stats st
        memset(&st, 0, sizeof(st))           # no residual trace
        cdef uint64_t it = 0
        cdef double mx = 0.0
        cdef int rc
        cdef int got_sigint = 0
        # SIGINT cancels the run while it is in the library, as the
        # reference's SignalHandler does (PageRank.cpp:55); if another handle
        # already holds SIGINT, this run goes without.
        cdef bint routed = nkg_sigint_cancels(self._g, 1, NULL) == 0
        with nogil:                           # base.pyx:28
            rc = nkg_pagerank_run(self._g, &self._p, &s[0], &it, &mx, &st)
        if routed:
            nkg_sigint_cancels(self._g, 0, &got_sigint)
        if rc != 0:
            if rc == NKG_ERR_CANCELLED and got_sigint:
                # Aux::SignalHandling::InterruptException (SignalHandling.hpp:26-30)
                raise RuntimeError("Received CTRL+C/SIGINT")
            _raise_last()
        self._scores = scores
        self._iters = it
        self._max = mx
        self._hasRun = True
        self.lastStats = {"iterations": st.iterations, "residual": st.residual,
                          "ms_total": st.ms_total, "kernel_launches": st.kernel_launches,
                          "fp64_sweeps": st.fp64_sweeps}
        return self

    def cancel(self):
        """Ends a run in progress with RuntimeError (the SIGINT check of
        PageRank.cpp:55); callable from another thread."""
        if self._g != NULL:
            nkg_cancel(self._g)

    def hasFinished(self):
        return self._hasRun

    cdef _assureFinished(self):
        # Algorithm::assureFinished (Algorithm.hpp:40-43)
        if not self._hasRun:
            raise RuntimeError("Error, run must be called first")

    property norm:                            # centrality.pyx:2021-2027
        def __get__(self):
            return self._p.norm

        def __set__(self, norm):
            if norm not in (0, 1):
                raise ValueError("norm must be Norm.l1norm or Norm.l2norm")
            self._p.norm = norm

    property maxIterations:                   # centrality.pyx:2029-2037
        def __get__(self):
            return self._p.max_iterations

        def __set__(self, maxIterations):
            if maxIterations < 0:
                raise Exception("Max iterations cannot be a negative number.")
            self._p.max_iterations = maxIterations

    def numberOfIterations(self):
        self._assureFinished()
        return self._iters

    def scores(self):
        self._assureFinished()
        return self._scores.tolist()

    def scoresArray(self):
        self._assureFinished()
        return self._scores

    def score(self, v):
        self._assureFinished()
        if v < 0 or v >= self._scores.shape[0]:
            raise IndexError("vector::_M_range_check")
        return float(self._scores[v])

    def maximum(self):
        self._assureFinished()
        return self._max

    def rankingArrays(self):
        """ranking() as (ids uint64[n], scores float64[n]), sorted on the GPU."""
        self._assureFinished()
        n = self._csr.n if self._csr is not None else 0
        ids = np.empty(n, np.uint64)
        vals = np.empty(n, np.float64)
        if n == 0:
            return ids, vals
        cdef const double[::1] s = self._scores
        cdef uint64_t[::1] iv = ids
        cdef double[::1] vv = vals
        if nkg_ranking(self._g, &s[0], &iv[0], &vv[0]) != 0:
            _raise_last()
        return ids, vals

    def ranking(self):
        """(node, score) pairs, score descending, ties by node id ascending
        (Centrality.cpp:29-41)."""
        ids, vals = self.rankingArrays()
        return list(zip(ids.tolist(), vals.tolist()))

    def centralization(self):
        """Centrality::centralization (Centrality.cpp:58-75)."""
        self._assureFinished()
        s = self._scores if self._exists is None else self._scores[self._exists != 0]
        center = 0.0
        for x in s:
            if x > center:
                center = x
        max_score = self.maximum()
        return float(np.sum(center - s)) / float(np.sum(max_score - s))
