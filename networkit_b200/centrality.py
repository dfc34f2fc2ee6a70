"""``networkit.centrality.PageRank`` (and the centralities that share its
sweep: EigenvectorCentrality, KatzCentrality) on the B200 path.

Mirrors the reference's Cython surface for this path
(networkit/centrality.pyx:24-100 Centrality, :1970-2037 Norm/PageRank,
networkit/base.pyx:3-69 Algorithm) with the same names, argument meanings and
error behaviour, plus the ``distributeSinks`` flag and a ``precision`` choice.
Every run goes through libnkgpu.so (include/nkgpu.h); there is no CPU path.
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np

from . import _capi
from .graph import Graph


def _run_interruptible(dg, call):
    """Run `call` (a library run on the handle dg) with SIGINT routed to
    dg's cancel flag, as the reference's SignalHandler routes it for the
    length of a run (SignalHandling.cpp:29-60): Ctrl-C ends the run at its
    next check with RuntimeError("Received CTRL+C/SIGINT"), the message of
    Aux::SignalHandling::InterruptException. If another handle holds SIGINT
    already, the run goes without."""
    try:
        dg.sigint_cancels(True)
        routed = True
    except _capi.NkgError:
        routed = False
    try:
        return call()
    except _capi.NkgError as e:
        got = dg.sigint_cancels(False) if routed else False
        routed = False
        if e.code == _capi.NKG_ERR_CANCELLED and got:
            raise RuntimeError("Received CTRL+C/SIGINT") from None
        raise
    finally:
        if routed:
            dg.sigint_cancels(False)


class Algorithm:
    """Abstract base class for algorithms (networkit/base.pyx:3-69)."""

    def __init__(self, *args, **kwargs):
        if type(self) is Algorithm:
            raise RuntimeError("Error, you may not use Algorithm directly, use a sub-class instead")
        self._hasRun = False

    def run(self):
        raise NotImplementedError

    def hasFinished(self) -> bool:
        return self._hasRun

    def _assureFinished(self):
        # Algorithm::assureFinished (include/networkit/base/Algorithm.hpp:40-43)
        if not self._hasRun:
            raise RuntimeError("Error, run must be called first")


class Centrality(Algorithm):
    """Abstract base class for centrality measures (networkit/centrality.pyx:34-100)."""

    def __init__(self, *args, **kwargs):
        if type(self) is Centrality:
            raise RuntimeError("Error, you may not use Centrality directly, use a sub-class instead")
        super().__init__()
        self._scores: Optional[np.ndarray] = None
        self._exists: Optional[np.ndarray] = None

    def scores(self) -> List[float]:
        """List of all scores, indexed by node id (Centrality.cpp:43-46)."""
        self._assureFinished()
        return self._scores.tolist()

    def scoresArray(self) -> np.ndarray:
        """The scores as a float64 numpy array (no list conversion)."""
        self._assureFinished()
        return self._scores

    def score(self, v: int) -> float:
        """Score of node v; std::vector::at semantics (Centrality.cpp:24-27)."""
        self._assureFinished()
        if v < 0 or v >= self._scores.shape[0]:
            raise IndexError("vector::_M_range_check")
        return float(self._scores[v])

    def ranking(self) -> List[Tuple[int, float]]:
        """(node, score) pairs, score descending, ties by node id ascending
        (Centrality.cpp:29-41); sorted on the GPU."""
        ids, vals = self.rankingArrays()
        return list(zip(ids.tolist(), vals.tolist()))

    def rankingArrays(self):
        raise NotImplementedError

    def maximum(self) -> float:
        raise RuntimeError("Not implemented: Compute the maximum centrality score in the "
                           "respective centrality subclass.")

    def centralization(self) -> float:
        """Centrality::centralization (Centrality.cpp:58-75)."""
        self._assureFinished()
        s = self._scores if self._exists is None else self._scores[self._exists != 0]
        center = 0.0
        for x in s:
            if x > center:
                center = x
        max_score = self.maximum()
        diff1 = float(np.sum(center - s))
        diff2 = float(np.sum(max_score - s))
        return diff1 / diff2


class Norm:
    """PageRank::Norm (PageRank.hpp:31; centrality.pyx:1970-1979)."""

    l1norm = 0
    l2norm = 1


_PRECISIONS = {
    "fp64": _capi.NKG_PREC_FP64,
    "fp32-refine": _capi.NKG_PREC_FP32_REFINE,
    "fp32": _capi.NKG_PREC_FP32,
}


class PageRank(Centrality):
    """Compute PageRank as node centrality measure.

    PageRank(G, damp=0.85, tol=1e-8, normalized=False, distributeSinks=False)
    (centrality.pyx:1989-2008; PageRank.hpp:40).

    Parameters
    ----------
    G : Graph
        Graph to be processed.
    damp : float
        Damping factor of the PageRank algorithm.
    tol : float
        Error tolerance for PageRank iteration.
    normalized : bool
        Divide by the lower bound of the scores (PageRank.cpp:81-92).
    distributeSinks : bool
        Spread the score of out-degree-0 nodes uniformly every iteration.
        False keeps the reference's semantics.
    precision : "fp64" (default, the reference arithmetic), "fp32-refine"
        (FP32 sweeps corrected by FP64 residual sweeps) or "fp32".
    device : CUDA device ordinal (-1: current).
    """

    def __init__(self, G: Graph, damp: float = 0.85, tol: float = 1e-8,
                 normalized: bool = False, distributeSinks: bool = False,
                 precision: str = "fp64", device: int = -1):
        super().__init__()
        if not isinstance(G, Graph):
            raise TypeError("G must be a networkit_b200.Graph")
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        self._G = G
        self._damp = float(damp)
        self._tol = float(tol)
        self._normalized = bool(normalized)
        self._distribute = bool(distributeSinks)
        self._precision = precision
        self._device = int(device)
        self._norm = Norm.l2norm            # PageRank.hpp:67
        self._maxIterations = _capi.UINT64_MAX  # PageRank.hpp:64
        self._iterations = 0
        self._max = 1.0
        self._dg: Optional[_capi.DeviceGraph] = None
        self._dg_key = None
        self.lastStats: dict = {}

    # -- properties (centrality.pyx:2021-2037) ---------------------------------
    @property
    def norm(self) -> int:
        return self._norm

    @norm.setter
    def norm(self, norm: int):
        if norm not in (Norm.l1norm, Norm.l2norm):
            raise ValueError("norm must be Norm.l1norm or Norm.l2norm")
        self._norm = int(norm)

    @property
    def maxIterations(self) -> int:
        return self._maxIterations

    @maxIterations.setter
    def maxIterations(self, maxIterations: int):
        if maxIterations < 0:
            raise Exception("Max iterations cannot be a negative number.")
        self._maxIterations = int(maxIterations)

    # -- run ------------------------------------------------------------------
    def _device_graph(self) -> _capi.DeviceGraph:
        csr = self._G.inCSR()
        key = id(csr)
        if self._dg is None or self._dg_key != key:
            self._dg = _capi.DeviceGraph(csr, device=self._device)
            self._dg_key = key
            self._csr = csr
        return self._dg

    def run(self, teleport=None):
        """Executes the algorithm (PageRank::run, PageRank.cpp:20-104); returns self.

        teleport: optional personalised teleport distribution (one entry per
        node id, summing to 1 over existing nodes)."""
        csr = self._G.inCSR()
        self._exists = csr.exists
        if csr.n == 0:
            # Nothing to iterate over: no nodes, as in the reference.
            self._scores = np.full(csr.z, np.inf)
            self._iterations = 1
            self._max = 1.0
            self._hasRun = True
            return self
        dg = self._device_graph()
        p = dg.params(self._damp, self._tol, self._norm, self._normalized, self._distribute,
                      _PRECISIONS[self._precision], self._maxIterations)
        scores, it, mx, st = _run_interruptible(dg, lambda: dg.run(p, teleport))
        self._scores = scores
        self._iterations = it
        self._max = mx
        self.lastStats = st
        self._hasRun = True
        return self

    def cancel(self):
        """Stop a run in progress (or the next run) with RuntimeError: the
        SIGINT check of PageRank.cpp:55, callable from another thread."""
        if self._dg is not None:
            self._dg.cancel()

    def numberOfIterations(self) -> int:
        """Number of iterations performed (PageRank.hpp:58-61)."""
        self._assureFinished()
        return self._iterations

    def maximum(self) -> float:
        """PageRank::maximum (PageRank.cpp:106-108): 1.0, or the largest score
        when normalized."""
        self._assureFinished()
        return self._max

    def rankingArrays(self):
        """ranking() as (ids uint64[n], scores float64[n]) arrays."""
        self._assureFinished()
        if self._scores.shape[0] == 0:
            return np.zeros(0, np.uint64), np.zeros(0)
        return self._device_graph().ranking(self._scores)


class _SweepCentrality(Centrality):
    """Shared upload / ranking of the centralities that run the pull sweep."""

    def __init__(self, G: Graph, device: int = -1):
        super().__init__()
        if not isinstance(G, Graph):
            raise TypeError("G must be a networkit_b200.Graph")
        self._G = G
        self._device = int(device)
        self._dg: Optional[_capi.DeviceGraph] = None
        self._dg_key = None
        self._iterations = 0
        self.lastStats: dict = {}

    def _device_graph(self) -> _capi.DeviceGraph:
        csr = self._G.inCSR()
        if self._dg is None or self._dg_key != id(csr):
            self._dg = _capi.DeviceGraph(csr, device=self._device)
            self._dg_key = id(csr)
            self._csr = csr
        return self._dg

    def _finish(self, scores, it, st):
        self._scores = scores
        self._iterations = it
        self.lastStats = st
        self._hasRun = True
        return self

    def numberOfIterations(self) -> int:
        """Iterations of the last run (the reference keeps no count)."""
        self._assureFinished()
        return self._iterations

    def rankingArrays(self):
        self._assureFinished()
        if self._scores.shape[0] == 0:
            return np.zeros(0, np.uint64), np.zeros(0)
        return self._device_graph().ranking(self._scores)


class EigenvectorCentrality(_SweepCentrality):
    """Leading eigenvector of the adjacency matrix, normalised in the 2-norm.

    EigenvectorCentrality(G, tol=1e-9) (centrality.pyx:1950-1968;
    EigenvectorCentrality.cpp:20-60): power iteration over the in-adjacency
    with the edge weights until the 2-norm of the product changes by at most
    tol."""

    def __init__(self, G: Graph, tol: float = 1e-9, device: int = -1):
        super().__init__(G, device)
        self._tol = float(tol)

    def run(self):
        csr = self._G.inCSR()
        self._exists = csr.exists
        if csr.n == 0:
            return self._finish(np.ones(csr.z), 0, {})
        scores, it, st = self._device_graph().eigenvector(self._tol)
        return self._finish(scores, it, st)


class EdgeDirection:
    """KatzCentrality::edgeDirection (KatzCentrality.hpp: InEdges = 0, OutEdges = 1)."""

    InEdges = 0
    OutEdges = 1


class KatzCentrality(_SweepCentrality):
    """Katz centrality.

    KatzCentrality(G, alpha=0, beta=0.1, tol=1e-8) (centrality.pyx:1678-1712;
    KatzCentrality.cpp:20-72). alpha 0 picks 1 / (1 + maximum degree); a
    negative alpha raises like the reference. ``edgeDirection`` counts in-edges
    (default) or out-edges."""

    def __init__(self, G: Graph, alpha: float = 0, beta: float = 0.1, tol: float = 1e-8,
                 device: int = -1):
        if alpha < 0:
            raise RuntimeError("Alpha must be non negative.")
        super().__init__(G, device)
        self._alpha = float(alpha)
        self._beta = float(beta)
        self._tol = float(tol)
        self._edgeDirection = EdgeDirection.InEdges

    @property
    def edgeDirection(self) -> int:
        return self._edgeDirection

    @edgeDirection.setter
    def edgeDirection(self, d: int):
        if d not in (EdgeDirection.InEdges, EdgeDirection.OutEdges):
            raise ValueError("edgeDirection must be EdgeDirection.InEdges or OutEdges")
        self._edgeDirection = int(d)

    def run(self):
        csr = self._G.inCSR()
        self._exists = csr.exists
        if csr.n == 0:
            return self._finish(np.ones(csr.z), 0, {})
        scores, it, st = self._device_graph().katz(self._alpha, self._beta, self._tol,
                                                   self._edgeDirection)
        return self._finish(scores, it, st)


def rankPerNode(ranking):
    """For each node (by id), its position in ``ranking``; tied scores share
    the position of the first of them (networkit/centrality.pyx:2197-2219)."""
    n_nodes = len(ranking)
    ranking_id = [0] * n_nodes
    for index, pair in enumerate(ranking):
        ranking_id[pair[0]] = index
    for index, pair in enumerate(ranking):
        if index == 0:
            continue
        if pair[1] == ranking[index - 1][1]:
            prev_node = ranking[index - 1][0]
            ranking_id[pair[0]] = ranking_id[prev_node]
    return ranking_id
