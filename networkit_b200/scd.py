"""Seeded (local) PageRank on the GPU: the mirror of ``networkit.scd``'s
``ApproximatePageRank`` and ``PageRankNibble`` (scd.pyx:87-151).

Both run on ``nkg_local_*`` (include/nkgpu.h): one warp per seed set, each in
the reference's FIFO push order, so the values are bit-identical to
ApproximatePageRank.cpp:18-55. ``PageRankNibble`` adds the sweep of
PageRankNibble.cpp:28-82 with ties of p/vol ordered by ascending node id (the
reference's unstable sort leaves that order open).

Both take every seed set of a call in one launch: ``run(seeds)`` of
PageRankNibble (one community per seed, SelectiveCommunityDetector.cpp:15-23)
and :meth:`ApproximatePageRank.runMany` fill the GPU with independent
problems.
"""
from __future__ import annotations

from typing import Dict, Iterable, List, Set, Tuple

import numpy as np

from . import _capi
from .graph import Graph, InCSR


def neighbour_csr(G) -> Tuple[int, np.ndarray, np.ndarray, object, object, bool]:
    """(z, row_ptr, col, w, exists, directed) in Graph::forNeighborsOf order:
    undirected graphs: the neighbour lists (the in-CSR); directed graphs: the
    out-lists in edge insertion order (Graph::addEdge appends to
    outEdges[u], Graph.cpp:549-596). A directed graph built from a CSR alone
    keeps no insertion order: its out-lists are ordered by target."""
    csr = G.inCSR() if isinstance(G, Graph) else G
    if not isinstance(csr, InCSR):
        raise TypeError("expected a networkit_b200 Graph or InCSR")
    if not csr.directed:
        return csr.z, csr.in_ptr, csr.in_col, csr.in_w, csr.exists, False
    if isinstance(G, Graph) and G._frozen_csr is None:
        s, d, w = G._edges()
        s = np.asarray(s, np.int64)
        order = np.argsort(s, kind="stable")
        counts = np.bincount(s, minlength=csr.z) if s.shape[0] else np.zeros(csr.z, np.int64)
        ptr = np.zeros(csr.z + 1, np.uint64)
        np.cumsum(counts, out=ptr[1:])
        ww = np.asarray(w, np.float64)[order] if G.isWeighted() else None
        return csr.z, ptr, np.asarray(d, np.int64)[order].astype(np.uint32), ww, csr.exists, True
    out_ptr, out_col, arc = csr.out_csr()
    ww = None if csr.in_w is None else csr.in_w[arc.astype(np.int64)]
    return csr.z, out_ptr, out_col, ww, csr.exists, True


class _Local:
    def __init__(self, G, alpha: float, epsilon: float):
        self._G = G
        self.alpha = float(alpha)
        self.epsilon = float(epsilon)
        self._dev = None
        # Pushes one problem may take (the reference has no bound);
        # nkg_local_run fails with NKG_ERR_TIMEOUT past it.
        self.maxPushes = _capi.UINT64_MAX

    def _device(self) -> _capi.DeviceLocal:
        if self._dev is None:
            z, ptr, col, w, ex, directed = neighbour_csr(self._G)
            self._dev = _capi.DeviceLocal(z, ptr, col, w, ex, directed)
        return self._dev


def _seed_list(seeds) -> List[int]:
    if isinstance(seeds, (int, np.integer)):
        return [int(seeds)]
    return sorted(set(int(s) for s in seeds))


class ApproximatePageRank(_Local):
    """ApproximatePageRank(G, alpha, epsilon=1e-12) (ApproximatePageRank.hpp:34).

    alpha: loop probability of the lazy random walk; epsilon: error
    tolerance."""

    def __init__(self, G, alpha: float, epsilon: float = 1e-12):
        super().__init__(G, alpha, epsilon)

    def run(self, seeds) -> List[Tuple[int, float]]:
        """Seed node or iterable of seed nodes -> list of (node, value) of
        every node in the result (ascending ids; the reference returns them
        in hash-map order)."""
        (nodes, vals), = self.runMany([seeds])
        return list(zip(nodes.tolist(), vals.tolist()))

    def runMany(self, seed_sets: Iterable) -> List[Tuple[np.ndarray, np.ndarray]]:
        """One independent run per entry (a node or an iterable of nodes),
        all in one launch: [(nodes ascending, values)]."""
        sets = [_seed_list(s) for s in seed_sets]
        supports, _, self.stats = self._device().run(sets, self.alpha, self.epsilon,
                                                     max_pushes=self.maxPushes)
        return supports


class PageRankNibble(_Local):
    """PageRankNibble(G, alpha, epsilon) (PageRankNibble.hpp:25, scd.pyx:143):
    a low-conductance cut around seeds from an approximate PageRank vector."""

    def run(self, seeds) -> Dict[int, Set[int]]:
        """SelectiveCommunityDetector::run: one community per seed."""
        sl = _seed_list(seeds)
        _, sets, self.stats = self._device().run(np.asarray(sl, np.int64), self.alpha,
                                                 self.epsilon, nibble=True,
                                                 max_pushes=self.maxPushes)
        return {s: set(c.tolist()) for s, c in zip(sl, sets)}

    def expandOneCommunity(self, seeds) -> Set[int]:
        """One community around a seed node or a set of seed nodes."""
        _, sets, self.stats = self._device().run([_seed_list(seeds)], self.alpha, self.epsilon,
                                                 nibble=True, max_pushes=self.maxPushes)
        return set(sets[0].tolist())

    def expandMany(self, seed_sets: Iterable) -> List[np.ndarray]:
        """One community per entry (a node or a set of nodes), all in one
        launch; each ascending."""
        sets_in = [_seed_list(s) for s in seed_sets]
        _, sets, self.stats = self._device().run(sets_in, self.alpha, self.epsilon, nibble=True,
                                                 max_pushes=self.maxPushes)
        return sets
