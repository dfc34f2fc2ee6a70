"""Host-side graph container feeding the PageRank boundary.

``Graph`` mirrors the part of ``networkit.Graph`` the PageRank path touches
(include/networkit/graph/Graph.hpp:991 ctor, :1144 removeNode, :1268 addEdge,
:1207 degree, :1245 weightedDegree) and produces the in-adjacency CSR that the
reference's ``Graph::forInEdgesOf`` walks (Graph.hpp:1917-1938):

* directed graphs: row u lists the sources of u's in-arcs (``inEdges[u]``),
* undirected graphs: row u lists all neighbours (``outEdges[u]``; both
  directions are stored and a self-loop is stored once, Graph.cpp:549-596),

each row in edge insertion order, which is the reference's storage order and
therefore its summation order.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np


@dataclass
class InCSR:
    """In-adjacency CSR plus the per-node data PageRank reads.

    z       upperNodeIdBound
    n       numberOfNodes (existing nodes)
    in_ptr  uint64[z+1]; in_col uint32[arcs]; in_w float64[arcs] or None
    wdeg    float64[z]  weightedDegree(u) (PageRank.cpp:29-30)
    outdeg  uint32[z]   degree(u): number of out-arcs (Graph.hpp:1207)
    exists  uint8[z] or None (all nodes exist)
    """

    z: int
    n: int
    in_ptr: np.ndarray
    in_col: np.ndarray
    in_w: Optional[np.ndarray]
    wdeg: np.ndarray
    outdeg: np.ndarray
    exists: Optional[np.ndarray]
    directed: bool

    @property
    def arcs(self) -> int:
        return int(self.in_col.shape[0])

    @property
    def weighted(self) -> bool:
        return self.in_w is not None

    def out_csr(self):
        """Out-adjacency (row v lists the targets of v's out-arcs) with, for
        every out-arc, the index of the matching in-arc. Used by the adjoint."""
        rows = np.repeat(np.arange(self.z, dtype=np.uint32), np.diff(self.in_ptr).astype(np.int64))
        order = np.argsort(self.in_col, kind="stable")
        out_col = rows[order]
        counts = np.bincount(self.in_col, minlength=self.z).astype(np.uint64)
        out_ptr = np.zeros(self.z + 1, np.uint64)
        np.cumsum(counts, out=out_ptr[1:])
        return out_ptr, out_col.astype(np.uint32), order.astype(np.uint64)


def concat_in_csr(csrs):
    """Block-diagonal union of unweighted in-CSRs without deleted nodes (the
    input of the many-graph batch): graph i's node v becomes
    node_offsets[i] + v. Returns (InCSR, node_offsets uint64[len + 1])."""
    offs = np.zeros(len(csrs) + 1, np.uint64)
    for i, c in enumerate(csrs):
        if c.exists is not None and not np.all(c.exists):
            raise ValueError("graphs of a batch must not have deleted nodes")
        offs[i + 1] = offs[i] + np.uint64(c.z)
    arc_offs = np.cumsum([0] + [c.arcs for c in csrs]).astype(np.uint64)
    z = int(offs[-1])
    in_ptr = np.empty(z + 1, np.uint64)
    in_col = np.empty(int(arc_offs[-1]), np.uint32)
    outdeg = np.empty(z, np.uint32)
    for i, c in enumerate(csrs):
        a, b = int(offs[i]), int(offs[i + 1])
        in_ptr[a:b] = c.in_ptr[:-1].astype(np.uint64) + arc_offs[i]
        in_col[int(arc_offs[i]):int(arc_offs[i + 1])] = c.in_col.astype(np.uint64) + offs[i]
        outdeg[a:b] = c.outdeg
    in_ptr[z] = arc_offs[-1]
    directed = any(c.directed for c in csrs)
    return InCSR(z, z, in_ptr, in_col, None, outdeg.astype(np.float64), outdeg, None,
                 directed), offs


def in_csr_from_edges(z, src, dst, w=None, directed=False, exists=None) -> InCSR:
    """Build the in-CSR of a graph whose edges were inserted in the given
    order (Graph::addEdge, Graph.cpp:549-596)."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    m = src.shape[0]
    if w is not None:
        w = np.asarray(w, dtype=np.float64)
    t = np.arange(m, dtype=np.int64)
    if directed:
        rows, cols, times, ws = dst, src, t, w
        out_rows, out_w = src, w
    else:
        nl = src != dst
        rows = np.concatenate([src, dst[nl]])
        cols = np.concatenate([dst, src[nl]])
        times = np.concatenate([t, t[nl]])
        ws = None if w is None else np.concatenate([w, w[nl]])
        out_rows, out_w = None, None
    order = np.lexsort((times, rows)) if rows.shape[0] else np.zeros(0, np.int64)
    in_col = cols[order].astype(np.uint32)
    in_w = None if ws is None else np.ascontiguousarray(ws[order])
    counts = np.bincount(rows, minlength=z) if rows.shape[0] else np.zeros(z, np.int64)
    in_ptr = np.zeros(z + 1, np.uint64)
    np.cumsum(counts, out=in_ptr[1:])
    if directed:
        outdeg = np.bincount(out_rows, minlength=z).astype(np.uint32) if m else np.zeros(z, np.uint32)
        if out_w is None:
            wdeg = outdeg.astype(np.float64)
        else:
            # Sequential per-node sums in insertion order (Graph.cpp:426-452).
            wdeg = np.bincount(out_rows, weights=out_w, minlength=z) if m else np.zeros(z)
    else:
        outdeg = counts.astype(np.uint32)
        if in_w is None:
            wdeg = outdeg.astype(np.float64)
        else:
            wdeg = np.bincount(rows[order], weights=in_w, minlength=z) if m else np.zeros(z)
    ex = None
    n = z
    if exists is not None:
        ex = np.ascontiguousarray(exists, np.uint8)
        n = int(np.count_nonzero(ex))
        if n == z:
            ex = None
    return InCSR(z, n, in_ptr, in_col, in_w, np.ascontiguousarray(wdeg, np.float64),
                 np.ascontiguousarray(outdeg, np.uint32), ex, bool(directed))


class Graph:
    """Minimal mirror of ``networkit.Graph`` for the PageRank path.

    Graph(n=0, weighted=False, directed=False) (Graph.hpp:991). Edges are kept
    in insertion order; ``addEdge`` performs no duplicate check, like the
    reference's (Graph.cpp:549).
    """

    def __init__(self, n: int = 0, weighted: bool = False, directed: bool = False):
        if n < 0:
            raise ValueError("number of nodes must be non-negative")
        self._z = int(n)
        self._weighted = bool(weighted)
        self._directed = bool(directed)
        self._src: list = []
        self._dst: list = []
        self._w: list = []
        self._bulk = []  # list of (src, dst, w) numpy chunks appended in order
        self._deleted: set = set()
        self._csr_cache: Optional[InCSR] = None
        self._frozen_csr: Optional[InCSR] = None

    # -- construction -----------------------------------------------------
    @classmethod
    def fromInCSR(cls, csr: InCSR) -> "Graph":
        """Wrap an already-built in-CSR (generators and readers produce it)."""
        g = cls(csr.z, csr.weighted, csr.directed)
        g._frozen_csr = csr
        if csr.exists is not None:
            g._deleted = set(np.flatnonzero(csr.exists == 0).tolist())
        return g

    def _mutable(self):
        if self._frozen_csr is not None:
            raise RuntimeError("graph was built from a CSR and is read-only")
        self._csr_cache = None

    def addNode(self) -> int:
        self._mutable()
        self._z += 1
        return self._z - 1

    def addNodes(self, k: int) -> int:
        self._mutable()
        self._z += int(k)
        return self._z - 1

    def removeNode(self, v: int) -> None:
        """Graph::removeNode: the node must have no incident edges here."""
        self._mutable()
        self._check_node(v)
        self._deleted.add(int(v))

    def restoreNode(self, v: int) -> None:
        self._mutable()
        self._deleted.discard(int(v))

    def _check_node(self, v):
        if v < 0 or v >= self._z or v in self._deleted:
            raise RuntimeError(f"node {v} does not exist")

    def addEdge(self, u: int, v: int, w: float = 1.0) -> None:
        self._mutable()
        self._check_node(u)
        self._check_node(v)
        self._src.append(int(u))
        self._dst.append(int(v))
        self._w.append(float(w))

    def addEdges(self, src, dst, w=None) -> None:
        """Append many edges at once, in array order."""
        self._mutable()
        src = np.asarray(src, dtype=np.int64)
        dst = np.asarray(dst, dtype=np.int64)
        if src.shape != dst.shape:
            raise ValueError("src and dst differ in length")
        if src.size and (src.min() < 0 or dst.min() < 0 or max(src.max(), dst.max()) >= self._z):
            raise RuntimeError("edge endpoint out of range")
        wa = np.ones(src.shape[0]) if w is None else np.asarray(w, dtype=np.float64)
        self._flush_lists()
        self._bulk.append((src, dst, wa))

    def _flush_lists(self):
        if self._src:
            self._bulk.append((np.asarray(self._src, np.int64), np.asarray(self._dst, np.int64),
                               np.asarray(self._w, np.float64)))
            self._src, self._dst, self._w = [], [], []

    def _edges(self):
        self._flush_lists()
        if not self._bulk:
            return (np.zeros(0, np.int64),) * 2 + (np.zeros(0),)
        if len(self._bulk) > 1:
            s = np.concatenate([b[0] for b in self._bulk])
            d = np.concatenate([b[1] for b in self._bulk])
            w = np.concatenate([b[2] for b in self._bulk])
            self._bulk = [(s, d, w)]
        return self._bulk[0]

    # -- properties ---------------------------------------------------------
    def numberOfNodes(self) -> int:
        return self._z - len(self._deleted)

    def upperNodeIdBound(self) -> int:
        return self._z

    def numberOfEdges(self) -> int:
        if self._frozen_csr is not None:
            c = self._frozen_csr
            if c.directed:
                return c.arcs
            loops = int(np.count_nonzero(
                c.in_col == np.repeat(np.arange(c.z, dtype=np.uint32),
                                      np.diff(c.in_ptr).astype(np.int64))))
            return (c.arcs - loops) // 2 + loops
        return int(self._edges()[0].shape[0])

    def isDirected(self) -> bool:
        return self._directed

    def isWeighted(self) -> bool:
        return self._weighted

    def hasNode(self, v: int) -> bool:
        return 0 <= v < self._z and v not in self._deleted

    def degree(self, v: int) -> int:
        return int(self.inCSR().outdeg[v])

    def weightedDegree(self, v: int) -> float:
        return float(self.inCSR().wdeg[v])

    def iterNodes(self):
        return (v for v in range(self._z) if v not in self._deleted)

    # -- boundary input -------------------------------------------------------
    def inCSR(self) -> InCSR:
        """The in-adjacency CSR the PageRank boundary consumes."""
        if self._frozen_csr is not None:
            return self._frozen_csr
        if self._csr_cache is None:
            s, d, w = self._edges()
            exists = None
            if self._deleted:
                exists = np.ones(self._z, np.uint8)
                exists[list(self._deleted)] = 0
            self._csr_cache = in_csr_from_edges(self._z, s, d, w if self._weighted else None,
                                                self._directed, exists)
        return self._csr_cache
