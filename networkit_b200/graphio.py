"""Graph file input for the PageRank path: the NetworkitBinaryGraph format.

Mirrors the part of ``networkit.graphio`` (graphio.pyx:145-151
``NetworkitBinaryReader``, :724-747 ``Format``, :786-812 ``readGraph``) that
loads the reference's own binary format, decoded by host C++/OpenMP
(``_lib/libnkgen.so``, one thread per file chunk) straight into the in-CSR the
device graph is built from - no intermediate edge list, no Graph object.

The adjacency is the one NetworkitBinaryReader.cpp:107-231 stores: directed
graphs take each node's transpose list as its in-row and its out list for the
degrees; undirected graphs take the out list followed by the transpose list
without self-loops, in file order (which is the reference's summation order).
"""
from __future__ import annotations

import ctypes as C
import enum
import os

import numpy as np

from . import build as _build
from .graph import Graph, InCSR

_lib = None


class _Graph(C.Structure):
    _fields_ = [
        ("z", C.c_uint64),
        ("arcs", C.c_uint64),
        ("in_ptr", C.POINTER(C.c_uint64)),
        ("in_col", C.POINTER(C.c_uint32)),
        ("outdeg", C.POINTER(C.c_uint32)),
        ("w", C.POINTER(C.c_double)),
        ("wdeg", C.POINTER(C.c_double)),
        ("exists", C.POINTER(C.c_uint8)),
        ("directed", C.c_int),
        ("weighted", C.c_int),
    ]


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_build.GEN_LIB):
            _build.build_gen()
        L = C.CDLL(_build.GEN_LIB)
        L.nkgen_io_last_error.restype = C.c_char_p
        L.nkgen_graph_free.argtypes = [C.POINTER(_Graph)]
        L.nkgen_read_nkbg.argtypes = [C.c_char_p, C.c_int, C.POINTER(_Graph)]
        _lib = L
    return _lib


def _array(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def read_nkbg(path: str, nthreads: int = 0) -> InCSR:
    """Decode a NetworkitBinaryGraph file into an :class:`InCSR`.

    Raises ``RuntimeError`` with the decoder's message for a file that is not
    in the format (wrong magic, sections outside the file, truncated lists,
    neighbour ids >= the node count)."""
    L = _load()
    g = _Graph()
    if L.nkgen_read_nkbg(os.fsencode(path), int(nthreads), C.byref(g)) != 0:
        raise RuntimeError(L.nkgen_io_last_error().decode())
    try:
        z, m = int(g.z), int(g.arcs)
        in_ptr = np.ctypeslib.as_array(g.in_ptr, shape=(z + 1,)).copy()
        in_col = _array(g.in_col, m, np.uint32)
        in_w = _array(g.w, m, np.float64) if g.weighted else None
        wdeg = _array(g.wdeg, z, np.float64)
        outdeg = _array(g.outdeg, z, np.uint32)
        exists = _array(g.exists, z, np.uint8)
        directed = bool(g.directed)
    finally:
        L.nkgen_graph_free(C.byref(g))
    n = int(exists.sum())
    return InCSR(z, n, in_ptr, in_col, in_w, wdeg, outdeg, None if n == z else exists, directed)


class NetworkitBinaryReader:
    """``networkit.graphio.NetworkitBinaryReader``: ``read(path)`` returns a
    :class:`~networkit_b200.graph.Graph` over the decoded in-CSR."""

    def __init__(self, nthreads: int = 0):
        self._nthreads = int(nthreads)

    def read(self, path: str) -> Graph:
        return Graph.fromInCSR(read_nkbg(path, self._nthreads))


class Format(enum.Enum):
    """The file formats this reader understands (a subset of graphio.pyx:724)."""

    NetworkitBinary = 1


def getReader(fileformat, *kargs, **kwargs):
    if fileformat == Format.NetworkitBinary:
        return NetworkitBinaryReader(*kargs, **kwargs)
    raise ValueError(f"unsupported format: {fileformat}")


def readGraph(path, fileformat, *kargs, **kwargs) -> Graph:
    """``networkit.graphio.readGraph``: a missing file raises ``IOError``, a
    file the reader rejects raises ``IOError`` naming the format and the
    reader's message (graphio.pyx:799-811)."""
    reader = getReader(fileformat, *kargs, **kwargs)
    if "~" in path:
        path = os.path.expanduser(path)
    if not os.path.isfile(path):
        raise IOError(f"{path} is not a file")
    try:
        return reader.read(path)
    except Exception as e:
        raise IOError(f"{path} is not a valid {fileformat} file: {e}") from e
