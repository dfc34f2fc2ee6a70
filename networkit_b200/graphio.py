"""Graph file input for the PageRank path: the NetworkitBinaryGraph format.

Mirrors the part of ``networkit.graphio`` (graphio.pyx:145-151
``NetworkitBinaryReader``, :153-159 ``NetworkitBinaryWriter``, :724-747
``Format``, :786-812 ``readGraph``) that reads and writes the reference's own
binary format, decoded and encoded by host C++/OpenMP
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
        _u64 = C.POINTER(C.c_uint64)
        _u32 = C.POINTER(C.c_uint32)
        _f64 = C.POINTER(C.c_double)
        L.nkgen_write_nkbg.argtypes = [C.c_char_p, C.c_uint64, C.c_int, _u64, _u32, _f64, _u64,
                                       _u32, _f64, C.c_uint64, C.c_int, C.c_int]
        _lib = L
    return _lib


def _array(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def decode_nkbg_device(data, device: int = -1):
    """Decode a NetworkitBinaryGraph file's bytes on the GPU (nkg_nkbg_decode)
    into an :class:`InCSR` on the host: the same arrays :func:`read_nkbg`
    returns, from the device decoder (used to check one against the other).
    Returns (csr, device milliseconds of the decode)."""
    from . import _capi

    arr = np.ascontiguousarray(np.frombuffer(data, np.uint8) if not isinstance(data, np.ndarray)
                               else data, np.uint8)
    L = _capi.lib()
    z, m = C.c_uint64(0), C.c_uint64(0)
    d, wt = C.c_int(0), C.c_int(0)
    ms = C.c_double(0.0)
    buf = C.c_void_p(arr.ctypes.data)
    _capi.check(L.nkg_nkbg_decode(buf, arr.shape[0], 0, int(device), C.byref(z), C.byref(m),
                                  C.byref(d), C.byref(wt), None, None, None, None, None, None,
                                  None))
    z, m = int(z.value), int(m.value)
    in_ptr = np.empty(z + 1, np.uint64)
    in_col = np.empty(max(m, 1), np.uint32)
    w = np.empty(max(m, 1), np.float64) if wt.value else None
    wdeg = np.empty(z, np.float64)
    outdeg = np.empty(z, np.uint32)
    ex = np.empty(z, np.uint8)
    p = lambda a, t: None if a is None else a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    _capi.check(L.nkg_nkbg_decode(buf, arr.shape[0], 0, int(device), None, None, None, None,
                                  p(in_ptr, C.c_uint64), p(in_col, C.c_uint32),
                                  p(w, C.c_double), p(wdeg, C.c_double), p(outdeg, C.c_uint32),
                                  p(ex, C.c_uint8), C.byref(ms)))
    exists = None if ex.all() else ex
    csr = InCSR(z, int(ex.sum()), in_ptr, in_col[:m], None if w is None else w[:m], wdeg,
                outdeg, exists, bool(d.value))
    return csr, float(ms.value)


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


class NetworkitBinaryWeights(enum.IntEnum):
    """NetworkitBinaryWriter.hpp:17-24."""

    none = 0
    unsignedFormat = 1
    signedFormat = 2
    doubleFormat = 3
    floatFormat = 4
    autoDetect = 5


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def write_nkbg(path: str, n: int, out_ptr, out_col, out_w=None, in_ptr=None, in_col=None,
               in_w=None, directed: bool = False, chunks: int = 32,
               weights: int = NetworkitBinaryWeights.autoDetect, nthreads: int = 0) -> None:
    """Write a graph given as its out-lists (outEdges order; neighbour lists
    for undirected graphs) and, when directed, its in-lists (inEdges order)
    in the NetworkitBinaryGraph format, byte for byte as the reference's
    NetworkitBinaryWriter."""
    c = lambda a, t: None if a is None else np.ascontiguousarray(a, t)  # noqa: E731
    op, oc, ow = c(out_ptr, np.uint64), c(out_col, np.uint32), c(out_w, np.float64)
    ip, ic, iw = c(in_ptr, np.uint64), c(in_col, np.uint32), c(in_w, np.float64)
    L = _load()
    if L.nkgen_write_nkbg(os.fsencode(path), int(n), int(bool(directed)), _p(op, C.c_uint64),
                          _p(oc, C.c_uint32), _p(ow, C.c_double), _p(ip, C.c_uint64),
                          _p(ic, C.c_uint32), _p(iw, C.c_double), int(chunks), int(weights),
                          int(nthreads)) != 0:
        raise RuntimeError(L.nkgen_io_last_error().decode())


class NetworkitBinaryWriter:
    """``networkit.graphio.NetworkitBinaryWriter(chunks=32, weightsType=autoDetect)``
    (NetworkitBinaryWriter.hpp:34): ``write(G, path)`` for a
    :class:`~networkit_b200.graph.Graph` without deleted nodes."""

    def __init__(self, chunks: int = 32, weightsType=NetworkitBinaryWeights.autoDetect):
        self._chunks = int(chunks)
        self._weights = int(weightsType)

    def write(self, G: Graph, path: str) -> None:
        from .scd import neighbour_csr

        csr = G.inCSR()
        if csr.exists is not None:
            raise RuntimeError("the binary format numbers only existing nodes: remove the "
                               "deleted ids first (the reference writer does not round trip them)")
        z, optr, ocol, ow, _, directed = neighbour_csr(G)
        if directed:
            write_nkbg(path, z, optr, ocol, ow, csr.in_ptr, csr.in_col, csr.in_w, True,
                       self._chunks, self._weights)
        else:
            write_nkbg(path, z, optr, ocol, ow, directed=False, chunks=self._chunks,
                       weights=self._weights)


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
