"""NetworkitBinaryGraph decoding (networkit_b200.graphio) against the
adjacency the reference's NetworkitBinaryReader builds from the same files
(NetworkitBinaryReader.cpp:19-235; fixtures written by the reference's
NetworkitBinaryWriter and read back by its reader, tests/golden/make_golden.py).

Bar: bit-exact in-CSR, weights, weighted degrees, degrees, node flags and
graph kind, for every weight encoding of the format."""
import glob
import os
import struct

import numpy as np
import pytest

from networkit_b200 import graphio

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("in_ptr", "in_col", "in_w", "wdeg", "outdeg", "exists", "directed", "weighted")
FORMAT_CASES = ["unsigned_dir", "signed_undir", "double_undir", "float_dir", "none_undir",
                "none_dir"]
GRAPH_CASES = sorted(os.path.basename(p)[:-5] for p in glob.glob(os.path.join(HERE, "*.nkbg"))
                     if not os.path.basename(p).startswith("nkbg_"))


def compare(csr, ref):
    np.testing.assert_array_equal(csr.in_ptr, ref["in_ptr"])
    np.testing.assert_array_equal(csr.in_col, ref["in_col"])
    if bool(ref["weighted"]):
        assert csr.in_w is not None
        np.testing.assert_array_equal(csr.in_w.view(np.uint64), ref["in_w"].view(np.uint64))
    else:
        assert csr.in_w is None
    np.testing.assert_array_equal(csr.wdeg.view(np.uint64), ref["wdeg"].view(np.uint64))
    np.testing.assert_array_equal(csr.outdeg, ref["outdeg"])
    ex = np.ones(csr.z, np.uint8) if csr.exists is None else csr.exists
    np.testing.assert_array_equal(ex, ref["exists"])
    assert csr.directed == bool(ref["directed"])
    assert csr.weighted == bool(ref["weighted"])
    assert csr.z == ref["exists"].shape[0]


def features(path):
    with open(path, "rb") as f:
        return struct.unpack("<Q", f.read(24)[16:24])[0]


@pytest.mark.parametrize("name", GRAPH_CASES)
def test_reference_test_graphs(name):
    d = np.load(os.path.join(HERE, f"{name}.npz"))
    ref = {k: d["nkbg_" + k] for k in FIELDS}
    compare(graphio.read_nkbg(os.path.join(HERE, f"{name}.nkbg")), ref)


@pytest.mark.parametrize("name", FORMAT_CASES)
@pytest.mark.parametrize("nthreads", [1, 0])
def test_weight_formats(name, nthreads):
    d = np.load(os.path.join(HERE, "nkbg_formats.npz"))
    path = os.path.join(HERE, f"nkbg_{name}.nkbg")
    want = {"none": 0, "unsigned": 1, "signed": 2, "double": 3, "float": 4}[name.split("_")[0]]
    assert (features(path) & 0xE) >> 1 == want
    ref = {k: d[f"{name}_{k}"] for k in FIELDS}
    compare(graphio.read_nkbg(path, nthreads), ref)


def test_reader_api_and_graph():
    path = os.path.join(HERE, "wikivote_directed.nkbg")
    g = graphio.readGraph(path, graphio.Format.NetworkitBinary)
    d = np.load(os.path.join(HERE, "wikivote_directed.npz"))
    assert g.isDirected() and not g.isWeighted()
    assert g.upperNodeIdBound() == d["nkbg_exists"].shape[0]
    assert g.numberOfEdges() == d["nkbg_in_col"].shape[0]
    g2 = graphio.NetworkitBinaryReader().read(path)
    assert g2.numberOfNodes() == g.numberOfNodes()


def test_deleted_flags(tmp_path):
    """A cleared flag byte deletes the node (NetworkitBinaryReader.cpp:72-80);
    nothing else of the decoded graph changes. Only isolated ids are cleared."""
    src = os.path.join(HERE, "nkbg_none_dir.nkbg")
    data = bytearray(open(src, "rb").read())
    base = graphio.read_nkbg(src)
    iso = np.flatnonzero((np.diff(base.in_ptr) == 0) & (base.outdeg == 0))[:5]
    assert iso.size == 5
    off = struct.unpack("<Q", bytes(data[40:48]))[0]
    for v in iso:
        data[off + int(v)] = 0
    p = tmp_path / "deleted.nkbg"
    p.write_bytes(bytes(data))
    g = graphio.read_nkbg(str(p))
    assert g.n == base.z - 5
    np.testing.assert_array_equal(np.flatnonzero(g.exists == 0), iso)
    np.testing.assert_array_equal(g.in_ptr, base.in_ptr)
    np.testing.assert_array_equal(g.in_col, base.in_col)


def test_errors(tmp_path):
    with pytest.raises(IOError, match="is not a file"):
        graphio.readGraph(str(tmp_path / "missing.nkbg"), graphio.Format.NetworkitBinary)
    bad = tmp_path / "bad.nkbg"
    bad.write_bytes(b"nkbg001" + b"\0" * 100)
    with pytest.raises(RuntimeError, match="magic"):
        graphio.read_nkbg(str(bad))
    with pytest.raises(IOError, match="not a valid"):
        graphio.readGraph(str(bad), graphio.Format.NetworkitBinary)
    # truncated list data
    data = open(os.path.join(HERE, "nkbg_signed_undir.nkbg"), "rb").read()
    cut = tmp_path / "cut.nkbg"
    cut.write_bytes(data[: len(data) // 2])
    with pytest.raises(RuntimeError):
        graphio.read_nkbg(str(cut))
    # a neighbour id past the node count
    d2 = bytearray(open(os.path.join(HERE, "nkbg_none_dir.nkbg"), "rb").read())
    struct.pack_into("<Q", d2, 24, 3)  # claim 3 nodes
    struct.pack_into("<Q", d2, 32, 1)  # in one chunk
    p2 = tmp_path / "ids.nkbg"
    p2.write_bytes(bytes(d2))
    with pytest.raises(RuntimeError):
        graphio.read_nkbg(str(p2))


@pytest.mark.gpu
@pytest.mark.parametrize("name", GRAPH_CASES + ["nkbg_none_undir", "nkbg_none_dir"])
def test_pagerank_on_decoded_graph(oracle_mod, name):
    """File -> host decode -> device graph -> PageRank, against the oracle on
    the decoded in-CSR: FP64 L1 <= 1e-10, iterations within 1. (The weight
    encoding files hold zero and 2^60 weights, made for the decoder, on which
    PageRank need not converge.)"""
    from networkit_b200 import _capi

    csr = graphio.read_nkbg(os.path.join(HERE, f"{name}.nkbg"))
    dg = _capi.DeviceGraph(csr)
    for norm in (0, 1):
        p = dg.params(0.85, 1e-10, norm, False, False, _capi.NKG_PREC_FP64, 10000)
        s, it, _, _ = dg.run(p)
        o = oracle_mod.pagerank(csr, tol=1e-10, norm=norm, max_iterations=10000)
        assert float(np.abs(s - o.scores).sum()) <= 1e-10
        assert abs(int(it) - o.iterations) <= 1


def test_reader_library_exports_header_symbols():
    """libnkgen.so exports every entry point include/nkgio.h declares."""
    import ctypes
    import re

    from networkit_b200 import build

    src = open(os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "nkgio.h")).read()
    syms = sorted(set(re.findall(r"NKGEN_API\s+[\w\s\*]+?\b(nkgen_\w+)\s*\(", src)))
    assert len(syms) == 4, syms
    build.build_gen()
    lib = ctypes.CDLL(build.GEN_LIB)
    for s in syms:
        assert hasattr(lib, s), s


@pytest.mark.parametrize("name", GRAPH_CASES)
def test_writer_bytes_match_reference_writer(tmp_path, name):
    """The writer, given a reference test graph's storage-order adjacency,
    produces the very bytes the reference's NetworkitBinaryWriter wrote
    (4 chunks, weight format auto-detected)."""
    d = np.load(os.path.join(HERE, f"{name}.npz"))
    directed = bool(d["directed"])
    w_out = d["out_w"] if bool(d["weighted"]) else None
    w_in = d["in_w"] if bool(d["weighted"]) else None
    out = tmp_path / "w.nkbg"
    if directed:
        graphio.write_nkbg(str(out), int(d["z"]), d["out_ptr"], d["out_col"], w_out,
                           d["in_ptr"], d["in_col"], w_in, directed=True, chunks=4)
    else:
        graphio.write_nkbg(str(out), int(d["z"]), d["out_ptr"], d["out_col"], w_out,
                           directed=False, chunks=4)
    assert out.read_bytes() == open(os.path.join(HERE, f"{name}.nkbg"), "rb").read()


@pytest.mark.parametrize("name,chunks", [("unsigned_dir", 5), ("float_dir", 2), ("none_dir", 1)])
def test_writer_round_trip_formats(tmp_path, name, chunks):
    """Directed files of every weight encoding: decode, encode again with the
    same chunks and encoding -> the same bytes."""
    src = os.path.join(HERE, f"nkbg_{name}.nkbg")
    fmt = (features(src) & 0xE) >> 1
    g = graphio.read_nkbg(src)  # in-lists = the file's transpose lists
    data = open(src, "rb").read()
    optr, ocol, ow = _file_out_lists(data)  # the file's adjacency lists, in order
    out = tmp_path / "w.nkbg"
    graphio.write_nkbg(str(out), g.z, optr, ocol, ow, g.in_ptr, g.in_col, g.in_w,
                       directed=True, chunks=chunks, weights=fmt)
    assert out.read_bytes() == data


def _file_out_lists(data):
    """(ptr, col, w) of a directed file's adjacency lists in file order, via
    the reader on a copy whose adjacency and transpose sections are swapped
    (its in-rows are then the file's out-lists)."""
    import tempfile

    b = bytearray(data)
    adj_off, tr_off, w_off, wt_off = struct.unpack("<4Q", bytes(b[48:80]))
    struct.pack_into("<4Q", b, 48, tr_off, adj_off, wt_off, w_off)
    with tempfile.NamedTemporaryFile(suffix=".nkbg", delete=False) as f:
        f.write(bytes(b))
        path = f.name
    try:
        g = graphio.read_nkbg(path)
    finally:
        os.unlink(path)
    return g.in_ptr, g.in_col, g.in_w


def test_writer_graph_api_and_errors(tmp_path):
    from networkit_b200.graph import Graph

    g = Graph(5, weighted=True, directed=True)
    for u, v, w in [(0, 1, 2.0), (1, 2, 3.5), (2, 0, 1.0), (4, 4, 7.0), (0, 3, 1.0)]:
        g.addEdge(u, v, w)
    p = tmp_path / "g.nkbg"
    graphio.NetworkitBinaryWriter(chunks=3).write(g, str(p))
    assert (features(str(p)) & 0xE) >> 1 == 4  # all weights are floats
    back = graphio.read_nkbg(str(p))
    ref = g.inCSR()
    np.testing.assert_array_equal(back.in_ptr, ref.in_ptr)
    np.testing.assert_array_equal(back.in_col, ref.in_col)
    np.testing.assert_array_equal(back.in_w, ref.in_w)
    np.testing.assert_array_equal(back.wdeg, ref.wdeg)
    h = Graph(3)
    h.removeNode(2)
    with pytest.raises(RuntimeError, match="existing nodes"):
        graphio.NetworkitBinaryWriter().write(h, str(p))
    with pytest.raises(RuntimeError, match="weights"):
        graphio.write_nkbg(str(p), 2, [0, 1, 1], [1], weights=9)
