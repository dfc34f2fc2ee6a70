"""NetworkitBinaryGraph decoded on the device (nkg_nkbg_decode,
nkg_graph_create_from_nkbg) against the host decoder, which is checked bit
for bit against the reference's NetworkitBinaryReader in test_graphio.py
(NetworkitBinaryReader.cpp:19-235).

Bar: bit-exact in-CSR, weights, weighted degrees, degrees, node flags and
graph kind, for every weight encoding, chunk count and direction; a graph
built from the file on the device runs PageRank bit for bit like one built
from the host-decoded arrays; malformed files are refused, not read past
their end."""
import glob
import os
import struct

import numpy as np
import pytest

from networkit_b200 import _capi, generators, graphio

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(glob.glob(os.path.join(HERE, "*.nkbg")))


def same(a, b):
    np.testing.assert_array_equal(a.in_ptr, b.in_ptr)
    np.testing.assert_array_equal(a.in_col, b.in_col)
    assert (a.in_w is None) == (b.in_w is None)
    if a.in_w is not None:
        np.testing.assert_array_equal(a.in_w.view(np.uint64), b.in_w.view(np.uint64))
    np.testing.assert_array_equal(np.asarray(a.wdeg).view(np.uint64),
                                  np.asarray(b.wdeg).view(np.uint64))
    np.testing.assert_array_equal(a.outdeg, b.outdeg)
    ea = np.ones(a.z, np.uint8) if a.exists is None else a.exists
    eb = np.ones(b.z, np.uint8) if b.exists is None else b.exists
    np.testing.assert_array_equal(ea, eb)
    assert a.directed == b.directed and a.z == b.z and a.n == b.n


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(p)[:-5] for p in FILES])
def test_device_decode_equals_host_decode(path):
    data = open(path, "rb").read()
    dev, ms = graphio.decode_nkbg_device(data)
    same(dev, graphio.read_nkbg(path))
    assert ms > 0


def _write(tmp_path, csr, chunks, weights=None, name="g"):
    out_ptr, out_col, order = csr.out_csr()
    out_w = None if weights is None else weights[order]
    p = str(tmp_path / f"{name}.nkbg")
    graphio.write_nkbg(p, csr.z, out_ptr, out_col, out_w, csr.in_ptr, csr.in_col, weights,
                       directed=True, chunks=chunks)
    return p


@pytest.mark.parametrize("chunks", [1, 7, 64])
@pytest.mark.parametrize("wkind", ["none", "double", "varint", "zigzag", "float"])
def test_generated_files(tmp_path, chunks, wkind):
    csr = generators.rmat_directed(14, 16, seed=11)
    rng = np.random.default_rng(chunks)
    w = {"none": None,
         "double": rng.uniform(0.1, 1.0, csr.arcs),
         "varint": rng.integers(1, 5000, csr.arcs).astype(np.float64),
         "zigzag": rng.integers(-300, 300, csr.arcs).astype(np.float64),
         "float": rng.uniform(0.1, 1.0, csr.arcs).astype(np.float32).astype(np.float64)}[wkind]
    p = _write(tmp_path, csr, chunks, w)
    dev, _ = graphio.decode_nkbg_device(open(p, "rb").read())
    same(dev, graphio.read_nkbg(p))


def test_undirected_graph_with_self_loops(tmp_path):
    g = graphio.read_nkbg(os.path.join(HERE, "looptest1.nkbg"))
    assert not g.directed
    for f in ("looptest1", "looptest2", "nkbg_signed_undir", "nkbg_double_undir"):
        p = os.path.join(HERE, f + ".nkbg")
        dev, _ = graphio.decode_nkbg_device(open(p, "rb").read())
        same(dev, graphio.read_nkbg(p))


# The format fixtures carry negative and zero weights (some weighted degrees
# are <= 0), on which PageRank does not converge, in the reference as here:
# the comparisons run a fixed number of sweeps.
SWEEPS = 40


@pytest.mark.parametrize("name", ["wikivote_directed", "nkbg_double_undir", "nkbg_float_dir"])
def test_graph_from_file_runs_like_host_decoded_graph(name):
    path = os.path.join(HERE, name + ".nkbg")
    host = graphio.read_nkbg(path)
    a = _capi.DeviceGraph(host)
    b = _capi.DeviceGraph.from_nkbg(open(path, "rb").read())
    assert b.info() == {**a.info(), "ms_create": b.info()["ms_create"]}
    p = a.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, SWEEPS)
    sa, ia, _, _ = a.run(p)
    sb, ib, _, _ = b.run(p)
    assert ia == ib
    np.testing.assert_array_equal(sa.view(np.uint64), sb.view(np.uint64))


def test_graph_from_file_in_device_memory():
    import torch

    path = os.path.join(HERE, "nkbg_unsigned_dir.nkbg")
    data = np.frombuffer(open(path, "rb").read(), np.uint8)
    d = torch.from_numpy(data.copy()).cuda()
    torch.cuda.synchronize()
    g = _capi.DeviceGraph.from_nkbg(d.data_ptr(), on_device=True, size=data.shape[0])
    h = _capi.DeviceGraph(graphio.read_nkbg(path))
    p = g.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, SWEEPS)
    np.testing.assert_array_equal(g.run(p)[0], h.run(p)[0])


def test_generated_weighted_file_converges_like_host_decoded_graph(tmp_path):
    csr = generators.rmat_directed(14, 16, seed=11)
    w = np.random.default_rng(3).uniform(0.1, 1.0, csr.arcs)
    p = _write(tmp_path, csr, 9, w)
    a = _capi.DeviceGraph(graphio.read_nkbg(p))
    b = _capi.DeviceGraph.from_nkbg(open(p, "rb").read())
    prm = a.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, 1000)
    sa, ia, _, _ = a.run(prm)
    sb, ib, _, _ = b.run(prm)
    assert ia == ib < 1000
    np.testing.assert_array_equal(sa.view(np.uint64), sb.view(np.uint64))


def test_malformed_files_are_refused(tmp_path):
    good = open(os.path.join(HERE, "nkbg_signed_undir.nkbg"), "rb").read()
    with pytest.raises(_capi.NkgError, match="magic"):
        graphio.decode_nkbg_device(b"nkbg001" + b"\0" * 100)
    with pytest.raises(_capi.NkgError):
        graphio.decode_nkbg_device(good[: len(good) // 2])   # truncated
    with pytest.raises(_capi.NkgError):
        graphio.decode_nkbg_device(good[:60])                # shorter than the header
    d2 = bytearray(open(os.path.join(HERE, "nkbg_none_dir.nkbg"), "rb").read())
    struct.pack_into("<Q", d2, 24, 3)   # claim 3 nodes
    struct.pack_into("<Q", d2, 32, 1)   # in one chunk
    with pytest.raises(_capi.NkgError):
        graphio.decode_nkbg_device(bytes(d2))
    # The next, valid file decodes normally.
    dev, _ = graphio.decode_nkbg_device(good)
    same(dev, graphio.read_nkbg(os.path.join(HERE, "nkbg_signed_undir.nkbg")))


@pytest.mark.parametrize("staging", [0, 4096, 4096 * 3 + 16, 100_000])
@pytest.mark.parametrize("name", ["wikivote_directed", "nkbg_double_undir", "nkbg_none_undir"])
def test_graph_from_file_path_equals_graph_from_bytes(name, staging):
    """nkg_graph_create_from_nkbg_file: reader threads, pieces of `staging`
    bytes (odd sizes: pieces that split varints and chunks), then the same
    decode: the same graph, the same PageRank bit for bit."""
    path = os.path.join(HERE, name + ".nkbg")
    a = _capi.DeviceGraph.from_nkbg(open(path, "rb").read())
    b = _capi.DeviceGraph.from_nkbg_file(path, staging_bytes=staging)
    assert b.info() == {**a.info(), "ms_create": b.info()["ms_create"]}
    assert b.s_load > 0 and b.ms_decode > 0
    p = a.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, SWEEPS)
    sa, ia, _, _ = a.run(p)
    sb, ib, _, _ = b.run(p)
    assert ia == ib
    np.testing.assert_array_equal(sa.view(np.uint64), sb.view(np.uint64))


def test_generated_file_path_many_pieces(tmp_path):
    csr = generators.rmat_directed(15, 16, seed=5)
    p = _write(tmp_path, csr, 13)
    a = _capi.DeviceGraph(graphio.read_nkbg(p))
    b = _capi.DeviceGraph.from_nkbg_file(p, staging_bytes=65536 + 8)  # dozens of pieces
    prm = a.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, SWEEPS)
    sa, ia, _, _ = a.run(prm)
    sb, ib, _, _ = b.run(prm)
    assert ia == ib
    np.testing.assert_array_equal(sa.view(np.uint64), sb.view(np.uint64))


def test_file_path_errors(tmp_path):
    with pytest.raises(_capi.NkgError, match="cannot open"):
        _capi.DeviceGraph.from_nkbg_file(str(tmp_path / "missing.nkbg"))
    with pytest.raises(_capi.NkgError, match="regular file"):
        _capi.DeviceGraph.from_nkbg_file(str(tmp_path))
    short = tmp_path / "short.nkbg"
    short.write_bytes(b"nkbg002" + b"\0" * 20)
    with pytest.raises(_capi.NkgError, match="NetworkitBinaryGraph"):
        _capi.DeviceGraph.from_nkbg_file(str(short))
    bad = tmp_path / "bad.nkbg"
    good = open(os.path.join(HERE, "nkbg_signed_undir.nkbg"), "rb").read()
    bad.write_bytes(good[: len(good) // 2])
    with pytest.raises(_capi.NkgError):
        _capi.DeviceGraph.from_nkbg_file(str(bad), staging_bytes=4096)
