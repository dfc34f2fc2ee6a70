"""GPU ingest (nkg_graph_create_from_edges): the graph built on the device
from an edge list in insertion order equals the one built from the host
in-CSR of the same edges (graph.in_csr_from_edges, which follows
Graph::addEdge, Graph.cpp:549-596): same shape, and bit-identical PageRank
scores and iteration counts, since the arc order and the weighted degrees
(summed in edge order) are the same."""
import numpy as np
import pytest

from networkit_b200 import _capi
from networkit_b200.graph import in_csr_from_edges

pytestmark = pytest.mark.gpu


def random_edges(z, m, seed, loops=True, dups=True):
    """Skewed endpoints (uneven rows, some split into chunks) below z - 1000,
    so the top 1000 ids are untouched."""
    rng = np.random.default_rng(seed)
    src = ((z - 1000) * rng.random(m) ** 3).astype(np.uint32)
    dst = ((z - 1000) * rng.random(m) ** 2).astype(np.uint32)
    if not loops:
        keep = src != dst
        src, dst = src[keep], dst[keep]
    if dups:
        src = np.concatenate([src, src[:50]])
        dst = np.concatenate([dst, dst[:50]])
    return src, dst


@pytest.mark.parametrize("directed", [True, False])
@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("deleted", [False, True])
def test_from_edges_equals_host_csr(directed, weighted, deleted):
    z, m = 20000, 300000
    src, dst = random_edges(z, m, seed=3)
    w = np.random.default_rng(4).random(src.shape[0]) + 0.1 if weighted else None
    exists = None
    if deleted:
        # delete ids that no edge touches
        touched = np.zeros(z, bool)
        touched[src] = True
        touched[dst] = True
        exists = touched.astype(np.uint8)
        assert exists.sum() < z
    csr = in_csr_from_edges(z, src, dst, w, directed=directed, exists=exists)
    a = _capi.DeviceGraph(csr)
    b = _capi.DeviceGraph.from_edges(z, src, dst, w, directed=directed, exists=exists)
    ia, ib = a.info(), b.info()
    for k in ("z", "n", "arcs", "sinks", "slots", "split_rows", "weighted"):
        assert ia[k] == ib[k], k
    for prec in (_capi.NKG_PREC_FP64, _capi.NKG_PREC_FP32):
        p = a.params(0.85, 1e-10 if prec == 0 else 1e-6, 0, False, True, prec, 1000)
        sa, ita, _, _ = a.run(p)
        sb, itb, _, _ = b.run(p)
        np.testing.assert_array_equal(sa, sb)
        assert ita == itb


def test_from_device_edges_and_errors():
    import torch

    z, m = 5000, 60000
    src, dst = random_edges(z, m, seed=9, loops=False, dups=False)
    csr = in_csr_from_edges(z, src, dst, directed=True)
    a = _capi.DeviceGraph(csr)
    ds = torch.from_numpy(src.view(np.int32)).cuda()
    dd = torch.from_numpy(dst.view(np.int32)).cuda()
    torch.cuda.synchronize()
    b = _capi.DeviceGraph.from_device_edges(z, src.shape[0], ds.data_ptr(), dd.data_ptr(),
                                            directed=True)
    p = a.params(0.85, 1e-10, 0, False, False, 0, 1000)
    np.testing.assert_array_equal(a.run(p)[0], b.run(p)[0])
    bad = dst.copy()
    bad[7] = z
    with pytest.raises(_capi.NkgError, match=">= z"):
        _capi.DeviceGraph.from_edges(z, src, bad, directed=True)
    ex = np.ones(z, np.uint8)
    ex[int(src[0])] = 0
    with pytest.raises(_capi.NkgError, match="non-existent"):
        _capi.DeviceGraph.from_edges(z, src, dst, directed=True, exists=ex)
    empty = _capi.DeviceGraph.from_edges(10, [], [], directed=False)
    s, it, _, _ = empty.run(p)
    np.testing.assert_allclose(s, np.full(10, 0.1))
