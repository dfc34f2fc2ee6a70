"""The row-partitioned PageRank (nkg_part_* through networkit_b200.distributed)
on one GPU: one process holding 1, 2 or 5 slices, swept one after another and
exchanged by copies, so the partitioned kernels and the collective logic run
without a second GPU. Bar: the oracle's parity bar (L1 <= 1e-10, iterations
within 1), and the single-GPU library path to rounding of the reductions."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden
from networkit_b200 import _capi, distributed, generators

pytestmark = pytest.mark.gpu

L1_FP64 = 1e-10


@pytest.fixture(scope="module")
def graphs():
    wiki, _ = load_golden("wikivote_directed")
    und, _ = load_golden("wikivote_undirected")
    return {
        "wikivote_directed": wiki,
        "wikivote_undirected": und,
        "rmat16": generators.rmat_directed(16, 16, seed=5),
        "rmat14_weighted": generators.with_uniform_weights(
            generators.rmat_directed(14, 16, seed=9), seed=4),
        "er": generators.erdos_renyi(20000, 10 / 19999, seed=42),
    }


CASES = [
    ("wikivote_directed", dict(norm=0, tol=1e-10)),
    ("wikivote_undirected", dict(norm=1, tol=1e-8, normalized=True)),
    ("rmat16", dict(norm=0, tol=1e-10)),
    ("rmat14_weighted", dict(norm=1, tol=1e-9)),
    ("er", dict(norm=1, tol=1e-8, distribute_sinks=True)),
    ("rmat16", dict(norm=0, tol=1e-10, distribute_sinks=True, normalized=True)),
]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("parts", [1, 2, 5])
def test_row_partition_on_one_gpu(graphs, oracle_mod, case, parts):
    name, kw = CASES[case]
    csr = graphs[name]
    s, it, mx, st = distributed.pagerank_row_partitioned(csr, parts_per_rank=parts, **kw)
    assert st["parts"] == parts and sum(st["slice_rows"]) == csr.z
    o = oracle_mod.pagerank(csr, **kw)
    scale = 1.0 if not kw.get("normalized") else float(np.abs(o.scores).sum())
    assert np.abs(s - o.scores).sum() <= L1_FP64 * scale, name
    assert abs(it - o.iterations) <= 1
    assert abs(mx - o.maximum) <= 1e-12 * max(1.0, abs(o.maximum))
    # The single-GPU library path: the same per-row arithmetic.
    dg = _capi.DeviceGraph(csr)
    p = dg.params(0.85, kw["tol"], kw["norm"], kw.get("normalized", False),
                  kw.get("distribute_sinks", False), _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
    s1, it1, _, _ = dg.run(p)
    if it1 == it:
        assert np.abs(s - s1).sum() <= 1e-13 * scale


def test_row_partition_reuse_timing_and_trace(graphs, oracle_mod):
    csr = graphs["rmat16"]
    pr = distributed.RowPartitionedPageRank(csr, parts_per_rank=3)
    try:
        s, it, _, st = pr.run(norm=0, tol=1e-10, timing=True)
        s2, it2, _, _ = pr.run(norm=0, tol=1e-10)
    finally:
        pr.close()
    np.testing.assert_array_equal(s, s2)
    assert it == it2
    assert st["ms_sweeps"] > 0 and st["ms_exchange"] >= 0
    o = oracle_mod.pagerank(csr, norm=0, tol=1e-10)
    k = min(len(st["residual_trace"]), o.trace.shape[0])
    np.testing.assert_allclose(st["residual_trace"][:k], o.trace[:k], rtol=1e-9, atol=1e-13)


def test_part_api_checks_its_input():
    L = _capi.lib()
    h = C.c_void_p()
    ptr = np.array([0, 2, 3], np.uint64)
    col = np.array([0, 9, 1], np.uint32)  # 9 is outside a shared iterate of 4 entries
    deg = np.array([1, 1], np.uint32)
    rc = L.nkg_part_create(C.byref(h), 4, 0, 2, 3, _capi.ptr(ptr, _capi._u64p),
                           _capi.ptr(col, _capi._u32p), None, _capi.ptr(deg, _capi._u32p), None, -1)
    assert rc == _capi.NKG_ERR_INVALID_ARG
    assert "outside the shared iterate" in L.nkg_last_error().decode()
    bad = np.array([0, 3, 2], np.uint64)
    rc = L.nkg_part_create(C.byref(h), 4, 0, 2, 3, _capi.ptr(bad, _capi._u64p),
                           _capi.ptr(np.array([0, 1, 1], np.uint32), _capi._u32p), None,
                           _capi.ptr(deg, _capi._u32p), None, -1)
    assert rc == _capi.NKG_ERR_INVALID_ARG
