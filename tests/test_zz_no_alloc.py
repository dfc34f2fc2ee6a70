"""The allocation-free entry point, nkg_pagerank_csr_noalloc.

It serves callers that cannot allocate device memory when they call in (a
framework whose caching allocator owns the device memory, a fixed memory
budget, a latency-critical loop where cudaMalloc/cudaFree would synchronise
the device): they hand in the graph and the output buffer in device memory
and the library works in a fixed 12.1 MB scratch array of its own.

This file is collected last so that a run stopping at the first failure has
already run every other test. Each check calls the new entry point twice in a
row through the C ABI (the scratch keeps the previous call's contents, so the
second call proves that it is reset) and compares it with the regular entry
point, nkg_pagerank_run, and with the oracle, within the FP64 parity
tolerance of the other tests. Malformed input (offsets that are not a CSR,
column ids >= n) must be refused before any sweep reads the graph: the test
arrays are allocated at the sizes the call is told, so the check itself
reads nothing out of bounds.
"""
import ctypes as C

import numpy as np
import pytest

from networkit_b200 import _capi, generators

pytestmark = pytest.mark.gpu

L1_FP64 = 1e-10


def _call(z, arcs, in_ptr, in_col, params):
    """One call on device copies of the given arrays (sized as given);
    returns (return code, scores, iterations)."""
    import torch

    dev = torch.device("cuda", 0)
    ptr = torch.from_numpy(np.ascontiguousarray(in_ptr, np.uint64).view(np.int64)).to(dev)
    col = torch.from_numpy(np.ascontiguousarray(in_col, np.uint32).view(np.int32)).to(dev)
    out = torch.empty(z, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    it = C.c_uint64(0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = _capi.lib().nkg_pagerank_csr_noalloc(
        z, arcs, C.c_void_p(ptr.data_ptr()), C.c_void_p(col.data_ptr() if arcs else None),
        C.byref(params), C.c_void_p(out.data_ptr()), C.byref(it), C.c_void_p(stream))
    return rc, out.cpu().numpy(), int(it.value)


def _noalloc(csr, params):
    rc, scores, it = _call(csr.z, csr.arcs, csr.in_ptr, csr.in_col, params)
    _capi.check(rc)
    return scores, it


@pytest.mark.parametrize("case", ["er", "rmat", "rmat_l2_normalized", "er_distribute"])
def test_noalloc_matches_regular_entry_point_twice(case):
    if case.startswith("er"):
        csr = generators.erdos_renyi(100000, 10 / 99999, seed=42)
    else:
        csr = generators.rmat_directed(15, 16, seed=7)
    norm = 1 if "l2" in case or case.startswith("er") else 0
    normalized = "normalized" in case
    distribute = "distribute" in case
    tol = 1e-8 if norm == 1 else 1e-10
    dg = _capi.DeviceGraph(csr)
    p = dg.params(0.85, tol, norm, normalized, distribute, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
    ref, it_ref, _, _ = dg.run(p)
    first, it1 = _noalloc(csr, p)
    second, it2 = _noalloc(csr, p)
    scale = 1.0 if not normalized else float(np.abs(ref).sum())
    for got, it in ((first, it1), (second, it2)):
        assert np.abs(got - ref).sum() <= L1_FP64 * scale
        assert abs(it - it_ref) <= 1
    np.testing.assert_array_equal(first, second)
    # The same bar against the oracle (the CPU restatement of PageRank.cpp).
    import oracle

    o = oracle.pagerank(csr, tol=tol, norm=norm, normalized=normalized,
                        distribute_sinks=distribute)
    assert np.abs(first - o.scores).sum() <= L1_FP64 * scale
    assert abs(it1 - o.iterations) <= 1


def test_noalloc_at_its_largest_graph():
    """n = 524,288, the most the fixed scratch holds (its layout is tightest
    there): two calls equal the regular entry point."""
    csr = generators.rmat_directed(19, 8, seed=3)
    assert csr.z == 524288
    dg = _capi.DeviceGraph(csr)
    p = dg.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
    ref, it_ref, _, _ = dg.run(p)
    for _ in range(2):
        got, it = _noalloc(csr, p)
        assert np.abs(got - ref).sum() <= L1_FP64
        assert abs(it - it_ref) <= 1


def _small():
    # 6 nodes, 8 arcs, rows of 0..3 arcs (node 5 has none).
    ptr = np.array([0, 2, 3, 6, 7, 8, 8], np.uint64)
    col = np.array([1, 2, 0, 0, 1, 4, 2, 3], np.uint32)
    return ptr, col


def _noalloc_small(p):
    ptr, col = _small()
    rc, scores, it = _call(6, 8, ptr, col, p)
    _capi.check(rc)
    return scores, it


@pytest.mark.parametrize("defect", ["first_offset", "decreasing", "last_beyond_arcs",
                                    "last_short_of_arcs"])
def test_noalloc_rejects_offsets_that_are_not_a_csr(defect):
    ptr, col = _small()
    ptr = ptr.copy()
    if defect == "first_offset":
        ptr[0] = 1
    elif defect == "decreasing":
        ptr[3] = 2
    elif defect == "last_beyond_arcs":
        ptr[6] = 9
    else:
        ptr[6] = 7
    p = _capi.PRParams(0.85, 1e-10, 0, 0, 0, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
    rc, _, _ = _call(6, 8, ptr, col, p)
    assert rc == _capi.NKG_ERR_INVALID_ARG
    assert "offset" in _capi.lib().nkg_last_error().decode()
    # The scratch is fine for the next, valid call.
    good, _ = _noalloc_small(p)
    import oracle
    from networkit_b200.graph import InCSR

    ptr0, col0 = _small()
    deg = np.bincount(col0, minlength=6)
    csr = InCSR(6, 6, ptr0, col0, None, deg.astype(np.float64), deg.astype(np.uint32), None, True)
    assert np.abs(good - oracle.pagerank(csr, tol=1e-10, norm=0).scores).sum() <= L1_FP64


def test_noalloc_rejects_column_ids_beyond_n():
    ptr, col = _small()
    col = col.copy()
    col[5] = 6
    p = _capi.PRParams(0.85, 1e-10, 0, 0, 0, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
    rc, _, _ = _call(6, 8, ptr, col, p)
    assert rc == _capi.NKG_ERR_INVALID_ARG
    assert ">= n" in _capi.lib().nkg_last_error().decode()


def test_noalloc_rejects_graphs_beyond_its_scratch():
    p = _capi.PRParams(0.85, 1e-8, 1, 0, 0, _capi.NKG_PREC_FP64, 100)
    rc = _capi.lib().nkg_pagerank_csr_noalloc(524289, 0, C.c_void_p(8), None, C.byref(p),
                                             C.c_void_p(8), None, None)
    assert rc == _capi.NKG_ERR_INVALID_ARG
    assert "524288" in _capi.lib().nkg_last_error().decode()
