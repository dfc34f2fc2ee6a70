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
point, nkg_pagerank_run, within the FP64 parity tolerance of the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from networkit_b200 import _capi, generators

pytestmark = pytest.mark.gpu

L1_FP64 = 1e-10


def _noalloc(csr, params):
    import torch

    dev = torch.device("cuda", 0)
    ptr = torch.from_numpy(np.ascontiguousarray(csr.in_ptr, np.uint64).view(np.int64)).to(dev)
    col = torch.from_numpy(np.ascontiguousarray(csr.in_col, np.uint32).view(np.int32)).to(dev)
    out = torch.empty(csr.z, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    it = C.c_uint64(0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    _capi.check(_capi.lib().nkg_pagerank_csr_noalloc(
        csr.z, csr.arcs, C.c_void_p(ptr.data_ptr()), C.c_void_p(col.data_ptr()),
        C.byref(params), C.c_void_p(out.data_ptr()), C.byref(it), C.c_void_p(stream)))
    return out.cpu().numpy(), int(it.value)


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


def test_noalloc_rejects_graphs_beyond_its_scratch():
    p = _capi.PRParams(0.85, 1e-8, 1, 0, 0, _capi.NKG_PREC_FP64, 100)
    rc = _capi.lib().nkg_pagerank_csr_noalloc(524289, 0, C.c_void_p(8), None, C.byref(p),
                                             C.c_void_p(8), None, None)
    assert rc == _capi.NKG_ERR_INVALID_ARG
    assert "524288" in _capi.lib().nkg_last_error().decode()
