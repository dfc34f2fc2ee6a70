"""Run control and layout options of the PageRank path, through the C ABI.

* The shared-memory tier of the sweep (nkg_graph_options.hot_tier_kb): every
  row sum is the same with or without it, so scores agree bit for bit at the
  same iteration count (without distributeSinks, whose sink mass is summed
  over the sweep's CTAs), and both meet the oracle's parity bar.
* The residual trace of nkg_stats: the stopping-test residual of every sweep,
  against the oracle's trace of the same run (PageRank.cpp:41-51).
* Cancellation (nkg_cancel, the SIGINT check of PageRank.cpp:55): from another
  thread during a run, before a run starts, and by SIGINT through
  nkg_sigint_cancels (Aux::SignalHandler, SignalHandling.cpp:29-66). The
  handle runs normally afterwards.
"""
import os
import signal
import threading
import time

import numpy as np
import pytest

from conftest import load_golden
from networkit_b200 import Graph, _capi, centrality, generators

pytestmark = pytest.mark.gpu

L1_FP64 = 1e-10


def _graphs():
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


@pytest.fixture(scope="module")
def graphs():
    return _graphs()


@pytest.mark.parametrize("name", ["wikivote_directed", "wikivote_undirected", "rmat16",
                                  "rmat14_weighted", "er"])
@pytest.mark.parametrize("kb", [1, 8, 96, 224])
@pytest.mark.parametrize("distribute", [False, True])
def test_hot_tier_fp64_same_rows_and_oracle_parity(graphs, oracle_mod, name, kb, distribute):
    csr = graphs[name]
    p = _capi.DeviceGraph.params(0.85, 1e-10, 0, False, distribute, _capi.NKG_PREC_FP64,
                                 _capi.UINT64_MAX)
    off = _capi.DeviceGraph(csr, hot_tier_kb=0)
    s0, it0, _, _ = off.run(p)
    on = _capi.DeviceGraph(csr, hot_tier_kb=kb)
    s1, it1, _, _ = on.run(p)
    if it0 == it1 and not distribute:
        np.testing.assert_array_equal(s0.view(np.uint64), s1.view(np.uint64))
    elif it0 == it1:
        # The sink mass is summed over the sweep's CTAs, whose number differs
        # with the tier: the sink term can differ in its last bits.
        assert np.abs(s0 - s1).sum() <= 1e-14
    o = oracle_mod.pagerank(csr, tol=1e-10, norm=0, distribute_sinks=distribute)
    assert np.abs(s1 - o.scores).sum() <= L1_FP64
    assert abs(it1 - o.iterations) <= 1


@pytest.mark.parametrize("prec", [_capi.NKG_PREC_FP32, _capi.NKG_PREC_FP32_REFINE])
def test_hot_tier_other_precisions(graphs, oracle_mod, prec):
    csr = graphs["rmat16"]
    p = _capi.DeviceGraph.params(0.85, 1e-10 if prec == _capi.NKG_PREC_FP32_REFINE else 1e-7, 0,
                                 False, False, prec, 500)
    s0, it0, _, _ = _capi.DeviceGraph(csr, hot_tier_kb=0).run(p)
    s1, it1, _, _ = _capi.DeviceGraph(csr, hot_tier_kb=224).run(p)
    if it0 == it1:
        np.testing.assert_array_equal(s0.view(np.uint64), s1.view(np.uint64))
    o = oracle_mod.pagerank(csr, tol=1e-12, norm=0)
    bar = 1e-9 if prec == _capi.NKG_PREC_FP32_REFINE else 1e-5
    assert np.abs(s1 - o.scores).sum() <= bar


def test_hot_tier_option_is_checked(graphs):
    with pytest.raises(_capi.NkgError, match="hot_tier_kb"):
        _capi.DeviceGraph(graphs["wikivote_directed"], hot_tier_kb=225)


@pytest.mark.parametrize("norm", [0, 1])
@pytest.mark.parametrize("prec", [_capi.NKG_PREC_FP64, _capi.NKG_PREC_FP32_REFINE])
def test_residual_trace_matches_oracle(oracle_mod, norm, prec):
    csr, _ = load_golden("wikivote_directed")
    dg = _capi.DeviceGraph(csr)
    tol = 1e-10 if norm == 0 else 1e-9
    p = dg.params(0.85, tol, norm, False, False, prec, _capi.UINT64_MAX)
    _, it, _, st = dg.run(p, trace=4096)
    tr = st["residual_trace"]
    assert st["trace_length"] == (it if prec == _capi.NKG_PREC_FP64 else st["fp64_sweeps"])
    assert tr.shape[0] == st["trace_length"]
    assert tr[-1] <= tol and (tr.shape[0] == 1 or tr[-2] > tol)
    if prec == _capi.NKG_PREC_FP64:
        o = oracle_mod.pagerank(csr, tol=tol, norm=norm)
        k = min(tr.shape[0], o.trace.shape[0])
        # Different summation orders and the gather form (x = y * deg) differ by
        # a few units in the last place per node: far below 1e-13 here.
        np.testing.assert_allclose(tr[:k], o.trace[:k], rtol=1e-9, atol=1e-13)


def test_residual_trace_capacity_and_plain_stats():
    csr, _ = load_golden("wikivote_directed")
    dg = _capi.DeviceGraph(csr)
    p = dg.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
    _, it, _, st = dg.run(p, trace=5)
    assert st["trace_length"] == it > 5
    assert st["residual_trace"].shape[0] == 5
    _, it2, _, st2 = dg.run(p)
    assert st2["trace_length"] == it2 and "residual_trace" not in st2


def _long_run_graph():
    csr = generators.rmat_directed(16, 16, seed=5)
    # tol 0: the run only ends at max_iterations (2e6 sweeps, many seconds),
    # unless it is cancelled.
    return csr, _capi.DeviceGraph.params(0.85, 0.0, 0, False, False, _capi.NKG_PREC_FP64,
                                         2_000_000)


def test_cancel_from_another_thread_then_run_again(oracle_mod):
    csr, p_long = _long_run_graph()
    dg = _capi.DeviceGraph(csr)
    dg.run(dg.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, 5))  # warm-up
    timer = threading.Timer(0.1, dg.cancel)
    t0 = time.perf_counter()
    timer.start()
    with pytest.raises(_capi.NkgError) as e:
        dg.run(p_long)
    timer.join()
    assert e.value.code == _capi.NKG_ERR_CANCELLED
    assert time.perf_counter() - t0 < 10.0
    p = dg.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, _capi.UINT64_MAX)
    s, it, _, _ = dg.run(p)
    o = oracle_mod.pagerank(csr, tol=1e-10, norm=0)
    assert np.abs(s - o.scores).sum() <= L1_FP64
    assert abs(it - o.iterations) <= 1


@pytest.mark.parametrize("prec", [_capi.NKG_PREC_FP64, _capi.NKG_PREC_FP32_REFINE])
def test_cancel_issued_before_the_run_is_kept(prec):
    csr, _ = _long_run_graph()
    dg = _capi.DeviceGraph(csr)
    p = dg.params(0.85, 1e-10, 0, False, False, prec, _capi.UINT64_MAX)
    dg.cancel()
    with pytest.raises(_capi.NkgError) as e:
        dg.run(p)
    assert e.value.code == _capi.NKG_ERR_CANCELLED
    # The request ended with that run: the next one completes.
    s, it, _, _ = dg.run(p)
    assert it > 1 and np.isfinite(s).all()


def _with_sigint_after(seconds, fn):
    """Call fn() while a timer sends this process SIGINT after `seconds`. A
    Python-level handler records a SIGINT that arrives outside the library's
    routing, so a late signal cannot stop the test session."""
    seen = []
    prev = signal.signal(signal.SIGINT, lambda *a: seen.append(1))
    timer = threading.Timer(seconds, os.kill, (os.getpid(), signal.SIGINT))
    try:
        timer.start()
        try:
            return fn(), seen
        finally:
            timer.join()
    finally:
        signal.signal(signal.SIGINT, prev)


def test_sigint_cancels_a_python_mirror_run():
    csr, _ = _long_run_graph()
    G = Graph.fromInCSR(csr)
    pr = centrality.PageRank(G, 0.85, 0.0)
    pr.norm = centrality.Norm.l1norm
    pr.maxIterations = 2_000_000

    def go():
        with pytest.raises(RuntimeError, match="Received CTRL\\+C/SIGINT"):
            pr.run()
        return True

    ok, seen = _with_sigint_after(0.2, go)
    assert ok and not seen
    # SIGINT is back with Python's handler chain, and a run completes.
    pr2 = centrality.PageRank(G, 0.85, 1e-10)
    pr2.norm = centrality.Norm.l1norm
    pr2.run()
    assert pr2.numberOfIterations() > 1


def test_sigint_cancels_a_cython_binding_run():
    cy = pytest.importorskip("networkit_b200._cypagerank")
    csr, _ = _long_run_graph()
    G = Graph.fromInCSR(csr)
    pr = cy.PageRank(G, 0.85, 0.0)
    pr.norm = 0
    pr.maxIterations = 2_000_000

    def go():
        with pytest.raises(RuntimeError, match="Received CTRL\\+C/SIGINT"):
            pr.run()
        return True

    ok, seen = _with_sigint_after(0.2, go)
    assert ok and not seen


def test_sigint_route_is_one_handle_at_a_time():
    a = _capi.DeviceGraph(generators.rmat_directed(10, 8, seed=1))
    b = _capi.DeviceGraph(generators.rmat_directed(10, 8, seed=2))
    a.sigint_cancels(True)
    try:
        with pytest.raises(_capi.NkgError, match="another graph handle"):
            b.sigint_cancels(True)
    finally:
        assert a.sigint_cancels(False) is False
    b.sigint_cancels(True)
    b.sigint_cancels(False)
