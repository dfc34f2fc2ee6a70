"""Many-graph batch (nkg_batch_*): every graph of a block-diagonal batch
against the oracle run on that graph alone.

Bars: FP64 L1 <= 1e-10 per graph (scaled by the sum for normalized scores)
and iterations within 1; FP32 L1 <= 2e-6 per graph (the FP32 rounding floor
of a unit-mass vector, hit before tol 1e-8)."""
import numpy as np
import pytest

from networkit_b200 import _capi, generators
from networkit_b200.graph import concat_in_csr

pytestmark = pytest.mark.gpu

DAMP = 0.85


def mixed_graphs():
    """Uneven shapes: hyperbolic graphs of several sizes (hubs above any
    split threshold), a directed R-MAT with sinks, an Erdos-Renyi graph with
    isolated nodes, a single node and a two-node path."""
    gs = [generators.hyperbolic_stream(n, 16, 3, seed=42 + i)
          for i, n in enumerate((200, 1500, 7000, 30000))]
    gs.append(generators.rmat_directed(12, 8, seed=3))
    gs.append(generators.erdos_renyi(3000, 1.5 / 2999, seed=5))
    from networkit_b200.graph import in_csr_from_edges
    gs.append(in_csr_from_edges(1, [], [], directed=True))
    gs.append(in_csr_from_edges(2, [0], [1], directed=True))
    return gs


@pytest.fixture(scope="module")
def batch():
    gs = mixed_graphs()
    csr, offs = concat_in_csr(gs)
    return gs, csr, offs, _capi.DeviceBatch(csr, offs)


def check(oracle_mod, gs, offs, scores, its, prec, norm, tol, distribute, normalized):
    for i, g in enumerate(gs):
        a, b = int(offs[i]), int(offs[i + 1])
        o = oracle_mod.pagerank(g, tol=tol, norm=norm, distribute_sinks=distribute,
                                normalized=normalized)
        got = scores[a:b]
        scale = max(1.0, float(np.abs(o.scores).sum())) if normalized else 1.0
        err = float(np.abs(got - o.scores).sum())
        if prec == _capi.NKG_PREC_FP64:
            assert err <= 1e-10 * scale, (i, err)
            assert abs(int(its[i]) - o.iterations) <= 1, (i, its[i], o.iterations)
        else:
            assert err <= 1e-6 * scale, (i, err)  # the companion forms' bar


@pytest.mark.parametrize("shape", [(1, 128, 4, 0), (2, 256, 32, 1), (4, 512, 128, 2), (8, 256, 1024, 3),
                                   (16, 256, 64, 0)])
@pytest.mark.parametrize("prec", [_capi.NKG_PREC_FP64, _capi.NKG_PREC_FP32])
def test_batch_matches_oracle_per_graph(oracle_mod, batch, shape, prec):
    gs, csr, offs, db = batch
    db.set_tuning(*shape)
    tol = 1e-10 if prec == _capi.NKG_PREC_FP64 else 1e-8
    p = _capi.PRParams(DAMP, tol, 0, 0, 0, prec, 10000)
    scores, its, floor, st = db.run(p)
    check(oracle_mod, gs, offs, scores, its, prec, 0, tol, False, False)
    assert st["iterations"] == int(its.sum())
    if prec == _capi.NKG_PREC_FP64:
        assert floor == 0
    start, end = db.graph_times()
    assert np.all(start >= 0) and np.all(end >= start) and end.max() <= st["ms_total"] + 1.0


@pytest.mark.parametrize("variant", ["l2", "distribute", "normalized"])
def test_batch_variants(oracle_mod, batch, variant):
    gs, csr, offs, db = batch
    db.set_tuning(4, 256, 64)
    norm = 1 if variant == "l2" else 0
    distribute = variant == "distribute"
    normalized = variant == "normalized"
    p = _capi.PRParams(DAMP, 1e-9, norm, int(normalized), int(distribute), _capi.NKG_PREC_FP64,
                       10000)
    scores, its, _, _ = db.run(p)
    check(oracle_mod, gs, offs, scores, its, _capi.NKG_PREC_FP64, norm, 1e-9, distribute,
          normalized)


def test_batch_runs_are_reproducible_and_device_output(batch):
    import torch

    gs, csr, offs, db = batch
    db.set_tuning(2, 512, 32)
    p = _capi.PRParams(DAMP, 1e-8, 0, 0, 0, _capi.NKG_PREC_FP32, 10000)
    a, its_a, _, _ = db.run(p)
    d = torch.empty(db.total, dtype=torch.float64, device="cuda:0")
    none, its_b, _, _ = db.run(p, d.data_ptr())
    assert none is None
    np.testing.assert_array_equal(d.cpu().numpy(), a)
    np.testing.assert_array_equal(its_a, its_b)


def test_batch_tuner(batch):
    gs, csr, offs, db = batch
    p = _capi.PRParams(DAMP, 1e-8, 0, 0, 0, _capi.NKG_PREC_FP32, 10000)
    best, table = db.tune(p, sweeps=4)
    assert len(table) >= 10
    assert best["ms"] == min(t["ms"] for t in table)
    assert db.tuning()["split"] == best["split"]
    for t in table:
        assert t["cluster"] in (1, 2, 4, 8, 16) and t["threads"] in (256, 512)
    # sweeps = 0: every candidate runs to convergence; the chosen shape then
    # gives the same results as any other within the bars.
    best0, table0 = db.tune(p, sweeps=0)
    assert best0["ms"] == min(t["ms"] for t in table0)
    scores, its, _, _ = db.run(p)
    check(__import__("oracle"), gs, offs, scores, its, _capi.NKG_PREC_FP32, 0, 1e-8, False, False)


def test_batch_rejects_bad_input():
    a = generators.rmat_directed(6, 4, seed=1)
    b = generators.rmat_directed(6, 4, seed=2)
    csr, offs = concat_in_csr([a, b])
    bad = csr.in_col.copy()
    bad[0] = np.uint32(offs[1] + 1)  # an arc into the other graph
    from networkit_b200.graph import InCSR
    c2 = InCSR(csr.z, csr.n, csr.in_ptr, bad, None, csr.wdeg, csr.outdeg, None, True)
    with pytest.raises(_capi.NkgError, match="different graphs"):
        _capi.DeviceBatch(c2, offs)
    db = _capi.DeviceBatch(csr, offs)
    with pytest.raises(_capi.NkgError, match="cluster"):
        db.set_tuning(3, 256, 64)
    with pytest.raises(_capi.NkgError, match="FP64 or FP32"):
        db.run(_capi.PRParams(DAMP, 1e-8, 0, 0, 0, _capi.NKG_PREC_FP32_REFINE, 100))
