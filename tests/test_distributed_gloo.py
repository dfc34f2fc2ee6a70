"""The sharded multi-GPU forms (networkit_b200.distributed) on CPU ranks.

Two gloo ranks run the collective logic of each form with the oracle's
arithmetic standing in for the GPU kernels:

* the 1-D row partition of one PageRank run: each rank sweeps its row slices
  with the oracle's restatement of PageRank.cpp:56-66 (nko_sweep_rows),
  all-gathers the slices and all-reduces the residual and sink partial sums.
  Every row is summed in the reference's arc order, so the result equals the
  single-process oracle bit for bit (at the same iteration count);
* batched personalised PageRank with its columns dealt to the ranks;
* the many-graph batch with its graphs dealt to the ranks by arc count.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from networkit_b200 import distributed, generators  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _graph(name):
    from conftest import load_golden

    if name == "rmat12":
        return generators.rmat_directed(12, 16, seed=7)
    if name == "rmat11_weighted":
        return generators.with_uniform_weights(generators.rmat_directed(11, 8, seed=3), seed=5)
    csr, _ = load_golden(name)
    return csr


CASES = [("wikivote_directed", dict(norm=0, tol=1e-10)),
         ("wikivote_undirected", dict(norm=1, tol=1e-8, normalized=True)),
         ("rmat12", dict(norm=0, tol=1e-10)),
         ("rmat11_weighted", dict(norm=1, tol=1e-9)),
         ("rmat12", dict(norm=0, tol=1e-10, distribute_sinks=True))]


def _sub(c, a, b):
    from networkit_b200.graph import InCSR

    pa, pb = int(c.in_ptr[a]), int(c.in_ptr[b])
    ptr = (c.in_ptr[a:b + 1] - c.in_ptr[a]).astype(np.uint64)
    col = (c.in_col[pa:pb].astype(np.int64) - a).astype(np.uint32)
    deg = np.bincount(col, minlength=b - a).astype(np.uint32)
    return InCSR(b - a, b - a, ptr, col, None, deg.astype(np.float64), deg, None, False)


def _worker(rank, world, port, parts_per_rank, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle

    from networkit_b200 import _capi

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        res = {}
        for i, (name, kw) in enumerate(CASES):
            csr = _graph(name)
            s, it, mx, st = distributed.pagerank_row_partitioned(
                csr, backend="oracle", parts_per_rank=parts_per_rank, **kw)
            res[i] = (s, it, mx, st["residual_trace"])
        # Batched personalised PageRank, columns dealt to the ranks.
        g = _graph("rmat12")
        seeds = np.array([5, 17, 400, 1023, 2048, 3000, 4000], np.uint32)

        def solve_ppr(block):
            rows = []
            for sd in block.tolist():
                t = np.zeros(g.z)
                t[sd] = 1.0
                rows.append(oracle.pagerank(g, tol=1e-9, norm=0, teleport=t).scores)
            return np.array(rows, np.float32).reshape(len(rows), g.z)

        p = _capi.PRParams(0.85, 1e-9, 0, 0, 0, _capi.NKG_PREC_FP32, 1000)
        res["ppr"] = distributed.ppr_column_sharded(g, seeds, p, solve=solve_ppr)
        # Many-graph batch, graphs dealt by arc count.
        sizes = [300, 50, 1200, 80, 700, 40, 500]
        csr_b, offs = generators.hyperbolic_batch(np.array(sizes, np.uint64), 8.0, 3.0, seed=9)

        def solve_batch(c, o):
            out = np.empty(int(o[-1]))
            for k in range(o.shape[0] - 1):
                a, b = int(o[k]), int(o[k + 1])
                out[a:b] = oracle.pagerank(_sub(c, a, b), tol=1e-12, norm=0).scores
            return out

        res["batch"] = distributed.batch_graph_sharded(csr_b, offs, p, solve=solve_batch)
        res["batch_in"] = (csr_b, offs)
        out[rank] = res
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module", params=[1, 2], ids=["1slice_per_rank", "2slices_per_rank"])
def gloo_results(request):
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), request.param, out), nprocs=world,
                       join=True, start_method="spawn")
    return dict(out), request.param


def test_row_partition_equals_single_process_oracle(gloo_results, oracle_mod):
    out, _ = gloo_results
    for i, (name, kw) in enumerate(CASES):
        csr = _graph(name)
        o = oracle_mod.pagerank(csr, **kw)
        s0, it0, mx0, tr0 = out[0][i]
        s1, it1, mx1, tr1 = out[1][i]
        # Every rank ends with the same scores.
        np.testing.assert_array_equal(s0, s1)
        assert it0 == it1 and mx0 == mx1
        assert abs(it0 - o.iterations) <= 1, (name, it0, o.iterations)
        if kw.get("distribute_sinks"):
            # The sink mass is reduced slice by slice: equal up to rounding.
            assert np.abs(s0 - o.scores).sum() <= 1e-12, name
        elif it0 == o.iterations:
            np.testing.assert_array_equal(s0.view(np.uint64), o.scores.view(np.uint64))
            assert mx0 == o.maximum
        else:
            assert np.abs(s0 - o.scores).sum() <= 1e-10, name
        k = min(len(tr0), o.trace.shape[0])
        np.testing.assert_allclose(tr0[:k], o.trace[:k], rtol=1e-9, atol=1e-14)


def test_ppr_columns_dealt_to_ranks(gloo_results, oracle_mod):
    out, _ = gloo_results
    g = _graph("rmat12")
    seeds = [5, 17, 400, 1023, 2048, 3000, 4000]
    a, b = out[0]["ppr"], out[1]["ppr"]
    np.testing.assert_array_equal(a, b)
    assert a.shape == (len(seeds), g.z)
    for j, sd in enumerate(seeds):
        t = np.zeros(g.z)
        t[sd] = 1.0
        ref = oracle_mod.pagerank(g, tol=1e-9, norm=0, teleport=t).scores.astype(np.float32)
        np.testing.assert_array_equal(a[j], ref)


def test_batch_graphs_dealt_to_ranks(gloo_results, oracle_mod):
    out, _ = gloo_results
    csr_b, offs = out[0]["batch_in"]
    a, b = out[0]["batch"], out[1]["batch"]
    np.testing.assert_array_equal(a, b)
    for k in range(offs.shape[0] - 1):
        lo, hi = int(offs[k]), int(offs[k + 1])
        ref = oracle_mod.pagerank(_sub(csr_b, lo, hi), tol=1e-12, norm=0).scores
        np.testing.assert_array_equal(a[lo:hi], ref)


def test_row_plan_balances_and_covers():
    g = generators.rmat_directed(14, 16, seed=1)
    for parts in (1, 2, 3, 8):
        plan = distributed.RowPlan(g.in_ptr, parts)
        assert plan.bounds[0] == 0 and plan.bounds[-1] == g.z
        assert np.all(np.diff(plan.bounds) >= 1)
        cost = [int(g.in_ptr[plan.bounds[q + 1]] - g.in_ptr[plan.bounds[q]])
                + int(plan.rows[q]) for q in range(parts)]
        # Every slice's cost is within one row's arcs of the even share.
        assert max(cost) - (g.arcs + g.z) / parts <= int(np.diff(g.in_ptr).max()) + 1
        ids = np.arange(g.z)
        pos = plan.position(ids)
        assert np.unique(pos).shape[0] == g.z and int(pos.max()) < plan.vec_len - 1
        v = np.zeros(plan.vec_len)
        v[pos] = ids
        np.testing.assert_array_equal(plan.unpad(v), ids)
    with pytest.raises(ValueError):
        distributed.RowPlan(np.array([0, 1, 2], np.uint64), 3)


def test_dealing_is_balanced_and_complete():
    cols = distributed.deal_columns(256, 3)
    assert cols[0][0] == 0 and cols[-1][1] == 256
    assert max(b - a for a, b in cols) - min(b - a for a, b in cols) <= 1
    arcs = np.array([100, 5, 90, 7, 60, 3, 30])
    own = distributed.deal_graphs(arcs, 2)
    assert sorted(own[0] + own[1]) == list(range(7))
    loads = [int(arcs[o].sum()) for o in own]
    assert abs(loads[0] - loads[1]) <= arcs.max()
