"""Parity of the CUDA PageRank path (through the C ABI) with the oracle.

Bar (plain FP64): L1(scores - oracle) <= 1e-10, |iterations - oracle| <= 1,
ranking identical apart from (near-)exact ties. FP32: 1e-5 L1 at tol 1e-8."""
import numpy as np
import pytest

from conftest import GOLDEN_NAMES, load_golden
from networkit_b200 import Graph, _capi, centrality, generators
from networkit_b200.graph import InCSR

pytestmark = pytest.mark.gpu

L1_FP64 = 1e-10


def gpu_run(csr, damp=0.85, tol=1e-8, norm=1, normalized=False, distribute=False,
            precision=_capi.NKG_PREC_FP64, max_iterations=_capi.UINT64_MAX, teleport=None):
    dg = _capi.DeviceGraph(csr)
    p = dg.params(damp, tol, norm, normalized, distribute, precision, max_iterations)
    scores, it, mx, st = dg.run(p, teleport)
    return dg, scores, it, mx, st


def assert_ranking_equal(ids_gpu, ids_ref, scores, rel=1e-12):
    """Identical except where the two orders swap nodes whose scores tie to
    within rounding."""
    ids_gpu = np.asarray(ids_gpu, np.int64)
    ids_ref = np.asarray(ids_ref, np.int64)
    assert ids_gpu.shape == ids_ref.shape
    diff = np.flatnonzero(ids_gpu != ids_ref)
    for i in diff:
        a, b = scores[ids_gpu[i]], scores[ids_ref[i]]
        assert abs(a - b) <= rel * max(abs(a), abs(b)), (i, ids_gpu[i], ids_ref[i], a, b)


@pytest.mark.parametrize("name", GOLDEN_NAMES)
@pytest.mark.parametrize("norm", [0, 1])
@pytest.mark.parametrize("normalized", [False, True])
def test_fp64_matches_reference_fixtures(name, norm, normalized):
    csr, ref = load_golden(name)
    key = f"n{norm}_z{int(normalized)}"
    dg, s, it, mx, st = gpu_run(csr, norm=norm, normalized=normalized)
    ref_s = ref[key + "_scores"]
    scale = 1.0 if not normalized else float(np.abs(ref_s).sum())
    assert np.abs(s - ref_s).sum() <= L1_FP64 * scale
    assert abs(it - int(ref[key + "_iterations"])) <= 1
    assert abs(mx - float(ref[key + "_maximum"])) <= 1e-10 * max(1.0, abs(mx))
    ids, vals = dg.ranking(s)
    assert_ranking_equal(ids, ref[key + "_rank_ids"], s)
    np.testing.assert_array_equal(vals, s[ids.astype(np.int64)])
    assert st["kernel_launches"] > 0 and st["fp64_sweeps"] == it


@pytest.mark.parametrize("name", ["wikivote_directed", "celegans"])
def test_max_iterations_two(name):
    csr, ref = load_golden(name)
    dg, s, it, mx, st = gpu_run(csr, norm=1, max_iterations=2)
    assert it == int(ref["n1_z0_max2_iterations"]) == 2
    assert np.abs(s - ref["n1_z0_max2_scores"]).sum() <= L1_FP64


@pytest.mark.parametrize("distribute", [False, True])
@pytest.mark.parametrize("scale", [10, 16])
@pytest.mark.parametrize("arc_order", [0, 1])
@pytest.mark.parametrize("shape", [-1, 1, 2, 3])
def test_rmat_parity_l1(oracle_mod, distribute, scale, arc_order, shape):
    csr = generators.rmat_directed(scale, 16, seed=42)
    o = oracle_mod.pagerank(csr, tol=1e-10, norm=0, distribute_sinks=distribute)
    dg = _capi.DeviceGraph(csr, sweep_shape=shape, arc_order=arc_order)
    s, it, mx, st = dg.run(dg.params(0.85, 1e-10, 0, False, distribute, 0, _capi.UINT64_MAX))
    info = dg.info()
    assert info["slots"] >= csr.arcs and info["n"] == csr.z
    assert np.abs(s - o.scores).sum() <= L1_FP64
    assert abs(it - o.iterations) <= 1
    ids_o, _ = oracle_mod.ranking(o.scores)
    ids, _ = dg.ranking(s)
    assert_ranking_equal(ids, ids_o, o.scores)


def test_er_config_parity(oracle_mod):
    """G(n=1e5, avg degree 10) undirected as the reference's generator draws
    it from seed 42 on 8 threads, L2 1e-8, with and without distributeSinks: against the
    oracle, and (without, as this reference has no sink redistribution)
    against the reference's own stored run on that graph
    (tests/golden/er_config.npz): iterations within 1, every stored score
    and the stored top-100 ranking."""
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "er_config.npz"))
    csr = generators.erdos_renyi_stream(int(g["n"]), float(g["p"]), int(g["seed"]),
                                        threads=int(g["threads"]))
    assert csr.in_ptr[-1] == int(g["arcs"])
    for distribute in (False, True):
        o = oracle_mod.pagerank(csr, tol=1e-8, norm=1, distribute_sinks=distribute)
        dg, s, it, mx, st = gpu_run(csr, tol=1e-8, norm=1, distribute=distribute)
        assert np.abs(s - o.scores).sum() <= L1_FP64
        assert abs(it - o.iterations) <= 1
        if not distribute:
            k = int(g["sample_every"])
            assert abs(it - int(g["iterations"])) <= 1
            assert np.abs(s[::k] - g["scores_sample"]).sum() <= L1_FP64
            ids, _ = dg.ranking(s)
            assert_ranking_equal(ids[:100], g["rank_ids_top100"], s)


@pytest.mark.parametrize("n, deg", [(100_000, 10), (400_000, 8)])
def test_graphs_without_split_rows(oracle_mod, n, deg):
    """Graphs with no row over 256 arcs: the smaller one has few enough work
    units that the sweep's last CTA closes every iteration (no fix-up
    launch); the larger one has more than 8,192 units, so a fix-up with no
    split rows adds the units' partials. Both against the oracle, with and
    without distributeSinks, and bit-identical on a second run."""
    csr = generators.erdos_renyi(n, deg / (n - 1), seed=5)
    assert int(np.diff(csr.in_ptr.astype(np.int64)).max()) <= 256
    slices = (n + 31) // 32
    assert (slices <= 8192) == (n == 100_000)
    for distribute in (False, True):
        o = oracle_mod.pagerank(csr, tol=1e-10, norm=0, distribute_sinks=distribute)
        dg, s, it, mx, st = gpu_run(csr, tol=1e-10, norm=0, distribute=distribute)
        assert dg.info()["split_rows"] == 0
        assert np.abs(s - o.scores).sum() <= L1_FP64
        assert abs(it - o.iterations) <= 1
        s2, it2, _, _ = dg.run(dg.params(0.85, 1e-10, 0, False, distribute, 0, _capi.UINT64_MAX))
        np.testing.assert_array_equal(s2, s)
        assert it2 == it


def test_weighted_parity(oracle_mod):
    csr = generators.with_uniform_weights(generators.rmat_directed(14, 16, seed=9), seed=43)
    for normalized in (False, True):
        o = oracle_mod.pagerank(csr, tol=1e-10, norm=0, normalized=normalized)
        dg, s, it, mx, st = gpu_run(csr, tol=1e-10, norm=0, normalized=normalized)
        scale = 1.0 if not normalized else float(np.abs(o.scores).sum())
        assert np.abs(s - o.scores).sum() <= L1_FP64 * scale
        assert abs(it - o.iterations) <= 1
        assert abs(mx - o.maximum) <= 1e-10 * max(1.0, o.maximum)


def test_personalised_teleport(oracle_mod):
    csr = generators.rmat_directed(13, 8, seed=11)
    rng = np.random.default_rng(3)
    t = rng.random(csr.z)
    t /= t.sum()
    for distribute in (False, True):
        o = oracle_mod.pagerank(csr, tol=1e-12, norm=0, distribute_sinks=distribute, teleport=t)
        dg, s, it, mx, st = gpu_run(csr, tol=1e-12, norm=0, distribute=distribute, teleport=t)
        assert np.abs(s - o.scores).sum() <= L1_FP64
        assert abs(it - o.iterations) <= 1


def test_hub_rows_span_many_tiles(oracle_mod):
    """Star-like graph: one row of 50k in-arcs crosses ~25 tiles, plus empty
    and tiny rows around it."""
    n = 60000
    src = np.arange(1, 50001, dtype=np.int64)
    dst = np.zeros(50000, np.int64)
    extra_s = np.arange(50001, n - 1, dtype=np.int64)
    extra_d = extra_s + 1
    s_all = np.concatenate([src, extra_s, [0]])
    d_all = np.concatenate([dst, extra_d, [7]])
    G = Graph(n, directed=True)
    G.addEdges(s_all, d_all)
    csr = G.inCSR()
    o = oracle_mod.pagerank(csr, tol=1e-12, norm=0)
    dg, s, it, mx, st = gpu_run(csr, tol=1e-12, norm=0)
    assert np.abs(s - o.scores).sum() <= L1_FP64
    assert abs(it - o.iterations) <= 1


def test_deleted_nodes_keep_one_over_n(oracle_mod):
    G = Graph(10, directed=True)
    for u, v in [(0, 1), (1, 2), (2, 0), (3, 0), (5, 6), (6, 5), (9, 0)]:
        G.addEdge(u, v)
    G.removeNode(4)
    G.removeNode(8)
    csr = G.inCSR()
    o = oracle_mod.pagerank(csr, tol=1e-12, norm=0)
    pr = centrality.PageRank(G, 0.85, 1e-12)
    pr.norm = centrality.Norm.l1norm
    pr.run()
    s = np.array(pr.scores())
    assert np.abs(s - o.scores).sum() <= L1_FP64
    assert s[4] == 1.0 / 8 and s[8] == 1.0 / 8
    r = pr.ranking()
    assert len(r) == 8 and 4 not in [u for u, _ in r]


@pytest.mark.parametrize("n,edges", [(1, []), (2, []), (3, [(0, 1), (1, 2), (2, 0)]),
                                     (5, [(0, 0), (1, 1)])])
def test_tiny_and_degenerate_graphs(oracle_mod, n, edges):
    for directed in (True, False):
        G = Graph(n, directed=directed)
        for u, v in edges:
            G.addEdge(u, v)
        csr = G.inCSR()
        o = oracle_mod.pagerank(csr, norm=1)
        dg, s, it, mx, st = gpu_run(csr, norm=1)
        assert np.abs(s - o.scores).sum() <= L1_FP64
        assert abs(it - o.iterations) <= 1


def test_python_api_end_to_end_matches_golden():
    csr, ref = load_golden("wikivote_directed")
    G = Graph.fromInCSR(csr)
    pr = centrality.PageRank(G)
    assert pr.run() is pr
    assert pr.hasFinished()
    s = np.array(pr.scores())
    assert np.abs(s - ref["n1_z0_scores"]).sum() <= L1_FP64
    top = pr.ranking()[0]
    assert top[0] == 326 and abs(top[1] - 0.00460) <= 1e-3
    assert abs(pr.score(326) - top[1]) == 0.0
    assert pr.maximum() == 1.0
    assert abs(pr.numberOfIterations() - int(ref["n1_z0_iterations"])) <= 1
    assert 0.0 <= pr.centralization() <= 1.0


def test_fp32_close_to_fp64(oracle_mod):
    csr = generators.rmat_directed(15, 16, seed=5)
    o = oracle_mod.pagerank(csr, tol=1e-8, norm=0)
    dg, s, it, mx, st = gpu_run(csr, tol=1e-8, norm=0, precision=_capi.NKG_PREC_FP32)
    assert np.abs(s - o.scores).sum() <= 1e-5
    assert st["fp32_sweeps"] == it


@pytest.mark.parametrize("case", ["rmat", "rmat_distribute", "er_l2", "weighted", "personal",
                                  "normalized"])
def test_fp32_refine_reaches_fp64_accuracy(oracle_mod, case):
    """FP32 BiCGSTAB bulk solve + FP64 residual/correction rounds: the FP64
    stopping test holds at tol, so the result is as close to the oracle as
    the FP64 path (the bar: 1e-8 L1 at tol 1e-10; the reference's own answer
    is within ~tol/(1-d) of the fixed point)."""
    if case == "er_l2":
        csr, norm, tol = generators.erdos_renyi(50000, 10 / 49999, seed=42), 1, 1e-8
    elif case == "weighted":
        csr = generators.with_uniform_weights(generators.rmat_directed(14, 16, seed=9), seed=43)
        norm, tol = 0, 1e-10
    else:
        csr, norm, tol = generators.rmat_directed(15, 16, seed=4), 0, 1e-10
    distribute = case == "rmat_distribute"
    normalized = case == "normalized"
    tele = None
    if case == "personal":
        rng = np.random.default_rng(2)
        tele = rng.random(csr.z)
        tele /= tele.sum()
    o = oracle_mod.pagerank(csr, tol=tol, norm=norm, distribute_sinks=distribute,
                            normalized=normalized, teleport=tele)
    dg = _capi.DeviceGraph(csr)
    p = dg.params(0.85, tol, norm, normalized, distribute, _capi.NKG_PREC_FP32_REFINE,
                  _capi.UINT64_MAX)
    s, it, mx, st = dg.run(p, tele)
    scale = 1.0 if not normalized else float(np.abs(o.scores).sum())
    err = np.abs(s - o.scores).sum() / scale
    assert err <= (1e-8 if norm == 0 else 1e-6), err
    assert 1 <= st["fp64_sweeps"] <= 6 and st["fp32_sweeps"] >= 2
    assert st["residual"] <= tol
    assert it == st["fp64_sweeps"] + st["fp32_sweeps"]


def test_invalid_arguments_raise():
    csr = generators.rmat_directed(8, 4, seed=1)
    bad = InCSR(csr.z, csr.n, csr.in_ptr, csr.in_col.copy(), None, csr.wdeg, csr.outdeg, None,
                True)
    bad.in_col[3] = csr.z + 5
    with pytest.raises(_capi.NkgError, match="node id >= z"):
        _capi.DeviceGraph(bad)
    bad2 = InCSR(csr.z, csr.n, csr.in_ptr.copy(), csr.in_col, None, csr.wdeg, csr.outdeg, None,
                 True)
    bad2.in_ptr[5] = bad2.in_ptr[6] + 1
    with pytest.raises(_capi.NkgError):
        _capi.DeviceGraph(bad2)
    dg = _capi.DeviceGraph(csr)
    with pytest.raises(_capi.NkgError, match="norm"):
        dg.run(dg.params(0.85, 1e-8, 7, False, False, 0, 100))


def test_repeated_runs_are_bit_identical():
    csr = generators.rmat_directed(14, 16, seed=2)
    dg = _capi.DeviceGraph(csr)
    p = dg.params(0.85, 1e-10, 0, False, True, 0, _capi.UINT64_MAX)
    a = dg.run(p)
    b = dg.run(p)
    np.testing.assert_array_equal(a[0], b[0])
    assert a[1] == b[1]


@pytest.mark.parametrize("norm", [0, 1])
def test_queued_sweep_sums_do_not_depend_on_the_schedule(norm):
    """Warps take the sweep's work units from a counter, so which warp runs
    which unit changes from sweep to sweep. Every unit's partial sums have a
    slot of their own and are added in a fixed order: the residual of every
    sweep, the iteration count and the scores repeat bit for bit (R-MAT 16,
    with rows split into chunks)."""
    csr = generators.rmat_directed(16, 16, seed=11)
    dg = _capi.DeviceGraph(csr)
    assert dg.info()["split_rows"] > 0
    p = dg.params(0.85, 1e-10, norm, False, True, 0, _capi.UINT64_MAX)
    runs = [dg.run(p, trace=256) for _ in range(3)]
    for s, it, mx, st in runs[1:]:
        np.testing.assert_array_equal(s, runs[0][0])
        assert it == runs[0][1]
        np.testing.assert_array_equal(st["residual_trace"].view(np.uint64),
                                      runs[0][3]["residual_trace"].view(np.uint64))
    assert runs[0][3]["residual_trace"].shape[0] == runs[0][1]


def test_memory_pool_reuse_and_release(oracle_mod):
    """Graphs created and destroyed in a loop reuse the library's cached
    device memory and give the same scores; nkg_release_cached_memory hands
    the cache back to the driver."""
    import torch

    from networkit_b200 import generators

    csr = generators.rmat_directed(14, 8, seed=5)
    free0 = torch.cuda.mem_get_info()[0]
    first = None
    for _ in range(3):
        g = _capi.DeviceGraph(csr)
        p = g.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, 1000)
        s, it, _, _ = g.run(p)
        g.close()
        if first is None:
            first = (s, it)
        np.testing.assert_array_equal(s, first[0])
    _capi.check(_capi.lib().nkg_release_cached_memory(-1))
    assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)
    o = oracle_mod.pagerank(csr, tol=1e-10, norm=0)
    assert np.abs(first[0] - o.scores).sum() <= 1e-10


@pytest.mark.parametrize("row_order", [0, 1, -1])
def test_row_order_relabelling(oracle_mod, row_order):
    """The half-octave bucket relabelling (and its automatic choice) changes
    only the layout: FP64 scores within 1e-10 L1 of the oracle and the
    iteration count within 1, on an angle-numbered hyperbolic graph (auto
    picks buckets) and on R-MAT (auto keeps in-degree order)."""
    from networkit_b200 import generators

    hyp = generators.hyperbolic(30000, 16, 3, seed=4)
    rmat = generators.rmat_directed(14, 16, seed=9)
    for csr, auto_pick in ((hyp, 1), (rmat, 0)):
        dg = _capi.DeviceGraph(csr, row_order=row_order)
        assert dg.info()["row_order"] == (auto_pick if row_order == -1 else row_order)
        p = dg.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP64, 10000)
        s, it, _, _ = dg.run(p)
        o = oracle_mod.pagerank(csr, tol=1e-10, norm=0)
        assert np.abs(s - o.scores).sum() <= 1e-10
        assert abs(it - o.iterations) <= 1
        p32 = dg.params(0.85, 1e-10, 0, False, False, _capi.NKG_PREC_FP32_REFINE, 10000)
        s32, _, _, _ = dg.run(p32)
        assert np.abs(s32 - o.scores).sum() <= 1e-9
        dg.close()


def test_rmat20_matches_the_reference_library(oracle_mod):
    """The benchmark's kind of graph at scale 20 against the reference's own
    PageRank::run() (oracle/_ref, all host cores), not only the C
    restatement: L1 <= 1e-10, iterations within 1, ranking identical apart
    from ties (the reference's ranking comes from its Centrality::ranking)."""
    import os

    if not oracle_mod.ref_available():
        pytest.skip("the reference library (oracle/_ref) is not built")
    csr = generators.rmat_directed(20, 16, seed=42)
    rows = np.repeat(np.arange(csr.z, dtype=np.uint32), np.diff(csr.in_ptr).astype(np.int64))
    rg = oracle_mod.RefGraph.from_edges(csr.z, csr.in_col, rows, directed=True)
    r = rg.pagerank(damp=0.85, tol=1e-10, norm=0, nthreads=os.cpu_count() or 1,
                    want_ranking=True)
    dg, s, it, _, _ = gpu_run(csr, tol=1e-10, norm=0)
    assert np.abs(s - r["scores"]).sum() <= L1_FP64
    assert abs(it - r["iterations"]) <= 1
    ids, _ = dg.ranking(s)
    assert_ranking_equal(ids, r["ranking_ids"], s)
