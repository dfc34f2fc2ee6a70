"""ApproximatePageRank / PageRankNibble on the GPU (nkg_local_*).

ApproximatePageRank: bit-exact against the reference's results
(tests/golden/local_ppr.npz) and against the oracle on generated graphs with
multi-edges, self-loops, isolated seeds, deleted nodes and weights; many
problems per launch. PageRankNibble: the same sets as the oracle's sweep (the
same tie order: ascending id), on unweighted graphs; on weighted graphs cut
and volume are rounded in another order, so the conductance may differ in the
last bits."""
import json
import os

import numpy as np
import pytest

from networkit_b200 import _capi, scd
from networkit_b200.graph import Graph

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# Every run is bounded: far above the pushes of any case here (< 10^6).
MAXP = 50_000_000
D = np.load(os.path.join(HERE, "local_ppr.npz"))
CASES = json.loads(str(D["cases"]))
GRAPHS = json.loads(str(D["graphs"]))


def fixture_graph(name):
    w = D[f"{name}_w"]
    return (D[f"{name}_ptr"], D[f"{name}_col"], w if w.shape[0] else None,
            bool(D[f"{name}_directed"]), int(D[f"{name}_m"]), int(D[f"{name}_n"]))


def total_volume(ptr, col, w, m, directed):
    if w is None:
        return 2.0 * m
    z = ptr.shape[0] - 1
    rows = np.repeat(np.arange(z), np.diff(ptr).astype(np.int64))
    s = 0.0
    for k in range(col.shape[0]):  # forEdges order
        if directed or rows[k] >= col[k]:
            s += w[k]
    return 2.0 * s


def bits(a):
    return np.asarray(a, np.float64).view(np.uint64)


@pytest.mark.parametrize("name", GRAPHS)
def test_apr_matches_reference_fixtures(name):
    ptr, col, w, directed, m, n = fixture_graph(name)
    z = ptr.shape[0] - 1
    dl = _capi.DeviceLocal(z, ptr, col, w, None, directed)
    for c, (alpha, eps, seeds) in enumerate(CASES):
        seeds = [s for s in seeds if s < z]
        if not seeds:
            continue
        (sup,), _, st = dl.run([seeds], alpha, eps, max_pushes=MAXP)
        np.testing.assert_array_equal(sup[0], D[f"{name}_{c}_apr_nodes"])
        np.testing.assert_array_equal(bits(sup[1]), bits(D[f"{name}_{c}_apr_values"]))
        assert st["support"] == sup[0].shape[0]


@pytest.mark.parametrize("name", [g for g in GRAPHS if not bool(D[f"{g}_directed"])])
def test_nibble_matches_oracle_and_reference(oracle_mod, name):
    ptr, col, w, directed, m, n = fixture_graph(name)
    z = ptr.shape[0] - 1
    vol = oracle_mod.volumes(z, ptr, col, w)
    tv = total_volume(ptr, col, w, m, directed)
    dl = _capi.DeviceLocal(z, ptr, col, w, None, directed)
    for c, (alpha, eps, seeds) in enumerate(CASES):
        seeds = [s for s in seeds if s < z]
        if not seeds:
            continue
        problems = [seeds] + [[s] for s in seeds]
        keys = ["joint"] + [f"each_{s}" for s in seeds]
        sups, sets, _ = dl.run(problems, alpha, eps, nibble=True, max_pushes=MAXP)
        for pr, key, (nodes, vals), got in zip(problems, keys, sups, sets):
            want = oracle_mod.sweep_set(z, ptr, col, w, vol, tv, n, nodes, vals)
            if w is None:
                np.testing.assert_array_equal(got, want)
            ref = D[f"{name}_{c}_{key}"]
            if not np.array_equal(got, ref):
                key_of = np.full(z, np.nan)
                key_of[nodes] = vals / vol[nodes]
                diff = np.setxor1d(got, ref)
                assert np.unique(key_of[diff]).shape[0] == 1, (name, c, key)


def random_graph(z, m, seed, directed, weighted, loops=True, dups=True):
    rng = np.random.default_rng(seed)
    src = ((z - 30) * rng.random(m) ** 2).astype(np.int64)
    dst = ((z - 30) * rng.random(m)).astype(np.int64)
    if not loops:
        keep = src != dst
        src, dst = src[keep], dst[keep]
    if dups:
        src = np.concatenate([src, src[: m // 10]])
        dst = np.concatenate([dst, dst[: m // 10]])
    g = Graph(z, weighted=weighted, directed=directed)
    w = rng.integers(1, 6, src.shape[0]).astype(np.float64) * 0.5 if weighted else None
    g.addEdges(src, dst, w)
    g.removeNode(z - 1)
    return g


@pytest.mark.parametrize("directed", [False, True])
@pytest.mark.parametrize("weighted", [False, True])
def test_many_problems_against_oracle(oracle_mod, directed, weighted):
    """Multi-edges (duplicate neighbours in one 32-arc chunk), self-loops,
    isolated seeds (volume 0: the residual halves until it underflows),
    deleted nodes and 300 problems in one launch."""
    g = random_graph(6000, 40000, 7, directed, weighted)
    z, ptr, col, w, ex, dr = scd.neighbour_csr(g)
    vol = oracle_mod.volumes(z, ptr, col, w)
    rng = np.random.default_rng(1)
    problems = [[int(s)] for s in rng.integers(0, z - 31, 250)]
    problems += [sorted(set(rng.integers(0, z - 31, 4).tolist())) for _ in range(40)]
    problems += [[z - 10], [z - 5, 3], [0, z - 2]]  # isolated ids
    dl = _capi.DeviceLocal(z, ptr, col, w, ex, dr)
    for alpha, eps in [(0.1, 1e-5), (0.3, 1e-7)]:
        sups, _, st = dl.run(problems, alpha, eps, max_pushes=MAXP)
        assert st["slots"] >= 1
        pushes = 0
        for pr, (nodes, vals) in zip(problems, sups):
            o = oracle_mod.apr(z, ptr, col, w, pr, alpha, eps, vol)
            np.testing.assert_array_equal(nodes, o.nodes)
            np.testing.assert_array_equal(bits(vals), bits(o.values))
            pushes += o.pushes
        assert st["pushes"] == pushes


def test_small_budget_and_reuse(oracle_mod):
    """One slot (a tiny memory budget) runs the problems one after another;
    the epoch stamps keep every problem's map separate."""
    g = random_graph(3000, 20000, 3, False, False)
    z, ptr, col, w, ex, dr = scd.neighbour_csr(g)
    dl = _capi.DeviceLocal(z, ptr, col, w, ex, dr, memory_budget=1)
    problems = [[5], [5], [7, 9], [5]]
    for _ in range(2):
        sups, _, st = dl.run(problems, 0.15, 1e-6, max_pushes=MAXP)
        assert st["slots"] == 1
        for pr, (nodes, vals) in zip(problems, sups):
            o = oracle_mod.apr(z, ptr, col, w, pr, 0.15, 1e-6)
            np.testing.assert_array_equal(nodes, o.nodes)
            np.testing.assert_array_equal(bits(vals), bits(o.values))


def test_python_mirror():
    g = random_graph(2000, 12000, 5, False, False, dups=False)
    apr = scd.ApproximatePageRank(g, 0.2, 1e-6)
    apr.maxPushes = MAXP
    res = apr.run(17)
    assert res and all(a < b for (a, _), (b, _) in zip(res, res[1:]))
    assert dict(res) == dict(apr.run({17}))
    prn = scd.PageRankNibble(g, 0.1, 1e-5)
    prn.maxPushes = MAXP
    comm = prn.run({3, 17})
    assert set(comm) == {3, 17}
    assert comm[17] == prn.expandOneCommunity(17)
    many = prn.expandMany([3, 17, {3, 17}])
    assert set(many[1].tolist()) == comm[17]


def test_errors():
    g = random_graph(500, 3000, 2, False, False)
    z, ptr, col, w, ex, dr = scd.neighbour_csr(g)
    dl = _capi.DeviceLocal(z, ptr, col, w, ex, dr)
    with pytest.raises(_capi.NkgError, match="epsilon"):
        dl.run([[1]], 0.1, 0.0, max_pushes=MAXP)
    with pytest.raises(_capi.NkgError, match="seed id"):
        dl.run([[z + 3]], 0.1, 1e-4, max_pushes=MAXP)
    with pytest.raises(_capi.NkgError, match="non-existent"):
        dl.run([[z - 1]], 0.1, 1e-4, max_pushes=MAXP)
    with pytest.raises(_capi.NkgError, match="alpha"):
        dl.run([[1]], 0.0, 1e-4, max_pushes=MAXP)
    with pytest.raises(_capi.NkgError, match="non-negative"):
        _capi.DeviceLocal(3, np.array([0, 1, 1, 1], np.uint64), np.array([2], np.uint32),
                          np.array([-1.0]))
    with pytest.raises(_capi.NkgError, match="push limit"):
        dl.run([[1]], 0.1, 1e-9, max_pushes=3)
    with pytest.raises(_capi.NkgError, match="neighbour id"):
        _capi.DeviceLocal(3, np.array([0, 1, 1, 1], np.uint64), np.array([7], np.uint32))
    # the handle stays usable after an error
    sups, _, _ = dl.run([[1]], 0.1, 1e-4, max_pushes=MAXP)
    assert sups[0][0].shape[0] >= 1
