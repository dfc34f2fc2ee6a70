"""The oracle's ApproximatePageRank and PageRankNibble sweep against the
reference's own results (tests/golden/local_ppr.npz, written by the reference
library compiled from its sources: ApproximatePageRank.cpp:18-55,
PageRankNibble.cpp:28-89, on the graphs of SelectiveCDGTest.cpp).

Bars: ApproximatePageRank bit-exact (support and every value). The nibble
sets equal the reference's, except where the reference's unstable sort put a
group of equal p/vol values in another order than ascending id: then the two
sets may differ only inside that tie group, and both are prefixes of the
sweep order."""
import json
import os

import numpy as np
import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
D = np.load(os.path.join(HERE, "local_ppr.npz"))
CASES = json.loads(str(D["cases"]))
GRAPHS = json.loads(str(D["graphs"]))


def graph(name):
    w = D[f"{name}_w"]
    return (D[f"{name}_ptr"], D[f"{name}_col"], w if w.shape[0] else None,
            bool(D[f"{name}_directed"]), int(D[f"{name}_m"]), int(D[f"{name}_n"]))


def case_seeds(name, c):
    ptr = D[f"{name}_ptr"]
    seeds = [s for s in CASES[c][2] if s < ptr.shape[0] - 1]
    if not seeds:
        pytest.skip("no seed of this case inside the graph")
    return seeds


def sweep_prefix_ok(keys_by_node, support, chosen):
    """Every chosen node's key >= every unchosen support node's key."""
    inside = np.isin(support, chosen)
    if inside.all() or not inside.any():
        return True
    return keys_by_node[support[inside]].min() >= keys_by_node[support[~inside]].max()


def check_set(mine, ref, support, values, vol):
    mine, ref = np.asarray(mine), np.asarray(ref)
    if np.array_equal(mine, ref):
        return
    key = np.full(vol.shape[0], np.nan)
    key[support] = values / vol[support]
    diff = np.setxor1d(mine, ref)
    assert np.unique(key[diff]).shape[0] == 1, "sets differ outside one tie group"
    assert sweep_prefix_ok(key, support, mine) and sweep_prefix_ok(key, support, ref)


@pytest.mark.parametrize("name", GRAPHS)
@pytest.mark.parametrize("c", range(len(CASES)))
def test_apr_oracle_matches_reference(oracle_mod, name, c):
    ptr, col, w, directed, m, n = graph(name)
    z = ptr.shape[0] - 1
    alpha, eps, _ = CASES[c]
    res = oracle_mod.apr(z, ptr, col, w, case_seeds(name, c), alpha, eps)
    np.testing.assert_array_equal(res.nodes, D[f"{name}_{c}_apr_nodes"])
    np.testing.assert_array_equal(res.values.view(np.uint64),
                                  D[f"{name}_{c}_apr_values"].view(np.uint64))


@pytest.mark.parametrize("name", [g for g in GRAPHS if not bool(D[f"{g}_directed"])])
@pytest.mark.parametrize("c", range(len(CASES)))
def test_sweep_oracle_matches_reference(oracle_mod, name, c):
    ptr, col, w, directed, m, n = graph(name)
    z = ptr.shape[0] - 1
    alpha, eps, _ = CASES[c]
    seeds = case_seeds(name, c)
    vol = oracle_mod.volumes(z, ptr, col, w)
    total = 2.0 * (float(np.sum(w[np.repeat(np.arange(z), np.diff(ptr).astype(np.int64)) >= col]))
                   if w is not None else m)
    res = oracle_mod.apr(z, ptr, col, w, seeds, alpha, eps, vol)
    mine = oracle_mod.sweep_set(z, ptr, col, w, vol, total, n, res.nodes, res.values)
    check_set(mine, D[f"{name}_{c}_joint"], res.nodes, res.values, vol)
    for sd in seeds:
        r1 = oracle_mod.apr(z, ptr, col, w, [sd], alpha, eps, vol)
        m1 = oracle_mod.sweep_set(z, ptr, col, w, vol, total, n, r1.nodes, r1.values)
        check_set(m1, D[f"{name}_{c}_each_{sd}"], r1.nodes, r1.values, vol)


def test_reference_scd_test_case(oracle_mod):
    """SelectiveCDGTest.cpp:52-111: PageRankNibble(G, 0.1, 1e-5) from seed 50
    on hep-th yields a non-empty cluster with conductance below 1."""
    ptr, col, w, directed, m, n = graph("hepth")
    z = ptr.shape[0] - 1
    vol = oracle_mod.volumes(z, ptr, col, w)
    res = oracle_mod.apr(z, ptr, col, w, [50], 0.1, 1e-5, vol)
    s = oracle_mod.sweep_set(z, ptr, col, w, vol, 2.0 * m, n, res.nodes, res.values)
    assert s.shape[0] > 0
    inside = np.zeros(z, bool)
    inside[s] = True
    rows = np.repeat(np.arange(z), np.diff(ptr).astype(np.int64))
    cut = np.count_nonzero(inside[rows] & ~inside[col])
    vs = np.diff(ptr)[s].sum()
    assert cut / min(vs, 2 * m - vs) < 1.0
