"""The Erdos-Renyi, Barabasi-Albert and random hyperbolic workload graphs
are the reference generators' own draws.

`generators.erdos_renyi_stream` restates NetworKit's ErdosRenyiGenerator on
a given number of OpenMP threads after setSeed(seed, False)
(ErdosRenyiGenerator.cpp:21-33, ErdosRenyiEnumerator.hpp). Pinned two ways:
the SHA-256 digests of the G(1e5, average degree 10) graph that the reference
itself drew on 8 threads (tests/golden/er_config.npz, made by
tests/golden/make_golden.py), and, where the reference library is built
(oracle/_ref), array equality with the reference's Graph on directed,
undirected, sparse and dense (complement-pass) cases and 1 to 16 threads. The oracle's PageRank on that graph then meets the reference's stored
run. `generators.barabasi_albert_stream` restates BarabasiAlbertGenerator's
default (Batagelj-Brandes) draw, pinned the same two ways: the digests of the
n = 4M, k = 8 graph of the batched-PPR workload (tests/golden/ba_config.npz)
and equality with the reference's Graph on small cases.
`generators.hyperbolic_stream` restates HyperbolicGenerator (threshold
model), pinned by the digests of three graphs up to the 4M-node one
(tests/golden/rhg_config.npz) and by equality with the reference's Graph
(one thread) on other sizes, degrees and exponents; its batch form draws
graph i as the single-graph form with seed + i."""
import hashlib
import os

import numpy as np
import pytest

from networkit_b200 import generators

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "er_config.npz")


def golden():
    return np.load(GOLDEN)


def er_graph():
    g = golden()
    return generators.erdos_renyi_stream(int(g["n"]), float(g["p"]), int(g["seed"]),
                                         threads=int(g["threads"]))


def test_stream_graph_matches_the_reference_digests():
    g = golden()
    csr = er_graph()
    assert csr.in_ptr[-1] == int(g["arcs"])
    assert hashlib.sha256(csr.in_ptr.astype(np.uint64).tobytes()).hexdigest() == \
        g["in_ptr_sha256"].item().decode()
    assert hashlib.sha256(csr.in_col.astype(np.uint32).tobytes()).hexdigest() == \
        g["in_col_sha256"].item().decode()
    np.testing.assert_array_equal(csr.outdeg, np.diff(csr.in_ptr))


@pytest.mark.parametrize("n,p,directed,threads", [
    (3000, 0.004, False, 1), (3000, 0.004, False, 3), (2500, 0.003, True, 1),
    (2500, 0.003, True, 8), (400, 0.95, False, 1), (400, 0.95, False, 4), (300, 0.92, True, 5),
    (60, 0.0, False, 2), (50, 1.0, True, 1), (1, 0.5, False, 1), (7, 0.5, False, 16),
    (20000, 5e-4, False, 8)])
def test_stream_graph_matches_the_reference_generator(oracle_mod, n, p, directed, threads):
    if not oracle_mod.ref_available():
        pytest.skip("the reference library (oracle/_ref) is not built")
    ours = generators.erdos_renyi_stream(n, p, 42, directed, threads=threads)
    e = oracle_mod.RefGraph.erdos_renyi(n, p, 42, directed, threads=threads).export()
    ptr, adj = (e["in_ptr"], e["in_adj"]) if directed else (e["out_ptr"], e["out_adj"])
    np.testing.assert_array_equal(ours.in_ptr, ptr)
    np.testing.assert_array_equal(ours.in_col, adj)
    np.testing.assert_array_equal(ours.outdeg, np.diff(e["out_ptr"]))


def test_oracle_on_the_reference_graph_meets_the_reference_run(oracle_mod):
    g = golden()
    o = oracle_mod.pagerank(er_graph(), tol=1e-8, norm=1)
    assert o.iterations == int(g["iterations"])
    k = int(g["sample_every"])
    np.testing.assert_allclose(o.scores[::k], g["scores_sample"], rtol=0, atol=1e-15)


def test_stream_generator_rejects_bad_arguments():
    with pytest.raises(RuntimeError, match="p must be"):
        generators.erdos_renyi_stream(10, 1.5)
    with pytest.raises(RuntimeError, match="n out of range"):
        generators.erdos_renyi_stream(0, 0.5)
    with pytest.raises(RuntimeError, match="threads"):
        generators.erdos_renyi_stream(10, 0.5, threads=0)


BA_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ba_config.npz")


def test_ba_stream_graph_matches_the_reference_digests():
    g = np.load(BA_GOLDEN)
    csr = generators.barabasi_albert_stream(int(g["k"]), int(g["n"]), int(g["seed"]))
    assert csr.in_ptr[-1] == int(g["arcs"])
    assert hashlib.sha256(csr.in_ptr.astype(np.uint64).tobytes()).hexdigest() == \
        g["in_ptr_sha256"].item().decode()
    assert hashlib.sha256(csr.in_col.astype(np.uint32).tobytes()).hexdigest() == \
        g["in_col_sha256"].item().decode()


@pytest.mark.parametrize("k,n,n0", [(8, 20000, 0), (1, 500, 0), (3, 1000, 10), (2, 2, 0),
                                    (5, 3000, 2), (4, 4, 4)])
def test_ba_stream_graph_matches_the_reference_generator(oracle_mod, k, n, n0):
    if not oracle_mod.ref_available():
        pytest.skip("the reference library (oracle/_ref) is not built")
    ours = generators.barabasi_albert_stream(k, n, 42, n0)
    e = oracle_mod.RefGraph.barabasi_albert(k, n, 42, n0).export()
    np.testing.assert_array_equal(ours.in_ptr, e["out_ptr"])
    np.testing.assert_array_equal(ours.in_col, e["out_adj"])
    np.testing.assert_array_equal(ours.outdeg, np.diff(e["out_ptr"]))


def test_ba_stream_generator_rejects_bad_arguments():
    with pytest.raises(RuntimeError, match="k must be"):
        generators.barabasi_albert_stream(0, 10)
    with pytest.raises(RuntimeError, match="larger than the number of nodes"):
        generators.barabasi_albert_stream(11, 10)
    with pytest.raises(RuntimeError, match="n0 may not"):
        generators.barabasi_albert_stream(2, 10, n0=11)


RHG_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "rhg_config.npz")


@pytest.mark.parametrize("n,seed", [(1000, 42), (200_000, 42), (4_000_000, 21)])
def test_hyperbolic_stream_graph_matches_the_reference_digests(n, seed):
    g = np.load(RHG_GOLDEN)
    key = f"{n}_{seed}_"
    csr = generators.hyperbolic_stream(n, 16.0, 3.0, seed)
    assert csr.in_ptr[-1] == int(g[key + "arcs"])
    assert hashlib.sha256(csr.in_ptr.astype(np.uint64).tobytes()).hexdigest() == \
        g[key + "in_ptr_sha256"].item().decode()
    assert hashlib.sha256(csr.in_col.astype(np.uint32).tobytes()).hexdigest() == \
        g[key + "in_col_sha256"].item().decode()


@pytest.mark.parametrize("n,deg,exp,seed", [(5000, 16, 3, 7), (20000, 8, 2.5, 1),
                                            (3000, 30, 4, 3), (300, 4, 2.1, 9)])
def test_hyperbolic_stream_graph_matches_the_reference_generator(oracle_mod, n, deg, exp, seed):
    if not oracle_mod.ref_available():
        pytest.skip("the reference library (oracle/_ref) is not built")
    ours = generators.hyperbolic_stream(n, deg, exp, seed)
    e = oracle_mod.RefGraph.hyperbolic(n, deg, exp, seed, threads=1).export()
    np.testing.assert_array_equal(ours.in_ptr, e["out_ptr"])
    np.testing.assert_array_equal(ours.in_col, e["out_adj"])


def test_hyperbolic_stream_batch_is_the_single_graphs():
    ns = [1000, 2500, 1200]
    csr, offs = generators.hyperbolic_stream_batch(ns, 16.0, 3.0, seed=5)
    np.testing.assert_array_equal(offs, np.cumsum([0] + ns))
    for i, n in enumerate(ns):
        g = generators.hyperbolic_stream(n, 16.0, 3.0, 5 + i)
        a, b = int(offs[i]), int(offs[i + 1])
        rows = csr.in_ptr[a:b + 1] - csr.in_ptr[a]
        np.testing.assert_array_equal(rows, g.in_ptr)
        np.testing.assert_array_equal(
            csr.in_col[int(csr.in_ptr[a]):int(csr.in_ptr[b])] - a, g.in_col)


def test_hyperbolic_stream_rejects_bad_arguments():
    with pytest.raises(RuntimeError, match="Exponent"):
        generators.hyperbolic_stream(1000, 16, 2.0)
    with pytest.raises(RuntimeError, match="Average Degree"):
        generators.hyperbolic_stream(10, 16, 3.0)
