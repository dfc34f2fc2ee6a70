"""The Erdos-Renyi workload graph is the reference generator's own draw.

`generators.erdos_renyi_stream` restates NetworKit's ErdosRenyiGenerator on
one OpenMP thread after setSeed(seed, False) (ErdosRenyiGenerator.cpp:21-33,
ErdosRenyiEnumerator.hpp). Pinned two ways: the SHA-256 digests of the
G(1e5, average degree 10) graph that the reference itself drew
(tests/golden/er_config.npz, made by tests/golden/make_golden.py), and, where
the reference library is built (oracle/_ref), array equality with the
reference's Graph on directed, undirected, sparse and dense (complement-pass)
cases. The oracle's PageRank on that graph then meets the reference's stored
run."""
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
    return generators.erdos_renyi_stream(int(g["n"]), float(g["p"]), int(g["seed"]))


def test_stream_graph_matches_the_reference_digests():
    g = golden()
    csr = er_graph()
    assert csr.in_ptr[-1] == int(g["arcs"])
    assert hashlib.sha256(csr.in_ptr.astype(np.uint64).tobytes()).hexdigest() == \
        g["in_ptr_sha256"].item().decode()
    assert hashlib.sha256(csr.in_col.astype(np.uint32).tobytes()).hexdigest() == \
        g["in_col_sha256"].item().decode()
    np.testing.assert_array_equal(csr.outdeg, np.diff(csr.in_ptr))


@pytest.mark.parametrize("n,p,directed", [(3000, 0.004, False), (2500, 0.003, True),
                                          (400, 0.95, False), (300, 0.92, True),
                                          (60, 0.0, False), (50, 1.0, True), (1, 0.5, False)])
def test_stream_graph_matches_the_reference_generator(oracle_mod, n, p, directed):
    if not oracle_mod.ref_available():
        pytest.skip("the reference library (oracle/_ref) is not built")
    ours = generators.erdos_renyi_stream(n, p, 42, directed)
    e = oracle_mod.RefGraph.erdos_renyi(n, p, 42, directed, threads=1).export()
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
