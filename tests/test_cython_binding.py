"""The compiled Cython PageRank (networkit_b200/_cypagerank.pyx over the
declarations in networkit_b200/_nkgpu.pxd): the binding a NetworKit build
carries in place of networkit/centrality.pyx:1989-2037.

CPU: the module is built against include/nkgpu.h and links the same
libnkgpu.so the ctypes layer loads; the reference's argument checks and error
texts. GPU: runs identical, bit for bit, to the Python mirror's, and within
the FP64 bar of the reference's golden scores."""
import importlib
import os

import numpy as np
import pytest

from conftest import GOLDEN_NAMES, ROOT, load_golden
from networkit_b200 import Graph, _capi, centrality


@pytest.fixture(scope="module")
def cy():
    from networkit_b200 import build

    if not os.path.exists(build.cython_target()):
        build.build_cython()
    return importlib.import_module("networkit_b200._cypagerank")


def small_graph():
    G = Graph(5, directed=True)
    for u, v in [(0, 1), (1, 2), (2, 0), (3, 2), (4, 3)]:
        G.addEdge(u, v)
    return G


def test_module_links_the_ctypes_library(cy):
    _capi.lib()
    maps = [line.split()[-1] for line in open("/proc/self/maps") if "libnkgpu.so" in line]
    assert len(set(maps)) == 1
    assert os.path.samefile(maps[0], os.path.join(ROOT, "networkit_b200", "_lib", "libnkgpu.so"))


def test_defaults_and_property_checks(cy):
    pr = cy.PageRank(small_graph())
    assert pr.norm == centrality.Norm.l2norm                # PageRank.hpp:67
    assert pr.maxIterations == _capi.UINT64_MAX             # PageRank.hpp:64
    assert not pr.hasFinished()
    pr.norm = centrality.Norm.l1norm
    assert pr.norm == 0
    with pytest.raises(Exception, match="Max iterations cannot be a negative number."):
        pr.maxIterations = -1
    pr.maxIterations = 7
    assert pr.maxIterations == 7
    with pytest.raises(ValueError):
        pr.norm = 3
    with pytest.raises(TypeError):
        cy.PageRank([[0, 1]])


def test_results_before_run_raise(cy):
    pr = cy.PageRank(small_graph())
    for call in (pr.scores, pr.ranking, pr.maximum, pr.numberOfIterations, pr.centralization,
                 lambda: pr.score(0)):
        with pytest.raises(RuntimeError, match="Error, run must be called first"):
            call()


def test_empty_graph_needs_no_device(cy):
    pr = cy.PageRank(Graph(0)).run()
    assert pr.hasFinished() and pr.scores() == [] and pr.ranking() == []


def test_library_error_text_reaches_python_without_device(cy):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(RuntimeError) as e:
        cy.PageRank(small_graph()).run()
    assert "cuda" in str(e.value).lower()


@pytest.mark.gpu
@pytest.mark.parametrize("name", GOLDEN_NAMES)
@pytest.mark.parametrize("norm", [0, 1])
@pytest.mark.parametrize("normalized", [False, True])
def test_cython_run_equals_python_mirror(cy, name, norm, normalized):
    csr, ref = load_golden(name)
    G = Graph.fromInCSR(csr)
    a = cy.PageRank(G, 0.85, 1e-8, normalized)
    a.norm = norm
    a.run()
    b = centrality.PageRank(G, 0.85, 1e-8, normalized)
    b.norm = norm
    b.run()
    np.testing.assert_array_equal(a.scoresArray(), b.scoresArray())
    assert a.numberOfIterations() == b.numberOfIterations()
    assert a.maximum() == b.maximum()
    assert a.ranking() == b.ranking()
    assert a.centralization() == b.centralization()
    key = f"n{norm}_z{int(normalized)}"
    ref_s = ref[key + "_scores"]
    scale = 1.0 if not normalized else float(np.abs(ref_s).sum())
    assert np.abs(a.scoresArray() - ref_s).sum() <= 1e-10 * scale
    assert abs(a.numberOfIterations() - int(ref[key + "_iterations"])) <= 1


@pytest.mark.gpu
def test_cython_golden_top_node_and_reruns(cy):
    csr, ref = load_golden("wikivote_directed")
    G = Graph.fromInCSR(csr)
    pr = cy.PageRank(G)
    assert pr.run() is pr
    top = pr.ranking()[0]
    assert top[0] == 326 and abs(top[1] - 0.00460) <= 1e-3   # CentralityGTest.cpp:496-500
    first = pr.scoresArray().copy()
    pr.maxIterations = 2
    pr.run()
    assert pr.numberOfIterations() == 2
    pr.maxIterations = _capi.UINT64_MAX
    np.testing.assert_array_equal(pr.run().scoresArray(), first)
    assert pr.lastStats["fp64_sweeps"] == pr.numberOfIterations()


@pytest.mark.gpu
def test_cython_distribute_sinks_and_weights(cy):
    csr, _ = load_golden("matlab8")
    G = Graph.fromInCSR(csr)
    for distribute in (False, True):
        a = cy.PageRank(G, 0.85, 1e-12, False, distribute).run()
        b = centrality.PageRank(G, 0.85, 1e-12, False, distribute).run()
        np.testing.assert_array_equal(a.scoresArray(), b.scoresArray())
