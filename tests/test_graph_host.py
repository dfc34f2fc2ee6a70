"""Host-side logic on the CPU: the in-CSR the boundary consumes, the Python
mirror of the reference API, the generators, and the C-ABI library loading
(no device call)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden
from networkit_b200 import Graph, centrality, generators, in_csr_from_edges


def test_incsr_directed_insertion_order():
    # in-lists keep insertion order (Graph.cpp:563-573)
    csr = in_csr_from_edges(4, [3, 1, 2, 0, 1], [0, 0, 0, 1, 3], directed=True)
    assert csr.in_ptr.tolist() == [0, 3, 4, 4, 5]
    assert csr.in_col.tolist() == [3, 1, 2, 0, 1]
    assert csr.outdeg.tolist() == [1, 2, 1, 1]


def test_incsr_undirected_selfloop_once():
    # undirected: both directions stored, self-loop once (Graph.cpp:577-592)
    csr = in_csr_from_edges(3, [0, 1, 2], [1, 1, 0], [2.0, 5.0, 3.0], directed=False)
    assert csr.in_ptr.tolist() == [0, 2, 4, 5]
    assert csr.in_col.tolist() == [1, 2, 0, 1, 0]
    assert csr.in_w.tolist() == [2.0, 3.0, 2.0, 5.0, 3.0]
    assert csr.outdeg.tolist() == [2, 2, 1]
    assert csr.wdeg.tolist() == [5.0, 7.0, 3.0]


def test_graph_builds_same_csr_as_reference_export():
    """Replaying the 8-node test graph through Graph.addEdge gives exactly the
    adjacency the reference stores."""
    csr_ref, _ = load_golden("matlab8")
    G = Graph(8, weighted=True)
    for u, v, w in [(0, 2, 3), (1, 2, 2), (2, 3, 3), (2, 4, 2), (2, 5, 1.5), (3, 5, 3), (4, 5, 2),
                    (5, 6, 3), (5, 7, 2)]:
        G.addEdge(u, v, w)
    c = G.inCSR()
    np.testing.assert_array_equal(c.in_ptr, csr_ref.in_ptr)
    np.testing.assert_array_equal(c.in_col, csr_ref.in_col)
    np.testing.assert_array_equal(c.in_w, csr_ref.in_w)
    np.testing.assert_array_equal(c.wdeg, csr_ref.wdeg)
    assert G.numberOfEdges() == 9 and G.numberOfNodes() == 8


def test_graph_api_errors():
    G = Graph(3)
    with pytest.raises(RuntimeError):
        G.addEdge(0, 3)
    G.removeNode(2)
    assert G.numberOfNodes() == 2 and G.upperNodeIdBound() == 3
    with pytest.raises(RuntimeError):
        G.addEdge(2, 0)
    with pytest.raises(ValueError):
        Graph(-1)


def test_pagerank_api_surface_without_gpu():
    """Constructor, properties and error behaviour of centrality.pyx:1989-2037
    (nothing here launches a kernel)."""
    G = Graph(3)
    G.addEdge(0, 1)
    pr = centrality.PageRank(G, 0.85, 1e-8)
    assert pr.norm == centrality.Norm.l2norm
    assert pr.maxIterations == 2**64 - 1
    pr.norm = centrality.Norm.l1norm
    assert pr.norm == 0
    pr.maxIterations = 2
    assert pr.maxIterations == 2
    with pytest.raises(Exception, match="Max iterations cannot be a negative number."):
        pr.maxIterations = -1
    assert not pr.hasFinished()
    for f in (pr.scores, pr.ranking, pr.numberOfIterations, pr.maximum):
        with pytest.raises(RuntimeError, match="Error, run must be called first"):
            f()
    with pytest.raises(RuntimeError):
        centrality.Centrality()
    with pytest.raises(ValueError):
        centrality.PageRank(G, precision="fp16")
    assert centrality.rankPerNode([(2, 0.5), (0, 0.3), (1, 0.3)]) == [1, 1, 0]


def test_generators_deterministic_and_shaped():
    a = generators.rmat_directed(10, 8, seed=1, nthreads=1)
    b = generators.rmat_directed(10, 8, seed=1, nthreads=4)
    np.testing.assert_array_equal(a.in_ptr, b.in_ptr)
    np.testing.assert_array_equal(a.in_col, b.in_col)
    rows = np.repeat(np.arange(a.z), np.diff(a.in_ptr).astype(np.int64))
    assert not np.any(rows == a.in_col)  # no self-loops
    key = rows.astype(np.int64) * a.z + a.in_col
    assert np.all(np.diff(key) > 0)  # sorted, no duplicates
    assert a.outdeg.sum() == a.arcs
    er = generators.erdos_renyi(2000, 0.01, seed=42)
    assert er.in_ptr[-1] == er.arcs and er.arcs % 2 == 0
    assert abs(er.arcs / 2 - 0.01 * 2000 * 1999 / 2) < 5 * np.sqrt(0.01 * 2000 * 1999 / 2)
    ba = generators.barabasi_albert(4, 3000, seed=42)
    assert ba.arcs == 2 * (4 + (3000 - 4) * 4)  # distinct neighbours: no duplicates


def _header_symbols():
    src = open(os.path.join(ROOT, "include", "nkgpu.h")).read()
    return sorted(set(re.findall(r"NKG_API\s+[\w\s\*]+?\b(nkg_\w+)\s*\(", src)))


def test_capi_library_exports_every_header_symbol():
    """The built C-ABI library loads here (no GPU needed to dlopen it) and
    exports every entry point include/nkgpu.h declares."""
    from networkit_b200 import _capi
    if not os.path.exists(_capi.LIB_PATH):
        from networkit_b200 import build
        build.build_gpu()
    lib = ctypes.CDLL(_capi.LIB_PATH)
    syms = _header_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) <= set(_capi.SIGNATURES), "every header symbol has a ctypes signature"
    L = _capi.lib()
    assert L.nkg_abi_version() == _capi.ABI_VERSION


def test_capi_structures_match_the_header(tmp_path):
    """The ctypes structures have the size and field offsets of the C
    structures of include/nkgpu.h (compiled here with gcc)."""
    import ctypes as C
    import shutil
    import subprocess

    from networkit_b200 import _capi
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    checks = {"nkg_stats": (_capi.Stats, ["iterations", "bytes_per_sweep_fp32", "residual_trace",
                                         "trace_capacity", "trace_length"]),
              "nkg_graph_options": (_capi.GraphOptions, ["row_order", "hot_tier_kb"]),
              "nkg_pr_params": (_capi.PRParams, ["precision", "max_iterations"]),
              "nkg_graph_info": (_capi.GraphInfo, ["row_order", "ms_create"])}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "nkgpu.h"', 'int main(void) {']
    for name, (_, fields) in checks.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for f in fields:
            lines.append(f'printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "sizes.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "sizes"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                 text=True).stdout.splitlines())
    for name, (cls, fields) in checks.items():
        assert int(got[name]) == C.sizeof(cls), name
        for f in fields:
            assert int(got[f"{name}.{f}"]) == getattr(cls, f).offset, (name, f)


def test_hyperbolic_generator_shape():
    """Threshold random hyperbolic graphs: symmetric, no self-loops, average
    degree at the target in expectation, independent of the thread count in
    batch form, and the batch equals the graphs generated one by one."""
    degs = [generators.hyperbolic(20000, 16, 3, seed=s).arcs / 20000 for s in range(8)]
    assert abs(np.mean(degs) - 16.0) < 0.6
    c = generators.hyperbolic(5000, 16, 3, seed=9)
    rows = np.repeat(np.arange(c.z, dtype=np.int64), np.diff(c.in_ptr).astype(np.int64))
    assert not np.any(rows == c.in_col)
    fwd = np.sort(rows * c.z + c.in_col)
    bwd = np.sort(c.in_col.astype(np.int64) * c.z + rows)
    np.testing.assert_array_equal(fwd, bwd)
    ns = [300, 2000, 900]
    b1, offs = generators.hyperbolic_batch(ns, 16, 3, seed=42, nthreads=1)
    b4, offs4 = generators.hyperbolic_batch(ns, 16, 3, seed=42, nthreads=4)
    np.testing.assert_array_equal(b1.in_col, b4.in_col)
    np.testing.assert_array_equal(offs, offs4)
    for i, n in enumerate(ns):
        g = generators.hyperbolic(n, 16, 3, seed=42 + i)
        a, b = int(offs[i]), int(offs[i + 1])
        np.testing.assert_array_equal(b1.in_ptr[a:b + 1] - b1.in_ptr[a], g.in_ptr)
        np.testing.assert_array_equal(b1.in_col[b1.in_ptr[a]:b1.in_ptr[b]] - a, g.in_col)


def test_concat_in_csr_block_diagonal():
    from networkit_b200.graph import concat_in_csr
    gs = [generators.rmat_directed(5, 4, seed=s) for s in range(3)]
    csr, offs = concat_in_csr(gs)
    assert csr.z == sum(g.z for g in gs) and csr.arcs == sum(g.arcs for g in gs)
    for i, g in enumerate(gs):
        a, b = int(offs[i]), int(offs[i + 1])
        np.testing.assert_array_equal(csr.in_ptr[a:b + 1] - csr.in_ptr[a], g.in_ptr)
        seg = csr.in_col[csr.in_ptr[a]:csr.in_ptr[b]]
        assert seg.min() >= a and seg.max() < b
