"""Generate the golden fixtures of the PageRank path from the reference itself.

Run from the repository root, where the reference sources are available:

    python tests/golden/make_golden.py [--ref /path/to/networkit]

It builds the reference subset (oracle/Makefile -> oracle/_ref/libnkref.so),
reads the reference's own test inputs with the reference's own readers
(SNAP: input/wiki-Vote.txt, METIS: input/celegans_metabolic.graph, GML:
input/looptest1.gml, input/looptest2.gml), builds the 8-node weighted graph of
CentralityGTest.cpp:582-607, runs NetworKit::PageRank on one OpenMP thread for
every (norm, normalized) combination (plus EigenvectorCentrality and
KatzCentrality in both edge directions) and stores, per graph, the in- and
out-adjacency in storage order plus the reference results in ``<name>.npz``. The GPU box has no
reference checkout: the tests read only these files.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def export_to_arrays(g):
    """In-adjacency CSR of a reference graph, as Graph::forInEdgesOf walks it."""
    ex = g.export()
    z = ex["exists"].shape[0]
    if ex["directed"]:
        ptr, adj, w = ex["in_ptr"], ex["in_adj"], ex["in_w"]
    else:
        ptr, adj, w = ex["out_ptr"], ex["out_adj"], ex["out_w"]
    outdeg = np.diff(ex["out_ptr"]).astype(np.uint32)
    rows = np.repeat(np.arange(z), np.diff(ex["out_ptr"]).astype(np.int64))
    # weightedDegree(u): out-weights summed in storage order (Graph.cpp:426-452)
    wdeg = np.zeros(z)
    for i in range(rows.shape[0]):
        wdeg[rows[i]] += ex["out_w"][i]
    if not ex["weighted"]:
        wdeg = outdeg.astype(np.float64)
    return dict(z=np.int64(z), in_ptr=ptr.astype(np.uint64), in_col=adj.astype(np.uint32),
                in_w=(w.astype(np.float64) if ex["weighted"] else np.zeros(0)),
                weighted=np.bool_(ex["weighted"]), wdeg=wdeg, outdeg=outdeg,
                exists=ex["exists"].astype(np.uint8), directed=np.bool_(ex["directed"]),
                out_ptr=ex["out_ptr"].astype(np.uint64), out_col=ex["out_adj"].astype(np.uint32),
                out_w=(ex["out_w"].astype(np.float64) if ex["weighted"] else np.zeros(0)))


def run_all(g, arrays, tag, damp=0.85, tol=1e-8):
    out = {}
    for norm in (0, 1):
        for normalized in (False, True):
            r = g.pagerank(damp=damp, tol=tol, normalized=normalized, norm=norm, nthreads=1)
            key = f"n{norm}_z{int(normalized)}"
            out[key + "_scores"] = r["scores"]
            out[key + "_iterations"] = np.int64(r["iterations"])
            out[key + "_maximum"] = np.float64(r["maximum"])
            out[key + "_rank_ids"] = r["ranking_ids"].astype(np.uint32)
            # maxIterations = 2 (CentralityGTest.cpp:503-506)
            r2 = g.pagerank(damp=damp, tol=tol, normalized=normalized, norm=norm,
                            max_iterations=2, nthreads=1)
            if key == "n1_z0":
                out[key + "_max2_scores"] = r2["scores"]
            out[key + "_max2_iterations"] = np.int64(r2["iterations"])
            print(f"  {tag} norm={norm} normalized={normalized}: it={r['iterations']} "
                  f"top={r['ranking_ids'][0]} {r['ranking_vals'][0]:.6g}")
    # EigenvectorCentrality (tol 1e-9, centrality.pyx:1966) and KatzCentrality
    # (alpha 0 = default, beta 0.1, tol 1e-8, centrality.pyx:1700) in both edge
    # directions, and Katz with alpha 5e-4 (CentralityGTest.cpp:216-225).
    out["ec_scores"] = g.eigenvector(tol=1e-9, nthreads=1)
    out["katz_in_scores"], ids = g.katz(0.0, 0.1, 1e-8, False, nthreads=1)
    out["katz_in_rank_ids"] = ids.astype(np.uint32)
    out["katz_out_scores"], _ = g.katz(0.0, 0.1, 1e-8, True, nthreads=1)
    out["katz5e4_scores"], ids = g.katz(5e-4, 0.1, 1e-8, False, nthreads=1)
    out["katz5e4_rank_ids"] = ids.astype(np.uint32)
    print(f"  {tag} katz(5e-4) top={ids[0]}")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={args.ref}", "all"],
                   check=True)
    import oracle as O

    inp = os.path.join(args.ref, "input")
    cases = [
        ("wikivote_directed", lambda: O.RefGraph.read(os.path.join(inp, "wiki-Vote.txt"), 0, True)),
        ("wikivote_undirected",
         lambda: O.RefGraph.read(os.path.join(inp, "wiki-Vote.txt"), 0, False)),
        ("celegans", lambda: O.RefGraph.read(os.path.join(inp, "celegans_metabolic.graph"), 1)),
        ("looptest1", lambda: O.RefGraph.read(os.path.join(inp, "looptest1.gml"), 2)),
        ("looptest2", lambda: O.RefGraph.read(os.path.join(inp, "looptest2.gml"), 2)),
        # CentralityGTest.cpp:582-607: 8 nodes, weighted, undirected
        ("matlab8", lambda: O.RefGraph.from_edges(
            8, [0, 1, 2, 2, 2, 3, 4, 5, 5], [2, 2, 3, 4, 5, 5, 5, 6, 7],
            [3, 2, 3, 2, 1.5, 3, 2, 3, 2], directed=False, weighted=True)),
    ]
    for name, make in cases:
        g = make()
        arrays = export_to_arrays(g)
        print(f"{name}: z={g.z} n={g.n} m={g.m} directed={g.directed} weighted={g.weighted}")
        res = run_all(g, arrays, name)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays, **res)


if __name__ == "__main__":
    main()
