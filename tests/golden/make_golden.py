"""Generate the golden fixtures of the PageRank path from the reference itself.

Run from the repository root, where the reference sources are available:

    python tests/golden/make_golden.py [--ref /path/to/networkit]  (default $NK_REFERENCE)

It builds the reference subset (oracle/Makefile -> oracle/_ref/libnkref.so),
reads the reference's own test inputs with the reference's own readers
(SNAP: input/wiki-Vote.txt, METIS: input/celegans_metabolic.graph, GML:
input/looptest1.gml, input/looptest2.gml), builds the 8-node weighted graph of
CentralityGTest.cpp:582-607, runs NetworKit::PageRank on one OpenMP thread for
every (norm, normalized) combination (plus EigenvectorCentrality and
KatzCentrality in both edge directions) and stores, per graph, the in- and
out-adjacency in storage order plus the reference results in ``<name>.npz``.
It also writes every graph with the reference's NetworkitBinaryWriter
(``<name>.nkbg``) and stores the adjacency the reference's reader builds from
that file (keys ``nkbg_*``), plus one file per weight encoding of the format
(``nkbg_<case>.nkbg``, ``nkbg_formats.npz``), and the reference's
ApproximatePageRank and PageRankNibble results on the reference's SCD test
graphs (``local_ppr.npz``), and the reference's Erdos-Renyi graph of the
G(1e5, average degree 10) workload with the reference's PageRank on it
(``er_config.npz``), and digests of the reference's Barabasi-Albert graph of
the batched-PPR workload (``ba_config.npz``) and of the reference's random
hyperbolic graphs (``rhg_config.npz``). The GPU box has no
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
    ap.add_argument("--ref", default=os.environ.get("NK_REFERENCE")
                    or os.path.join(os.path.dirname(ROOT), "reference"),
                    help="the reference checkout (default: $NK_REFERENCE, else `reference` "
                         "beside this repository)")
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
        # NetworkitBinaryGraph round trip: the reference writer (4 node chunks)
        # and the adjacency the reference reader stores for that file.
        nkbg = os.path.join(HERE, f"{name}.nkbg")
        g.write_nkbg(nkbg, chunks=4)
        back = export_to_arrays(O.RefGraph.read_nkbg(nkbg))
        res.update({"nkbg_" + k: back[k] for k in NKBG_KEYS})
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays, **res)
    nkbg_formats(O)
    local_ppr(O, inp)
    er_config(O)
    ba_config(O)
    rhg_config(O)


# (alpha, epsilon, seeds) of the local PageRank fixtures. SelectiveCDGTest.cpp
# runs ApproximatePageRank(G, 0.4) from seed 0 on wiki-Vote (epsilon default
# 1e-12) and PageRankNibble(G, 0.1, 1e-5) from seed 50 on hep-th.
LOCAL_CASES = [(0.4, 1e-12, [0]), (0.1, 1e-5, [50]), (0.1, 1e-7, [3, 17, 50]),
               (0.05, 1e-6, [100]), (0.2, 1e-4, [1, 2, 5, 8, 13, 21])]


def local_ppr(O, inp):
    """ApproximatePageRank and PageRankNibble fixtures (``local_ppr.npz``):
    per graph its neighbour CSR in forNeighborsOf order (``<g>_ptr``,
    ``<g>_col``, ``<g>_w``, ``<g>_directed``, ``<g>_m``, ``<g>_n``) and per
    case the reference's result: ``<g>_<c>_apr_nodes`` / ``_apr_values``
    (ascending ids), ``<g>_<c>_joint`` (expandOneCommunity(seeds)) and
    ``<g>_<c>_each_<seed>`` (run(seeds), one community per seed; undirected
    graphs only)."""
    import json
    graphs = [
        ("hepth", O.RefGraph.read(os.path.join(inp, "hep-th.graph"), 1)),
        ("wikivote_undirected", O.RefGraph.read(os.path.join(inp, "wiki-Vote.txt"), 0, False)),
        ("wikivote_directed", O.RefGraph.read(os.path.join(inp, "wiki-Vote.txt"), 0, True)),
        ("celegans", O.RefGraph.read(os.path.join(inp, "celegans_metabolic.graph"), 1)),
        ("matlab8", O.RefGraph.from_edges(
            8, [0, 1, 2, 2, 2, 3, 4, 5, 5], [2, 2, 3, 4, 5, 5, 5, 6, 7],
            [3, 2, 3, 2, 1.5, 3, 2, 3, 2], directed=False, weighted=True)),
    ]
    out = {"cases": np.array(json.dumps(LOCAL_CASES)),
           "graphs": np.array(json.dumps([g for g, _ in graphs]))}
    for gname, g in graphs:
        ex = g.export()
        out[f"{gname}_ptr"] = ex["out_ptr"].astype(np.uint64)
        out[f"{gname}_col"] = ex["out_adj"].astype(np.uint32)
        out[f"{gname}_w"] = ex["out_w"].astype(np.float64) if ex["weighted"] else np.zeros(0)
        out[f"{gname}_directed"] = np.bool_(ex["directed"])
        out[f"{gname}_m"] = np.int64(g.m)
        out[f"{gname}_n"] = np.int64(g.n)
        for c, (alpha, eps, seeds) in enumerate(LOCAL_CASES):
            seeds = [s for s in seeds if s < g.z]
            nodes, vals, _ = g.apr(alpha, eps, seeds)
            out[f"{gname}_{c}_apr_nodes"] = nodes
            out[f"{gname}_{c}_apr_values"] = vals
            if ex["directed"]:
                continue
            sets, _ = g.prn(alpha, eps, seeds, joint=True)
            out[f"{gname}_{c}_joint"] = sets[0]
            each, _ = g.prn(alpha, eps, seeds)
            for sd, st in zip(sorted(seeds), each):
                out[f"{gname}_{c}_each_{sd}"] = st
        print(f"local_ppr {gname}: z={g.z} m={g.m}")
    np.savez_compressed(os.path.join(HERE, "local_ppr.npz"), **out)


NKBG_KEYS = ("in_ptr", "in_col", "in_w", "wdeg", "outdeg", "exists", "directed", "weighted")


def nkbg_formats(O):
    """One small file per weight encoding of the binary format (none,
    unsigned varint, signed varint, double, float), with isolated nodes,
    self-loops, duplicate edges, several chunk counts and ids / weights that
    need every varint length (1..9 bytes). Stored: the files
    (``nkbg_<case>.nkbg``) and the adjacency the reference reader builds from
    each (``nkbg_formats.npz``, keys ``<case>_<field>``).

    No case has deleted nodes: the reference writer lists only existing nodes
    (forNodes) under ids 0..numberOfNodes()-1 (NetworkitBinaryWriter.cpp:128,
    :253-290), so such a graph does not round trip, and the reference reader
    asserts that a node exists before preallocating its lists
    (Graph.cpp:173), so a file with a cleared flag byte stops it."""
    rng = np.random.default_rng(2024)
    out = {}
    cases = [
        # name, nodes, edges, directed, weights type, chunks
        ("unsigned_dir", 3000, 12000, True, 1, 5),
        ("signed_undir", 2500, 9000, False, 2, 3),
        ("double_undir", 1800, 7000, False, 3, 7),
        ("float_dir", 2200, 8000, True, 4, 2),
        ("none_undir", 70000, 6000, False, 0, 9),
        ("none_dir", 500, 3000, True, 0, 1),
    ]
    for name, z, m, directed, wtype, chunks in cases:
        # endpoints below z - 40: the top 40 ids stay isolated
        src = ((z - 40) * rng.random(m) ** 2).astype(np.uint32)
        dst = ((z - 40) * rng.random(m)).astype(np.uint32)
        src[:25] = dst[:25]  # self-loops
        src = np.concatenate([src, src[:30]])  # duplicates
        dst = np.concatenate([dst, dst[:30]])
        w = None
        if wtype == 1:
            w = rng.integers(0, 300, src.shape[0]).astype(np.float64)
            w[:4] = [2.0 ** 20, 2.0 ** 40, 2.0 ** 55, 2.0 ** 60]
        elif wtype == 2:
            w = rng.integers(-200, 200, src.shape[0]).astype(np.float64)
            w[:3] = [-(2.0 ** 50), 2.0 ** 45, -1.0]
        elif wtype == 3:
            w = rng.random(src.shape[0]) * 10 - 2
        elif wtype == 4:
            w = rng.integers(-4000, 4000, src.shape[0]) / 8.0
        g = O.RefGraph.from_edges(z, src, dst, w, directed=directed, weighted=w is not None)
        path = os.path.join(HERE, f"nkbg_{name}.nkbg")
        g.write_nkbg(path, chunks=chunks, weights=wtype)
        back = export_to_arrays(O.RefGraph.read_nkbg(path))
        out.update({f"{name}_{k}": back[k] for k in NKBG_KEYS})
        print(f"nkbg_{name}: z={z} m={src.shape[0]} {os.path.getsize(path)} bytes")
    np.savez_compressed(os.path.join(HERE, "nkbg_formats.npz"), **out)


# The Erdos-Renyi workload: G(n = 100000, average degree 10), undirected,
# edges drawn from seed 42 on 8 OpenMP threads (the reference's graph depends
# on the thread count).
ER_N, ER_P, ER_SEED, ER_THREADS = 100000, 10.0 / 99999.0, 42, 8
ER_SAMPLE = 97  # every 97th score is stored


def er_config(O):
    """The reference's ErdosRenyiGenerator(100000, 10 / 99999) graph, drawn
    on 8 OpenMP threads after setSeed(42, False), and the reference's
    PageRank on it (damp 0.85, tol 1e-8, L2, not normalized; this reference
    has no sink redistribution) in ``er_config.npz``: SHA-256 digests of the
    in-adjacency (row offsets as uint64, ids as uint32), the arc count, the
    iteration count, maximum(), every ER_SAMPLE-th score and the first 100
    ranking ids."""
    import hashlib

    g = O.RefGraph.erdos_renyi(ER_N, ER_P, ER_SEED, directed=False, threads=ER_THREADS)
    a = export_to_arrays(g)
    r = g.pagerank(damp=0.85, tol=1e-8, normalized=False, norm=1, nthreads=1)
    out = dict(
        n=np.int64(ER_N), p=np.float64(ER_P), seed=np.int64(ER_SEED),
        threads=np.int64(ER_THREADS),
        arcs=np.int64(a["in_ptr"][-1]),
        in_ptr_sha256=np.bytes_(hashlib.sha256(a["in_ptr"].tobytes()).hexdigest()),
        in_col_sha256=np.bytes_(hashlib.sha256(a["in_col"].tobytes()).hexdigest()),
        iterations=np.int64(r["iterations"]), maximum=np.float64(r["maximum"]),
        sample_every=np.int64(ER_SAMPLE), scores_sample=r["scores"][::ER_SAMPLE].copy(),
        rank_ids_top100=r["ranking_ids"][:100].astype(np.uint32))
    np.savez_compressed(os.path.join(HERE, "er_config.npz"), **out)
    print(f"er_config: arcs={int(out['arcs'])} it={r['iterations']} max={r['maximum']:.6g}")


# The batched-PPR workload: Barabasi-Albert, n = 4M, k = 8 attachments per
# new node, seed 42.
BA_K, BA_N, BA_SEED = 8, 4_000_000, 42


def ba_config(O):
    """The reference's BarabasiAlbertGenerator(8, 4000000) graph after
    setSeed(42, False), as SHA-256 digests of its in-adjacency (row offsets as
    uint64, ids as uint32) and its arc count, in ``ba_config.npz``."""
    import hashlib

    a = export_to_arrays(O.RefGraph.barabasi_albert(BA_K, BA_N, BA_SEED))
    out = dict(k=np.int64(BA_K), n=np.int64(BA_N), seed=np.int64(BA_SEED),
               arcs=np.int64(a["in_ptr"][-1]),
               in_ptr_sha256=np.bytes_(hashlib.sha256(a["in_ptr"].tobytes()).hexdigest()),
               in_col_sha256=np.bytes_(hashlib.sha256(a["in_col"].tobytes()).hexdigest()))
    np.savez_compressed(os.path.join(HERE, "ba_config.npz"), **out)
    print(f"ba_config: arcs={int(out['arcs'])}")


# Random hyperbolic graphs (average degree 16, exponent 3): a small one, the
# largest size of the many-graph batch, and the 4M graph of the locality
# workload.
RHG_CASES = [(1000, 42), (200_000, 42), (4_000_000, 21)]


def rhg_config(O):
    """The reference's HyperbolicGenerator(n, 16, 3) graphs of RHG_CASES,
    drawn on one OpenMP thread after setSeed(seed, False), as SHA-256
    digests of their in-adjacency and their arc counts (``rhg_config.npz``,
    keys ``<n>_<seed>_<field>``)."""
    import hashlib

    out = {}
    for n, seed in RHG_CASES:
        a = export_to_arrays(O.RefGraph.hyperbolic(n, 16.0, 3.0, seed, threads=1))
        key = f"{n}_{seed}_"
        out[key + "arcs"] = np.int64(a["in_ptr"][-1])
        out[key + "in_ptr_sha256"] = np.bytes_(hashlib.sha256(a["in_ptr"].tobytes()).hexdigest())
        out[key + "in_col_sha256"] = np.bytes_(hashlib.sha256(a["in_col"].tobytes()).hexdigest())
        print(f"rhg_config: n={n} seed={seed} arcs={int(out[key + 'arcs'])}")
    np.savez_compressed(os.path.join(HERE, "rhg_config.npz"), **out)


if __name__ == "__main__":
    main()
