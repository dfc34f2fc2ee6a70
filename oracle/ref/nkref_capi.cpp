// Test infrastructure only (the oracle): a small extern "C" driver around the
// reference's own PageRank, compiled together with the reference sources by
// oracle/Makefile into oracle/_ref/libnkref.so. Nothing in the product path
// links or loads this library; only the tests, the smoke check and the CPU
// baseline of bench.py do.
//
// It builds a NetworKit::Graph through Graph::addEdge in the caller's edge
// order (the in-edge order of each node is insertion order, Graph.cpp:549-596),
// runs NetworKit::PageRank::run() (PageRank.cpp:20-104) and hands back scores,
// the iteration count, maximum() and ranking() (Centrality.cpp:29-41).
// The SNAP, METIS and GML readers are exported so that fixtures can be
// produced with exactly the reference's node numbering and edge order.

#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <algorithm>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include <omp.h>

#include <networkit/centrality/EigenvectorCentrality.hpp>
#include <networkit/centrality/KatzCentrality.hpp>
#include <networkit/centrality/PageRank.hpp>
#include <networkit/auxiliary/Random.hpp>
#include <networkit/generators/BarabasiAlbertGenerator.hpp>
#include <networkit/generators/ErdosRenyiGenerator.hpp>
#include <networkit/generators/HyperbolicGenerator.hpp>
#include <networkit/graph/Graph.hpp>
#include <networkit/io/GMLGraphReader.hpp>
#include <networkit/io/NetworkitBinaryReader.hpp>
#include <networkit/io/NetworkitBinaryWriter.hpp>
#include <networkit/io/METISGraphReader.hpp>
#include <networkit/io/SNAPGraphReader.hpp>
#include <networkit/scd/ApproximatePageRank.hpp>
#include <networkit/scd/PageRankNibble.hpp>

namespace {
thread_local std::string g_err;

struct RefGraph {
    std::unique_ptr<NetworKit::Graph> G;
};

int fail(const std::exception &e) {
    g_err = e.what();
    return -1;
}
} // namespace

extern "C" {

const char *nkref_last_error(void) { return g_err.c_str(); }

// Build a graph from an ordered edge list. exists (nullable, length n) marks
// nodes to delete after insertion (deleted nodes must have no edges).
int nkref_graph_create(void **out, uint64_t n, int weighted, int directed, uint64_t m,
                       const uint32_t *src, const uint32_t *dst, const double *w,
                       const uint8_t *exists) {
    try {
        auto *h = new RefGraph();
        h->G.reset(new NetworKit::Graph(n, weighted != 0, directed != 0));
        for (uint64_t e = 0; e < m; ++e) {
            h->G->addEdge(src[e], dst[e], w ? w[e] : NetworKit::defaultEdgeWeight);
        }
        if (exists) {
            for (uint64_t v = 0; v < n; ++v)
                if (!exists[v])
                    h->G->removeNode(v);
        }
        *out = h;
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// NetworKit::ErdosRenyiGenerator(n, p, directed).generate() run with
// `threads` OpenMP threads after Aux::Random::setSeed(seed, false); the
// previous thread count is restored afterwards.
int nkref_erdos_renyi(void **out, uint64_t n, double p, uint64_t seed, int directed,
                      int threads) {
    const int prev = omp_get_max_threads();
    try {
        Aux::Random::setSeed(seed, false);
        omp_set_num_threads(threads);
        auto *rg = new RefGraph;
        rg->G.reset(new NetworKit::Graph(
            NetworKit::ErdosRenyiGenerator(n, p, directed != 0).generate()));
        omp_set_num_threads(prev);
        *out = rg;
        return 0;
    } catch (const std::exception &e) {
        omp_set_num_threads(prev);
        return fail(e);
    }
}

// NetworKit::BarabasiAlbertGenerator(k, n, n0).generate() (Batagelj-Brandes,
// sequential) after Aux::Random::setSeed(seed, false).
int nkref_barabasi_albert(void **out, uint64_t k, uint64_t n, uint64_t n0, uint64_t seed) {
    try {
        Aux::Random::setSeed(seed, false);
        auto *rg = new RefGraph;
        rg->G.reset(new NetworKit::Graph(NetworKit::BarabasiAlbertGenerator(k, n, n0).generate()));
        *out = rg;
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// NetworKit::HyperbolicGenerator(n, avg_deg, exponent).generate() run with
// `threads` OpenMP threads after Aux::Random::setSeed(seed, false).
int nkref_hyperbolic(void **out, uint64_t n, double avg_deg, double exponent, uint64_t seed,
                     int threads) {
    const int prev = omp_get_max_threads();
    try {
        Aux::Random::setSeed(seed, false);
        omp_set_num_threads(threads);
        auto *rg = new RefGraph;
        rg->G.reset(new NetworKit::Graph(
            NetworKit::HyperbolicGenerator(n, avg_deg, exponent).generate()));
        omp_set_num_threads(prev);
        *out = rg;
        return 0;
    } catch (const std::exception &e) {
        omp_set_num_threads(prev);
        return fail(e);
    }
}

void nkref_graph_destroy(void *g) { delete static_cast<RefGraph *>(g); }

uint64_t nkref_graph_num_nodes(void *g) { return static_cast<RefGraph *>(g)->G->numberOfNodes(); }
uint64_t nkref_graph_upper_node_id(void *g) {
    return static_cast<RefGraph *>(g)->G->upperNodeIdBound();
}
uint64_t nkref_graph_num_edges(void *g) { return static_cast<RefGraph *>(g)->G->numberOfEdges(); }

// Run the reference PageRank. norm: 0 = L1Norm, 1 = L2Norm (PageRank.hpp:31).
// scores_out has upperNodeIdBound() entries; ranking_* (nullable) have
// numberOfNodes() entries. nthreads <= 0 keeps the OpenMP default.
int nkref_pagerank(void *g, double damp, double tol, int normalized, int norm,
                   uint64_t max_iterations, int nthreads, double *scores_out,
                   uint64_t *iterations_out, double *max_out, uint64_t *ranking_ids_out,
                   double *ranking_vals_out, double *run_seconds_out) {
    try {
        if (nthreads > 0)
            omp_set_num_threads(nthreads);
        auto &G = *static_cast<RefGraph *>(g)->G;
        NetworKit::PageRank pr(G, damp, tol, normalized != 0);
        pr.norm = norm == 0 ? NetworKit::PageRank::L1Norm : NetworKit::PageRank::L2Norm;
        pr.maxIterations = max_iterations;
        auto t0 = std::chrono::steady_clock::now();
        pr.run();
        auto t1 = std::chrono::steady_clock::now();
        if (run_seconds_out)
            *run_seconds_out = std::chrono::duration<double>(t1 - t0).count();
        const auto &s = pr.scores();
        std::memcpy(scores_out, s.data(), s.size() * sizeof(double));
        if (iterations_out)
            *iterations_out = pr.numberOfIterations();
        if (max_out)
            *max_out = pr.maximum();
        if (ranking_ids_out || ranking_vals_out) {
            auto r = pr.ranking();
            for (size_t i = 0; i < r.size(); ++i) {
                if (ranking_ids_out)
                    ranking_ids_out[i] = r[i].first;
                if (ranking_vals_out)
                    ranking_vals_out[i] = r[i].second;
            }
        }
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Run the reference EigenvectorCentrality (EigenvectorCentrality.cpp:20-60);
// scores_out has upperNodeIdBound() entries.
int nkref_eigenvector(void *g, double tol, int nthreads, double *scores_out,
                      double *run_seconds_out) {
    try {
        if (nthreads > 0)
            omp_set_num_threads(nthreads);
        auto &G = *static_cast<RefGraph *>(g)->G;
        NetworKit::EigenvectorCentrality ec(G, tol);
        auto t0 = std::chrono::steady_clock::now();
        ec.run();
        auto t1 = std::chrono::steady_clock::now();
        if (run_seconds_out)
            *run_seconds_out = std::chrono::duration<double>(t1 - t0).count();
        const auto &sc = ec.scores();
        std::memcpy(scores_out, sc.data(), sc.size() * sizeof(double));
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Run the reference KatzCentrality (KatzCentrality.cpp:20-72); out_edges
// selects EdgeDirection::OutEdges. ranking_ids_out (nullable) gets ranking().
int nkref_katz(void *g, double alpha, double beta, double tol, int out_edges, int nthreads,
               double *scores_out, uint64_t *ranking_ids_out, double *run_seconds_out) {
    try {
        if (nthreads > 0)
            omp_set_num_threads(nthreads);
        auto &G = *static_cast<RefGraph *>(g)->G;
        NetworKit::KatzCentrality kc(G, alpha, beta, tol);
        kc.edgeDirection = out_edges ? NetworKit::EdgeDirection::OutEdges
                                     : NetworKit::EdgeDirection::InEdges;
        auto t0 = std::chrono::steady_clock::now();
        kc.run();
        auto t1 = std::chrono::steady_clock::now();
        if (run_seconds_out)
            *run_seconds_out = std::chrono::duration<double>(t1 - t0).count();
        const auto &sc = kc.scores();
        std::memcpy(scores_out, sc.data(), sc.size() * sizeof(double));
        if (ranking_ids_out) {
            auto r = kc.ranking();
            for (size_t i = 0; i < r.size(); ++i)
                ranking_ids_out[i] = r[i].first;
        }
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// ApproximatePageRank(G, alpha, eps).run(seeds) (ApproximatePageRank.cpp:18-55):
// the support (every node the result holds) ascending by id with its value.
// *count = support size; nothing is written when it exceeds cap.
int nkref_apr(void *g, double alpha, double eps, const uint32_t *seeds, uint64_t nseeds,
              uint64_t cap, uint32_t *nodes, double *values, uint64_t *count,
              double *run_seconds_out) {
    try {
        auto &G = *static_cast<RefGraph *>(g)->G;
        std::set<NetworKit::node> s(seeds, seeds + nseeds);
        NetworKit::ApproximatePageRank apr(G, alpha, eps);
        auto t0 = std::chrono::steady_clock::now();
        auto pr = apr.run(s);
        auto t1 = std::chrono::steady_clock::now();
        if (run_seconds_out)
            *run_seconds_out = std::chrono::duration<double>(t1 - t0).count();
        std::sort(pr.begin(), pr.end());
        *count = pr.size();
        if (pr.size() <= cap)
            for (size_t i = 0; i < pr.size(); ++i) {
                nodes[i] = static_cast<uint32_t>(pr[i].first);
                values[i] = pr[i].second;
            }
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// PageRankNibble(G, alpha, eps): one community per seed, as
// SelectiveCommunityDetector::run(seeds) builds them
// (SelectiveCommunityDetector.cpp:15-23, PageRankNibble.cpp:84-89), or one
// community of the whole seed set (expandOneCommunity(seeds)) when `joint`.
// Sets are ascending, concatenated; offsets[k..k+1] delimit set k.
// *total = sum of the set sizes; nothing past cap is written.
int nkref_prn(void *g, double alpha, double eps, const uint32_t *seeds, uint64_t nseeds,
              int joint, uint64_t cap, uint64_t *offsets, uint32_t *sets, uint64_t *total,
              double *run_seconds_out) {
    try {
        auto &G = *static_cast<RefGraph *>(g)->G;
        std::set<NetworKit::node> s(seeds, seeds + nseeds);
        NetworKit::PageRankNibble prn(G, alpha, eps);
        std::vector<std::set<NetworKit::node>> out;
        auto t0 = std::chrono::steady_clock::now();
        if (joint) {
            out.push_back(prn.expandOneCommunity(s));
        } else {
            auto res = prn.run(s);
            for (NetworKit::node x : s)
                out.push_back(res[x]);
        }
        auto t1 = std::chrono::steady_clock::now();
        if (run_seconds_out)
            *run_seconds_out = std::chrono::duration<double>(t1 - t0).count();
        uint64_t pos = 0;
        offsets[0] = 0;
        for (size_t k = 0; k < out.size(); ++k) {
            for (NetworKit::node x : out[k]) {
                if (pos < cap)
                    sets[pos] = static_cast<uint32_t>(x);
                ++pos;
            }
            offsets[k + 1] = pos;
        }
        *total = pos;
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Write the graph in the NetworkitBinaryGraph format (NetworkitBinaryWriter,
// `chunks` node chunks; `weights` = the NetworkitBinaryWeights value: 0 none,
// 1 unsigned varint, 2 signed varint, 3 double, 4 float, 5 auto-detect).
int nkref_write_nkbg(void *g, const char *path, uint64_t chunks, int weights) {
    try {
        if (weights < 0 || weights > 5)
            throw std::runtime_error("weights must be in 0..5");
        NetworKit::NetworkitBinaryWriter w(chunks,
                                           static_cast<NetworKit::NetworkitBinaryWeights>(weights));
        w.write(*static_cast<RefGraph *>(g)->G, path);
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Read a NetworkitBinaryGraph file with the reference's reader.
int nkref_read_nkbg(void **out, const char *path) {
    try {
        NetworKit::NetworkitBinaryReader r;
        auto *rg = new RefGraph();
        rg->G.reset(new NetworKit::Graph(r.read(path)));
        *out = rg;
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

// Read a file with the reference's SNAP (kind 0), METIS (kind 1) or GML
// (kind 2) reader into a graph handle.
int nkref_graph_read(void **out, const char *path, int kind, int directed) {
    try {
        auto *h = new RefGraph();
        h->G.reset(new NetworKit::Graph(
            kind == 0   ? NetworKit::SNAPGraphReader(directed != 0).read(path)
            : kind == 1 ? NetworKit::METISGraphReader().read(path)
                        : NetworKit::GMLGraphReader().read(path)));
        *out = h;
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int nkref_graph_is_directed(void *g) { return static_cast<RefGraph *>(g)->G->isDirected(); }
int nkref_graph_is_weighted(void *g) { return static_cast<RefGraph *>(g)->G->isWeighted(); }

// Number of stored out-arcs (undirected: both directions, self-loops once) and
// in-arcs (directed only; 0 otherwise).
void nkref_graph_arc_counts(void *g, uint64_t *out_arcs, uint64_t *in_arcs) {
    auto &G = *static_cast<RefGraph *>(g)->G;
    uint64_t o = 0, i = 0;
    for (uint64_t u = 0; u < G.upperNodeIdBound(); ++u) {
        o += G.degreeOut(u);
        if (G.isDirected())
            i += G.degreeIn(u);
    }
    *out_arcs = o;
    *in_arcs = i;
}

// Export the adjacency in storage order: per node u its out-list outEdges[u]
// (with weights when out_w is non-null) and, for directed graphs, its in-list
// inEdges[u] (with weights when in_w is non-null). exists_out (nullable) gets
// the node-existence mask. Buffers are sized with nkref_graph_arc_counts.
int nkref_graph_export(void *g, uint64_t *out_ptr, uint32_t *out_adj, double *out_w,
                       uint64_t *in_ptr, uint32_t *in_adj, double *in_w, uint8_t *exists_out) {
    try {
        auto &G = *static_cast<RefGraph *>(g)->G;
        const uint64_t z = G.upperNodeIdBound();
        uint64_t o = 0, i = 0;
        out_ptr[0] = 0;
        if (in_ptr)
            in_ptr[0] = 0;
        for (uint64_t u = 0; u < z; ++u) {
            if (exists_out)
                exists_out[u] = G.hasNode(u) ? 1 : 0;
            G.forNeighborsOf(u, [&](NetworKit::node v, NetworKit::edgeweight ew) {
                out_adj[o] = static_cast<uint32_t>(v);
                if (out_w)
                    out_w[o] = ew;
                ++o;
            });
            out_ptr[u + 1] = o;
            if (G.isDirected() && in_ptr) {
                G.forInNeighborsOf(u, [&](NetworKit::node v, NetworKit::edgeweight ew) {
                    in_adj[i] = static_cast<uint32_t>(v);
                    if (in_w)
                        in_w[i] = ew;
                    ++i;
                });
                in_ptr[u + 1] = i;
            }
        }
        return 0;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

} // extern "C"
