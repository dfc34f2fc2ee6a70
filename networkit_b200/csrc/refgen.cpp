// Generators that draw the reference generators' own graphs: the same random
// stream, the same arithmetic, the same adjacency order as the NetworKit Graph
// they build, for the workloads that name a NetworKit generator and a seed.
// Each restates one reference generator run on one OpenMP thread after
// Aux::Random::setSeed(seed, false), whose random source is then one
// std::mt19937_64 seeded with `seed` (Random.cpp: getURNG / getSeed_), with
// the standard library's distributions on it.
//
// This file is compiled without floating-point contraction and for the
// baseline x86-64 instruction set, as the reference is, so that every
// product and sum rounds as it does there (a fused multiply-add would change
// which point pairs pass a distance test).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <limits>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "nkgen.hpp"

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

// In-CSR of an undirected graph (or the in-lists of a directed one) that
// GraphBuilder::toGraph(true, ...) on one thread makes from half edges
// own[u] = (u, v...) (GraphBuilder.cpp:192-362): row u holds own[u] in order
// (undirected), then every v with u in own[v], v ascending. outdeg: the
// number of out-arcs (directed: |own[u]|; undirected: the row length).
void half_edges_to_csr(const std::vector<std::vector<uint32_t>> &own, bool directed,
                       nkgen_csr *out) {
    const uint64_t n = own.size();
    std::vector<uint64_t> deg(n, 0);
    for (uint64_t v = 0; v < n; ++v) {
        if (!directed)
            deg[v] += own[v].size();
        for (uint32_t u : own[v])
            ++deg[u];
    }
    out->z = n;
    out->w = nullptr;
    out->in_ptr = static_cast<uint64_t *>(calloc(n + 1, sizeof(uint64_t)));
    for (uint64_t u = 0; u < n; ++u)
        out->in_ptr[u + 1] = out->in_ptr[u] + deg[u];
    out->arcs = out->in_ptr[n];
    out->in_col = static_cast<uint32_t *>(malloc(std::max<uint64_t>(out->arcs, 1) * 4));
    std::vector<uint64_t> fill(out->in_ptr, out->in_ptr + n);
    if (!directed)
        for (uint64_t u = 0; u < n; ++u)
            for (uint32_t v : own[u])
                out->in_col[fill[u]++] = v;
    for (uint64_t v = 0; v < n; ++v)
        for (uint32_t u : own[v])
            out->in_col[fill[u]++] = static_cast<uint32_t>(v);
    out->outdeg = static_cast<uint32_t *>(malloc(std::max<uint64_t>(n, 1) * sizeof(uint32_t)));
    for (uint64_t v = 0; v < n; ++v)
        out->outdeg[v] = static_cast<uint32_t>(directed ? own[v].size() : deg[v]);
}

// ---- Random hyperbolic graphs, threshold model (HyperbolicGenerator, T = 0).

// Expected average degree of a threshold RHG with n points, dispersion alpha,
// disc radius R (HyperbolicSpace.hpp getExpectedDegree), written in the same
// order of operations.
double expected_degree(double n, double alpha, double R) {
    const double gamma = 2 * alpha + 1;
    const double xi = (gamma - 1) / (gamma - 2);
    const double first = std::exp(-R / 2);
    const double second =
        std::exp(-alpha * R) *
        (alpha * (R / 2) * ((kPi / 4) * std::pow((1 / alpha), 2) - (kPi - 1) * (1 / alpha) +
                            (kPi - 2)) -
         1);
    return (2 / kPi) * xi * xi * n * (first + second);
}

// Bisection for the disc radius whose expected degree is within epsilon of k
// (HyperbolicSpace.hpp searchTargetRadiusForColdGraphs).
double target_radius(double n, double k, double alpha, double epsilon) {
    const double gamma = 2 * alpha + 1;
    const double xi_inv = (gamma - 2) / (gamma - 1);
    const double v = k * (kPi / 2) * xi_inv * xi_inv;
    double r = 2 * std::log(n / v);
    double lo = r / 2, hi = r * 2;
    do {
        r = (lo + hi) / 2;
        if (expected_degree(n, alpha, r) < k)
            hi = r;
        else
            lo = r;
    } while (std::fabs(expected_degree(n, alpha, r) - k) > epsilon);
    return r;
}

// Band boundaries: c_0 = 0, band widths in a geometric series of ratio 0.9
// over ceil(log n) - 1 inner boundaries, c_last = R
// (HyperbolicGenerator.hpp getBandRadii; n passes as an int there).
std::vector<double> band_radii(int n, double R) {
    const double ratio = 0.9;
    std::vector<double> b{0.0};
    const double a = R * (1 - ratio) / (1 - std::pow(ratio, std::log(n)));
    const double logn = std::log(n);
    for (int i = 1; i < logn; i++)
        b.push_back(a * ((1 - std::pow(ratio, i)) / (1 - ratio)));
    b.push_back(R);
    return b;
}

struct BandPoint {
    double angle, radius;
    uint32_t id;
};

// The candidates of band `band` for a point: the band's points (in angle
// order) whose angles fall in [lo, hi] as the reference's
// getPointsWithinAngles cuts that range at 0 and 2 pi: no wrap; a forward
// wrap (hi > 2 pi, tested first); a backward wrap (lo < 0). Appends them to
// `out`, duplicates included where both pieces overlap.
void points_within(double lo, double hi, const std::vector<BandPoint> &band,
                   const std::vector<double> &angles, std::vector<BandPoint> &out) {
    auto take = [&](double a, double b) {
        const size_t first = std::lower_bound(angles.begin(), angles.end(), a) - angles.begin();
        const size_t last = std::upper_bound(angles.begin(), angles.end(), b) - angles.begin();
        for (size_t i = first; i < last; ++i)
            out.push_back(band[i]);
    };
    if (lo == -2 * kPi)
        lo = 0;
    if (hi <= 2 * kPi && lo >= 0) {
        take(lo, hi);
    } else if (hi > 2 * kPi) {
        take(lo, 2 * kPi);
        take(0, std::fmod(hi, 2 * kPi));
    } else if (lo < 0) {
        take(2 * kPi + lo, 2 * kPi);
        take(0, hi);
    }
}

// One threshold RHG: points drawn from `urng`, numbered by angle, then the
// band search of HyperbolicGenerator::generateCold. Row order as toGraph
// builds it on one thread.
void hyperbolic_one(uint64_t n, double avg_deg, double exponent, std::mt19937_64 &urng,
                    int parallel_rows, nkgen_csr *out) {
    if (exponent <= 2)
        throw std::runtime_error("Exponent of power-law degree distribution must be > 2");
    if (avg_deg >= static_cast<double>(n))
        throw std::runtime_error("Average Degree must be at most n-1");
    const double alpha = 0.5 * (exponent - 1);
    // HyperbolicGenerator(n, avgDegree, plexp, 0): R = getTargetRadius(n,
    // n * avgDegree / 2, alpha, 0) with epsilon 0.01.
    const double nd = static_cast<double>(n);
    const double m = nd * avg_deg / 2;
    const double R = target_radius(nd, (m / nd) * 2, alpha, 0.01);
    // HyperbolicSpace::fillPoints over [0, 2 pi) x [0, R).
    std::vector<double> ang(n), rad(n);
    {
        std::uniform_real_distribution<double> phi{0.0, 2 * kPi};
        std::uniform_real_distribution<double> cdf{std::cosh(alpha * 0.0), std::cosh(alpha * R)};
        for (uint64_t i = 0; i < n; ++i) {
            ang[i] = phi(urng);
            const double u = cdf(urng);
            rad[i] = std::acosh(u) / alpha;
            if (rad[i] == R)
                rad[i] = std::nextafter(rad[i], 0);
        }
    }
    // Node ids in (angle, radius) order.
    std::vector<uint64_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::sort(perm.begin(), perm.end(), [&](uint64_t i, uint64_t j) {
        return ang[i] < ang[j] || (ang[i] == ang[j] && rad[i] < rad[j]);
    });
    std::vector<double> a(n), r(n);
    for (uint64_t j = 0; j < n; ++j) {
        a[j] = ang[perm[j]];
        r[j] = rad[perm[j]];
    }
    // Bands, each in angle order (a point on a boundary joins both bands).
    const std::vector<double> br = band_radii(static_cast<int>(n), R);
    const size_t nb = br.size() - 1;
    std::vector<std::vector<BandPoint>> bands(nb);
    std::vector<std::vector<double>> band_ang(nb);
    for (size_t j = 0; j < nb; ++j) {
        for (uint64_t i = 0; i < n; ++i)
            if (r[i] >= br[j] && r[i] <= br[j + 1])
                bands[j].push_back({a[i], r[i], static_cast<uint32_t>(i)});
        band_ang[j].resize(bands[j].size());
        for (size_t q = 0; q < bands[j].size(); ++q)
            band_ang[j][q] = bands[j][q].angle;
    }
    const double cosh_R = std::cosh(R);
    std::vector<std::vector<uint32_t>> own(n);
#pragma omp parallel for schedule(dynamic, 256) if (parallel_rows)
    for (int64_t ii = 0; ii < static_cast<int64_t>(n); ++ii) {
        const uint64_t i = static_cast<uint64_t>(ii);
        const double cosh_r = std::cosh(r[i]);
        const double sinh_r = std::sinh(r[i]);
        std::vector<BandPoint> cand;
        std::vector<uint32_t> near;
        for (size_t j = 0; j < nb; ++j) {
            if (!(br[j + 1] > r[i]))
                continue;
            // getMinMaxTheta: the angular half-width of the disc of radius R
            // around point i where it meets radius br[j].
            double lo = 0.0, hi = 2 * kPi;
            if (br[j] != 0) {
                double c = (std::cosh(r[i]) * std::cosh(br[j]) - std::cosh(R)) /
                           (std::sinh(r[i]) * std::sinh(br[j]));
                if (c < -1)
                    c = -1;
                else if (c > 1)
                    c = 1;
                c = std::acos(c);
                hi = a[i] + c;
                lo = a[i] - c;
            }
            cand.clear();
            points_within(lo, hi, bands[j], band_ang[j], cand);
            for (const BandPoint &w : cand) {
                const double dphi = kPi - std::fabs(kPi - std::fabs(a[i] - w.angle));
                if (cosh_r * std::cosh(w.radius) - sinh_r * std::sinh(w.radius) * std::cos(dphi) <=
                    cosh_R) {
                    if (w.id != i)
                        near.push_back(w.id);
                }
            }
        }
        for (uint32_t j : near)
            if (r[j] > r[i] || (r[j] == r[i] && a[j] < a[i]))
                own[i].push_back(j);
    }
    half_edges_to_csr(own, false, out);
}

} // namespace

extern "C" {

// G(n, p) as NetworKit's ErdosRenyiGenerator(n, p, directed) draws it with
// `threads` OpenMP threads (ErdosRenyiGenerator.cpp:21-33,
// ErdosRenyiEnumerator.hpp). Thread t takes a range of rows: ceil(n / T) rows
// each (directed), or, undirected, rows whose lower-triangle cells add up to
// about 1/T of all cells (the reference's sqrt-based boundaries), the last
// thread to n. Every thread's generator is seeded with the same `seed`
// (setSeed(seed, false)), so every range restarts the same stream. Within a
// range: 64-bit fixed-point uniforms X in [1, 2^64 - 1]
// (std::uniform_int_distribution) and geometric skips
// 1 + floor((log2 X - 64) / log2(1 - q)) over the range's cells in row order
// (Batagelj & Brandes): columns 0..n-1 (directed) or 0..u-1 (undirected, rows
// from 1). q = p; for p > 0.9 the draw runs with q = 1 - p and the range's
// cells are emitted in order from a cursor that stops at each drawn cell and
// goes on from it, as the reference's complement pass does (so every cell is
// emitted). No draws when q < n^-3. Self-loops of the directed draw are
// dropped. Rows as GraphBuilder::toGraph(true, false) builds them.
int nkgen_erdos_renyi_stream(uint64_t n, double p, uint64_t seed, int directed, int threads,
                             nkgen_csr *out) {
    try {
        if (n < 1 || n >= 0xffffffffull)
            throw std::runtime_error("n out of range");
        if (!(p >= 0.0 && p <= 1.0))
            throw std::runtime_error("p must be in [0, 1]");
        if (threads < 1)
            throw std::runtime_error("threads must be at least 1");
        const bool dir = directed != 0;
        std::vector<std::vector<uint32_t>> own(n);
        auto emit = [&](uint64_t u, uint64_t v) {
            if (u != v)
                own[u].push_back(static_cast<uint32_t>(v));
        };
        const bool complement = p > 0.9;
        const double q = complement ? 1.0 - p : p;
        // One thread's range [begin, end) of rows, drawn as the reference does.
        auto draw_range = [&](uint64_t begin, uint64_t end) {
            uint64_t cu = begin, cv = 0;  // complement cursor
            if (!dir && cu == 0)
                cu = 1;
            auto cover_to = [&](uint64_t u, uint64_t v) {
                while (!(cu == u && cv == v)) {
                    emit(cu, cv);
                    if (++cv == (dir ? n : cu)) {
                        cv = 0;
                        ++cu;
                    }
                }
            };
            if (!(q < std::pow(static_cast<double>(n), -3.0))) {
                const double inv_log2 = 1.0 / std::log2(1.0 - q);
                std::mt19937_64 urng(seed);
                std::uniform_int_distribution<unsigned long long> uni{
                    1, std::numeric_limits<unsigned long long>::max()};
                uint64_t cur = begin;
                if (!dir && cur == 0)
                    cur = 1;
                uint64_t nxt = ~0ull;
                while (cur < end) {
                    const double x = static_cast<double>(uni(urng));
                    nxt += 1 + static_cast<uint64_t>(std::floor((std::log2(x) - 64.0) * inv_log2));
                    while (nxt >= (dir ? n : cur)) {
                        nxt -= dir ? n : cur;
                        ++cur;
                    }
                    if (cur < end) {
                        if (complement)
                            cover_to(cur, nxt);
                        else
                            emit(cur, nxt);
                    }
                }
            }
            if (complement)
                cover_to(end, 0);
        };
        const uint64_t T = static_cast<uint64_t>(threads);
        if (dir) {
            const uint64_t chunk = (n + T - 1) / T;
            for (uint64_t t = 0; t < T; ++t) {
                const uint64_t b = std::min(n, t * chunk), e = std::min(n, (t + 1) * chunk);
                if (b < e)
                    draw_range(b, e);
            }
        } else {
            // ErdosRenyiEnumerator::forEdgesParallel, undirected: boundaries in
            // double arithmetic as the reference computes them.
            const uint64_t chunk = (n * (n - 1) / 2 + T - 1) / T;
            double last = 0.0;
            for (uint64_t t = 0; t < T; ++t) {
                const double first = last;
                const uint64_t upper = static_cast<uint64_t>(
                    std::ceil(std::sqrt(0.25 + first * first + first + 2 * chunk)));
                last = static_cast<double>(std::min<uint64_t>(n, upper));
                double end = last;
                if (t + 1 == T)
                    end = static_cast<double>(n);
                if (first < end)
                    draw_range(static_cast<uint64_t>(first), static_cast<uint64_t>(end));
            }
        }
        half_edges_to_csr(own, dir, out);
        return 0;
    } catch (const std::exception &e) {
        nkgen_set_error(e.what());
        return -1;
    }
}

// Barabasi-Albert as NetworKit's BarabasiAlbertGenerator(k, n, n0) draws it
// (its default, Batagelj & Brandes' edge-list method;
// BarabasiAlbertGenerator.cpp generateBatagelj): a ring over the first
// max(n0, k) nodes (edges (v, v+1), then (0, n0-1)); every later node v draws
// uniform indices into the edge-endpoint list as it stood before v
// (std::uniform_int_distribution over [0, size - 1]) and keeps an endpoint
// unless v already links to it, until it has k neighbours. The adjacency is
// the Graph that adds the listed edges in order (Graph::addEdge: a
// self-loop, the ring's for n0 = 1, is stored once).
int nkgen_barabasi_albert_stream(uint64_t k, uint64_t n, uint64_t n0, uint64_t seed,
                                 nkgen_csr *out) {
    try {
        if (k < 1)
            throw std::runtime_error("k must be at least 1");
        if (k > n)
            throw std::runtime_error("k may not be larger than the number of nodes");
        if (n0 > n)
            throw std::runtime_error("n0 may not be larger than the number of nodes");
        if (n >= 0xffffffffull)
            throw std::runtime_error("n out of range");
        if (n0 < k)
            n0 = k;
        std::vector<uint32_t> M;
        M.reserve(2 * n0 + 2 * (n - n0) * k);
        auto add = [&](uint64_t u, uint64_t v) {
            M.push_back(static_cast<uint32_t>(u));
            M.push_back(static_cast<uint32_t>(v));
        };
        for (uint64_t v = 0; v + 1 < n0; ++v)
            add(v, v + 1);
        add(0, n0 - 1);
        std::mt19937_64 urng(seed);
        for (uint64_t v = n0; v < n; ++v) {
            std::uniform_int_distribution<size_t> pick{0, M.size() - 1};
            const size_t first = M.size() + 1;  // v's neighbours: odd positions from here
            for (uint64_t i = 0; i < k; ++i) {
                for (;;) {
                    const uint32_t w = M[pick(urng)];
                    bool linked = false;
                    for (size_t j = first; j < M.size(); j += 2)
                        if (M[j] == w) {
                            linked = true;
                            break;
                        }
                    if (!linked) {
                        add(v, w);
                        break;
                    }
                }
            }
        }
        std::vector<uint64_t> deg(n, 0);
        for (size_t i = 0; i < M.size(); i += 2) {
            ++deg[M[i]];
            if (M[i] != M[i + 1])
                ++deg[M[i + 1]];
        }
        out->z = n;
        out->w = nullptr;
        out->in_ptr = static_cast<uint64_t *>(calloc(n + 1, sizeof(uint64_t)));
        for (uint64_t u = 0; u < n; ++u)
            out->in_ptr[u + 1] = out->in_ptr[u] + deg[u];
        out->arcs = out->in_ptr[n];
        out->in_col = static_cast<uint32_t *>(malloc(std::max<uint64_t>(out->arcs, 1) * 4));
        std::vector<uint64_t> fill(out->in_ptr, out->in_ptr + n);
        for (size_t i = 0; i < M.size(); i += 2) {
            const uint32_t a = M[i], b = M[i + 1];
            out->in_col[fill[a]++] = b;
            if (a != b)
                out->in_col[fill[b]++] = a;
        }
        out->outdeg = static_cast<uint32_t *>(malloc(n * sizeof(uint32_t)));
        for (uint64_t u = 0; u < n; ++u)
            out->outdeg[u] = static_cast<uint32_t>(deg[u]);
        return 0;
    } catch (const std::exception &e) {
        nkgen_set_error(e.what());
        return -1;
    }
}

// Threshold random hyperbolic graph as NetworKit's HyperbolicGenerator(n,
// avg_deg, exponent).generate() draws it (temperature 0;
// HyperbolicGenerator.cpp:37-205, HyperbolicSpace fillPoints and
// getTargetRadius): alpha = (exponent - 1) / 2, the disc radius whose
// expected degree is within 0.01 of avg_deg, n points (angle uniform in
// [0, 2 pi), then cosh(alpha r) uniform in [1, cosh(alpha R)]) numbered by
// angle, and every pair at hyperbolic distance <= R found through the radial
// bands, as the half edge of its point with the smaller radius. Rows as
// GraphBuilder::toGraph builds them on one thread. The rows' neighbour
// search runs on all threads; the result does not depend on their number.
int nkgen_hyperbolic_stream(uint64_t n, double avg_deg, double exponent, uint64_t seed,
                            nkgen_csr *out) {
    try {
        if (n < 2 || n >= 0x7fffffffull)
            throw std::runtime_error("n out of range");
        std::mt19937_64 urng(seed);
        hyperbolic_one(n, avg_deg, exponent, urng, 1, out);
        return 0;
    } catch (const std::exception &e) {
        nkgen_set_error(e.what());
        return -1;
    }
}

// count graphs of nkgen_hyperbolic_stream, graph i with ns[i] nodes and seed
// seed + i, as one block-diagonal in-CSR (graph i = nodes
// [node_offsets[i], node_offsets[i + 1])). Graphs are drawn in parallel.
int nkgen_hyperbolic_stream_batch(uint64_t count, const uint64_t *ns, double avg_deg,
                                  double exponent, uint64_t seed, nkgen_csr *out,
                                  uint64_t *node_offsets) {
    try {
        std::vector<nkgen_csr> parts(count);
        for (uint64_t i = 0; i < count; ++i)
            if (ns[i] < 2 || ns[i] >= 0x7fffffffull)
                throw std::runtime_error("n out of range");
        node_offsets[0] = 0;
        for (uint64_t i = 0; i < count; ++i)
            node_offsets[i + 1] = node_offsets[i] + ns[i];
        if (node_offsets[count] >= 0xffffffffull)
            throw std::runtime_error("too many nodes in the batch");
        std::vector<std::string> errs(count);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t i = 0; i < static_cast<int64_t>(count); ++i) {
            try {
                std::mt19937_64 urng(seed + static_cast<uint64_t>(i));
                hyperbolic_one(ns[i], avg_deg, exponent, urng, 0, &parts[i]);
            } catch (const std::exception &e) {
                errs[i] = e.what();
            }
        }
        for (uint64_t i = 0; i < count; ++i)
            if (!errs[i].empty()) {
                for (auto &p : parts) {
                    free(p.in_ptr);
                    free(p.in_col);
                    free(p.outdeg);
                }
                throw std::runtime_error(errs[i]);
            }
        uint64_t arcs = 0;
        for (auto &p : parts)
            arcs += p.arcs;
        const uint64_t z = node_offsets[count];
        out->z = z;
        out->arcs = arcs;
        out->w = nullptr;
        out->in_ptr = static_cast<uint64_t *>(malloc((z + 1) * sizeof(uint64_t)));
        out->in_col = static_cast<uint32_t *>(malloc(std::max<uint64_t>(arcs, 1) * 4));
        out->outdeg = static_cast<uint32_t *>(malloc(std::max<uint64_t>(z, 1) * 4));
        uint64_t a0 = 0;
        out->in_ptr[0] = 0;
        for (uint64_t i = 0; i < count; ++i) {
            const nkgen_csr &p = parts[i];
            const uint64_t v0 = node_offsets[i];
            for (uint64_t v = 0; v < p.z; ++v) {
                out->in_ptr[v0 + v + 1] = a0 + p.in_ptr[v + 1];
                out->outdeg[v0 + v] = p.outdeg[v];
            }
            for (uint64_t e = 0; e < p.arcs; ++e)
                out->in_col[a0 + e] = p.in_col[e] + static_cast<uint32_t>(v0);
            a0 += p.arcs;
            free(p.in_ptr);
            free(p.in_col);
            free(p.outdeg);
        }
        return 0;
    } catch (const std::exception &e) {
        nkgen_set_error(e.what());
        return -1;
    }
}

} // extern "C"
