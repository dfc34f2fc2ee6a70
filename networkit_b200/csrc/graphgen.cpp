// Host-side synthetic graph generators (C++/OpenMP) for the benchmark and
// test workloads. Every random draw comes from a counter-based hash of
// (seed, stream, counter), so the output does not depend on the number of
// threads. Output is the canonical in-CSR the PageRank boundary takes:
// edges are taken as inserted in lexicographic (u, v) order, which makes every
// in-row ascending (directed: sources of v; undirected: neighbours of v).
//
//   R-MAT    - the recursive quadrant draw of RmatGenerator.cpp:37-65
//              (quadrant 0/1/2/3 with probabilities a/b/c/d, bit of u from
//              q>>1, bit of v from q&1), directed, duplicates and self-loops
//              dropped.
//   G(n,p)   - Erdos-Renyi by geometric skipping (Batagelj & Brandes, "Efficient
//              generation of large random networks", Phys. Rev. E 71, 2005).
//   BA       - preferential attachment as in the same paper (edge-list
//              sampling), with the reference's distinct-neighbour rule and
//              initial ring of k nodes (BarabasiAlbertGenerator.cpp).
//   RHG      - threshold random hyperbolic graphs (Krioukov et al. 2010) with a
//              radial band index (von Looz et al., "Generating massive complex
//              networks with hyperbolic geometry faster in practice", 2016).
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "nkgen.hpp"

namespace {

// SplitMix64 output function (Steele, Lea, Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014).
inline uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

inline uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t ctr) {
    return mix64(mix64(seed ^ mix64(stream * 0x2545f4914f6cdd1dull)) + ctr);
}

// Uniform double in [0, 1) with 53 random bits.
inline double u01(uint64_t h) { return static_cast<double>(h >> 11) * (1.0 / 9007199254740992.0); }

thread_local std::string g_err;

// Parallel LSD radix sort of 64-bit keys on their low `bits` bits.
void radix_sort(std::vector<uint64_t> &keys, int bits) {
    const size_t n = keys.size();
    std::vector<uint64_t> tmp(n);
    const int D = 11;
    const size_t B = size_t(1) << D;
    const int nt = omp_get_max_threads();
    std::vector<size_t> hist(static_cast<size_t>(nt) * B);
    uint64_t *src = keys.data(), *dst = tmp.data();
    int passes = 0;
    for (int shift = 0; shift < bits; shift += D) {
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nt)
        {
            const int t = omp_get_thread_num();
            const size_t lo = n * t / nt, hi = n * (t + 1) / nt;
            size_t *h = hist.data() + static_cast<size_t>(t) * B;
            for (size_t i = lo; i < hi; ++i)
                ++h[(src[i] >> shift) & (B - 1)];
#pragma omp barrier
#pragma omp single
            {
                size_t run = 0;
                for (size_t d = 0; d < B; ++d)
                    for (int tt = 0; tt < nt; ++tt) {
                        size_t &c = hist[static_cast<size_t>(tt) * B + d];
                        const size_t v = c;
                        c = run;
                        run += v;
                    }
            }
            for (size_t i = lo; i < hi; ++i) {
                const uint64_t k = src[i];
                dst[h[(k >> shift) & (B - 1)]++] = k;
            }
        }
        std::swap(src, dst);
        ++passes;
    }
    if (passes & 1)
        keys.swap(tmp);
}

struct Csr {
    uint64_t z = 0, arcs = 0;
    uint64_t *in_ptr = nullptr;
    uint32_t *in_col = nullptr;
    uint32_t *outdeg = nullptr;
    double *w = nullptr;
};

// Sorted unique keys (dst << shift | src) -> in-CSR.
void keys_to_csr(const std::vector<uint64_t> &keys, uint64_t z, int shift, Csr &out) {
    const uint64_t mask = (uint64_t(1) << shift) - 1;
    const uint64_t m = keys.size();
    out.z = z;
    out.arcs = m;
    out.in_ptr = static_cast<uint64_t *>(calloc(z + 1, sizeof(uint64_t)));
    out.in_col = static_cast<uint32_t *>(malloc(std::max<uint64_t>(m, 1) * sizeof(uint32_t)));
    out.outdeg = static_cast<uint32_t *>(calloc(z, sizeof(uint32_t)));
    if (!out.in_ptr || !out.in_col || !out.outdeg)
        throw std::bad_alloc();
    std::vector<std::atomic<uint32_t>> cnt(z);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < static_cast<int64_t>(z); ++i)
        cnt[i].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < static_cast<int64_t>(m); ++e) {
        const uint64_t k = keys[e];
        out.in_col[e] = static_cast<uint32_t>(k & mask);
        cnt[k >> shift].fetch_add(1, std::memory_order_relaxed);
        __atomic_fetch_add(&out.outdeg[k & mask], 1u, __ATOMIC_RELAXED);
    }
    uint64_t run = 0;
    out.in_ptr[0] = 0;
    for (uint64_t v = 0; v < z; ++v) {
        run += cnt[v].load(std::memory_order_relaxed);
        out.in_ptr[v + 1] = run;
    }
}

void dedupe_sorted(std::vector<uint64_t> &keys) {
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
}

// ---------------------------------------------------------------------------
// Random hyperbolic graphs (threshold model, temperature 0)

// Model (Krioukov, Papadopoulos, Kitsak, Vahdat, Boguna, "Hyperbolic geometry
// of complex networks", Phys. Rev. E 82, 2010): n points in a disc of
// radius R of the hyperbolic plane, angles uniform, radii with density
// alpha sinh(alpha r) / (cosh(alpha R) - 1), alpha = (exponent - 1) / 2; two
// points are adjacent iff their hyperbolic distance is at most R, where
//     cosh d = cosh r1 cosh r2 - sinh r1 sinh r2 cos(theta1 - theta2).
struct RhgPoint {
    double theta, r, ch, sh;
};

// Largest angular difference at which radii r1, r2 are still within
// distance R (pi when every angle is).
inline double max_angle(double r1, double ch1, double sh1, double r2, double ch2, double sh2,
                        double R, double chR) {
    if (r1 + r2 <= R || sh1 == 0.0 || sh2 == 0.0)
        return M_PI;
    const double c = (ch1 * ch2 - chR) / (sh1 * sh2);
    if (c <= -1.0)
        return M_PI;
    if (c >= 1.0)
        return 0.0;
    return std::acos(c);
}

// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on the
// Legendre polynomial P_m from the usual cosine starting guesses).
void gauss_legendre(int m, std::vector<double> &x, std::vector<double> &w) {
    x.assign(m, 0.0);
    w.assign(m, 0.0);
    for (int i = 0; i < (m + 1) / 2; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (m + 0.5)), dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = 0.0;
            for (int j = 1; j <= m; ++j) {
                const double p2 = p1;
                p1 = p0;
                p0 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j;
            }
            dp = m * (z * p0 - p1) / (z * z - 1.0);
            const double dz = p0 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-15)
                break;
        }
        x[i] = -z;
        x[m - 1 - i] = z;
        w[i] = w[m - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

// Probability that two random points are within distance R:
//     P = int f(r1) [ F(R - r1) + int_{R-r1}^{R} f(r2) theta_max(r1, r2) / pi dr2 ] dr1
// with f, F the radial density and its CDF (theta_max = pi below r1 + r2 = R).
// The inner integral has a square-root edge at r2 = R - r1, removed by
// r2 = R - r1 + r1 t^2; both integrals use composite Gauss-Legendre rules
// (outer: panels of width <= 1, 8 nodes each; inner: 16 nodes on t in [0, 1]).
double rhg_pair_probability(double R, double alpha) {
    static thread_local std::vector<double> xo, wo, xi, wi;
    if (xo.empty()) {
        gauss_legendre(8, xo, wo);
        gauss_legendre(16, xi, wi);
    }
    const double span = std::cosh(alpha * R) - 1.0;
    const double chR = std::cosh(R);
    const int panels = std::max(1, static_cast<int>(std::ceil(R)));
    const double h = R / panels;
    double total = 0.0;
    for (int pnl = 0; pnl < panels; ++pnl) {
        for (size_t a = 0; a < xo.size(); ++a) {
            const double r1 = (pnl + 0.5) * h + 0.5 * h * xo[a];
            const double f1 = alpha * std::sinh(alpha * r1) / span;
            const double ch1 = std::cosh(r1), sh1 = std::sinh(r1);
            double inner = (std::cosh(alpha * (R - r1)) - 1.0) / span;
            for (size_t b = 0; b < xi.size(); ++b) {
                const double t = 0.5 * (xi[b] + 1.0);
                const double r2 = R - r1 + r1 * t * t;
                const double th = max_angle(r1, ch1, sh1, r2, std::cosh(r2), std::sinh(r2), R, chR);
                inner += 0.5 * wi[b] * alpha * std::sinh(alpha * r2) / span * (th / M_PI) * 2.0 *
                         r1 * t;
            }
            total += 0.5 * h * wo[a] * f1 * inner;
        }
    }
    return total;
}

// Disc radius that gives expected average degree avg_deg: solve
// (n - 1) P(R) = avg_deg by bisection (P decreases in R).
double rhg_radius(uint64_t n, double avg_deg, double alpha) {
    const double target = avg_deg / static_cast<double>(n - 1);
    // Bracket around the large-n estimate avg_deg ~ (2/pi) xi^2 n e^{-R/2},
    // xi = alpha / (alpha - 1/2).
    const double xi = alpha > 0.5 ? alpha / (alpha - 0.5) : 2.0;
    const double r0 = 2.0 * std::log(2.0 / M_PI * xi * xi * static_cast<double>(n) / avg_deg);
    double lo = std::max(1e-6, r0 - 8.0), hi = r0 + 8.0;
    while (lo > 1e-6 && rhg_pair_probability(lo, alpha) < target)
        lo = std::max(1e-6, lo - 4.0);
    while (rhg_pair_probability(hi, alpha) > target)
        hi += 4.0;
    for (int it = 0; it < 80 && hi - lo > 1e-12; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (rhg_pair_probability(mid, alpha) > target)
            lo = mid;
        else
            hi = mid;
    }
    return 0.5 * (lo + hi);
}

// One graph: its neighbour lists (rows ascending). Node ids follow the
// points sorted by angle, then radius, as HyperbolicGenerator numbers them
// (HyperbolicGenerator.cpp:75-92): angularly close nodes get close ids.
// Bands of radial width 1 counted from the rim (the inner band takes the
// rest) hold their points sorted by angle; a point queries every band over
// the angular window that the band's inner radius allows, then tests each
// candidate exactly. Both ends of an edge evaluate the same symmetric
// expression, so the lists are symmetric.
void rhg_rows(uint64_t n, double avg_deg, double exponent, uint64_t seed,
              std::vector<uint64_t> &ptr, std::vector<uint32_t> &col) {
    const double alpha = (exponent - 1.0) / 2.0;
    const double R = rhg_radius(n, avg_deg, alpha);
    const double chR = std::cosh(R);
    const double span = std::cosh(alpha * R) - 1.0;
    std::vector<RhgPoint> drawn(n);
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t h1 = hash3(seed, 1, i), h2 = hash3(seed, 2, i);
        RhgPoint &p = drawn[i];
        p.theta = 2.0 * M_PI * u01(h1);
        p.r = std::acosh(1.0 + u01(h2) * span) / alpha;
        p.ch = std::cosh(p.r);
        p.sh = std::sinh(p.r);
    }
    std::vector<uint32_t> by_angle(n);
    std::iota(by_angle.begin(), by_angle.end(), 0u);
    std::sort(by_angle.begin(), by_angle.end(), [&](uint32_t x, uint32_t y) {
        return drawn[x].theta < drawn[y].theta ||
               (drawn[x].theta == drawn[y].theta &&
                (drawn[x].r < drawn[y].r || (drawn[x].r == drawn[y].r && x < y)));
    });
    std::vector<RhgPoint> pts(n);
    for (uint64_t j = 0; j < n; ++j)
        pts[j] = drawn[by_angle[j]];
    drawn.clear();
    const int nb = std::max(1, static_cast<int>(std::ceil(R)));
    std::vector<double> inner(nb);
    for (int b = 0; b < nb; ++b)
        inner[b] = std::max(0.0, R - (b + 1));  // band b: [R-b-1, R-b), band nb-1 reaches 0
    inner[nb - 1] = 0.0;
    std::vector<std::vector<uint32_t>> band(nb);
    for (uint64_t i = 0; i < n; ++i) {
        int b = static_cast<int>(std::floor(R - pts[i].r));
        b = std::min(std::max(b, 0), nb - 1);
        band[b].push_back(static_cast<uint32_t>(i));
    }
    std::vector<std::vector<double>> bth(nb);
    for (int b = 0; b < nb; ++b) {
        std::sort(band[b].begin(), band[b].end(), [&](uint32_t x, uint32_t y) {
            return pts[x].theta < pts[y].theta || (pts[x].theta == pts[y].theta && x < y);
        });
        bth[b].resize(band[b].size());
        for (size_t k = 0; k < band[b].size(); ++k)
            bth[b][k] = pts[band[b][k]].theta;
    }
    std::vector<std::vector<uint32_t>> rows(n);
    for (uint64_t i = 0; i < n; ++i) {
        const RhgPoint &p = pts[i];
        std::vector<uint32_t> &row = rows[i];
        for (int b = 0; b < nb; ++b) {
            if (band[b].empty())
                continue;
            const double ri = inner[b];
            const double d = max_angle(p.r, p.ch, p.sh, ri, std::cosh(ri), std::sinh(ri), R, chR) +
                             1e-9;
            const std::vector<double> &th = bth[b];
            auto scan = [&](double lo, double hi) {  // [lo, hi] within [0, 2 pi)
                size_t k = std::lower_bound(th.begin(), th.end(), lo) - th.begin();
                for (; k < th.size() && th[k] <= hi; ++k) {
                    const uint32_t j = band[b][k];
                    if (j == i)
                        continue;
                    const RhgPoint &q = pts[j];
                    const double cd = p.ch * q.ch - p.sh * q.sh * std::cos(p.theta - q.theta);
                    if (cd <= chR)
                        row.push_back(j);
                }
            };
            if (d >= M_PI) {
                scan(0.0, 2.0 * M_PI);
            } else {
                const double lo = p.theta - d, hi = p.theta + d;
                if (lo < 0.0) {
                    scan(0.0, hi);
                    scan(lo + 2.0 * M_PI, 2.0 * M_PI);
                } else if (hi >= 2.0 * M_PI) {
                    scan(lo, 2.0 * M_PI);
                    scan(0.0, hi - 2.0 * M_PI);
                } else {
                    scan(lo, hi);
                }
            }
        }
        std::sort(row.begin(), row.end());
    }
    ptr.assign(n + 1, 0);
    for (uint64_t i = 0; i < n; ++i)
        ptr[i + 1] = ptr[i] + rows[i].size();
    col.resize(ptr[n]);
    for (uint64_t i = 0; i < n; ++i)
        std::copy(rows[i].begin(), rows[i].end(), col.begin() + ptr[i]);
}

} // namespace

void nkgen_set_error(const char *msg) { g_err = msg; }

extern "C" {

const char *nkgen_last_error(void) { return g_err.c_str(); }

void nkgen_free(nkgen_csr *c) {
    if (!c)
        return;
    free(c->in_ptr);
    free(c->in_col);
    free(c->outdeg);
    free(c->w);
    std::memset(c, 0, sizeof(*c));
}

static void export_csr(const Csr &c, nkgen_csr *out) {
    out->z = c.z;
    out->arcs = c.arcs;
    out->in_ptr = c.in_ptr;
    out->in_col = c.in_col;
    out->outdeg = c.outdeg;
    out->w = c.w;
}

// Directed R-MAT: edgefactor * 2^scale draws, then duplicates and self-loops
// removed. a, b, c as in RmatGenerator (d = 1 - a - b - c).
int nkgen_rmat(int scale, uint64_t edgefactor, double a, double b, double c, uint64_t seed,
               int nthreads, nkgen_csr *out) {
    try {
        if (scale < 1 || scale > 31)
            throw std::runtime_error("scale must be in [1, 31]");
        if (nthreads > 0)
            omp_set_num_threads(nthreads);
        const uint64_t z = uint64_t(1) << scale;
        const uint64_t draws = edgefactor * z;
        const double S = 4294967296.0;
        const uint64_t ta = static_cast<uint64_t>(a * S), tab = static_cast<uint64_t>((a + b) * S),
                       tabc = static_cast<uint64_t>((a + b + c) * S);
        std::vector<uint64_t> keys(draws);
        const uint64_t loop_key = uint64_t(1) << (2 * scale);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < static_cast<int64_t>(draws); ++i) {
            uint64_t u = 0, v = 0, h = 0;
            for (int l = 0; l < scale; ++l) {
                if ((l & 1) == 0)
                    h = hash3(seed, static_cast<uint64_t>(i), static_cast<uint64_t>(l >> 1));
                const uint64_t r = (l & 1) ? (h >> 32) : (h & 0xffffffffu);
                const unsigned q = r < ta ? 0u : r < tab ? 1u : r < tabc ? 2u : 3u;
                u = (u << 1) | (q >> 1);
                v = (v << 1) | (q & 1u);
            }
            // self-loops get a key above every edge and are cut off below
            keys[i] = (u == v) ? loop_key : ((v << scale) | u);
        }
        radix_sort(keys, 2 * scale + 1);
        while (!keys.empty() && keys.back() == loop_key)
            keys.pop_back();
        dedupe_sorted(keys);
        Csr cs;
        keys_to_csr(keys, z, scale, cs);
        export_csr(cs, out);
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

// Undirected G(n, p): every pair {w, v} (w < v) independently with
// probability p. Node v draws its lower neighbours with its own stream.
int nkgen_erdos_renyi(uint64_t n, double p, uint64_t seed, int nthreads, nkgen_csr *out) {
    try {
        if (n < 1 || n >= 0xffffffffull)
            throw std::runtime_error("n out of range");
        if (!(p >= 0.0 && p <= 1.0))
            throw std::runtime_error("p must be in [0, 1]");
        if (nthreads > 0)
            omp_set_num_threads(nthreads);
        std::vector<std::vector<uint32_t>> lower(n);
        const double lp = std::log(1.0 - p);
#pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t v = 1; v < static_cast<int64_t>(n); ++v) {
            if (p <= 0.0)
                continue;
            int64_t w = -1;
            uint64_t ctr = 0;
            for (;;) {
                if (p >= 1.0) {
                    ++w;
                } else {
                    const double r = u01(hash3(seed, static_cast<uint64_t>(v), ctr++));
                    w += 1 + static_cast<int64_t>(std::floor(std::log(1.0 - r) / lp));
                }
                if (w >= v)
                    break;
                lower[v].push_back(static_cast<uint32_t>(w));
            }
        }
        std::vector<uint64_t> deg(n, 0);
        for (uint64_t v = 0; v < n; ++v) {
            deg[v] += lower[v].size();
            for (uint32_t w : lower[v])
                deg[w] += 1;
        }
        Csr cs;
        cs.z = n;
        cs.in_ptr = static_cast<uint64_t *>(calloc(n + 1, sizeof(uint64_t)));
        for (uint64_t v = 0; v < n; ++v)
            cs.in_ptr[v + 1] = cs.in_ptr[v] + deg[v];
        cs.arcs = cs.in_ptr[n];
        cs.in_col = static_cast<uint32_t *>(malloc(std::max<uint64_t>(cs.arcs, 1) * sizeof(uint32_t)));
        cs.outdeg = static_cast<uint32_t *>(malloc(n * sizeof(uint32_t)));
        std::vector<uint64_t> fill(cs.in_ptr, cs.in_ptr + n);
        // Rows ascending: lower neighbours first (ascending), then upper ones
        // appended in increasing v.
        for (uint64_t v = 0; v < n; ++v)
            for (uint32_t w : lower[v])
                cs.in_col[fill[v]++] = w;
        for (uint64_t v = 0; v < n; ++v)
            for (uint32_t w : lower[v])
                cs.in_col[fill[w]++] = static_cast<uint32_t>(v);
        for (uint64_t v = 0; v < n; ++v)
            cs.outdeg[v] = static_cast<uint32_t>(deg[v]);
        export_csr(cs, out);
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

// Undirected Barabasi-Albert: initial ring of k nodes, then every new node
// attaches to k distinct nodes drawn from the endpoint list of the edges that
// existed before it (preferential attachment by degree).
int nkgen_barabasi_albert(uint64_t k, uint64_t n, uint64_t seed, nkgen_csr *out) {
    try {
        if (k < 1 || n <= k || n >= 0xffffffffull)
            throw std::runtime_error("need 1 <= k < n < 2^32");
        std::vector<uint32_t> M;
        M.reserve(2 * k + 2 * (n - k) * k);
        for (uint64_t v = 0; v + 1 < k; ++v) {
            M.push_back(static_cast<uint32_t>(v));
            M.push_back(static_cast<uint32_t>(v + 1));
        }
        if (k >= 2) {
            M.push_back(0);
            M.push_back(static_cast<uint32_t>(k - 1));
        }
        uint64_t ctr = 0;
        for (uint64_t v = k; v < n; ++v) {
            const uint64_t range = M.size();
            const size_t first = M.size() + 1;
            for (uint64_t i = 0; i < k; ++i) {
                for (;;) {
                    uint32_t nb;
                    if (range == 0) {
                        nb = static_cast<uint32_t>(i);  // k == 1: attach to node 0
                    } else {
                        const uint64_t idx = static_cast<uint64_t>(u01(hash3(seed, 0, ctr++)) * range);
                        nb = M[idx < range ? idx : range - 1];
                    }
                    bool dup = false;
                    for (size_t j = first; j < M.size(); j += 2)
                        if (M[j] == nb) {
                            dup = true;
                            break;
                        }
                    if (!dup) {
                        M.push_back(static_cast<uint32_t>(v));
                        M.push_back(nb);
                        break;
                    }
                }
            }
        }
        // Canonical key (dst << 32 | src) for both directions, sorted.
        const uint64_t m = M.size() / 2;
        std::vector<uint64_t> keys(2 * m);
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < static_cast<int64_t>(m); ++e) {
            const uint64_t u = M[2 * e], v = M[2 * e + 1];
            keys[2 * e] = (v << 32) | u;
            keys[2 * e + 1] = (u << 32) | v;
        }
        radix_sort(keys, 64);
        dedupe_sorted(keys);
        Csr cs;
        keys_to_csr(keys, n, 32, cs);
        export_csr(cs, out);
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

// Undirected threshold random hyperbolic graph (see rhg_rows).
int nkgen_hyperbolic(uint64_t n, double avg_deg, double exponent, uint64_t seed, nkgen_csr *out) {
    try {
        if (n < 2 || n >= 0xffffffffull)
            throw std::runtime_error("need 2 <= n < 2^32");
        if (!(avg_deg > 0.0) || !(avg_deg < static_cast<double>(n - 1)))
            throw std::runtime_error("avg_deg must be in (0, n - 1)");
        if (!(exponent > 2.0))
            throw std::runtime_error("exponent must be > 2");
        std::vector<uint64_t> ptr;
        std::vector<uint32_t> col;
        rhg_rows(n, avg_deg, exponent, seed, ptr, col);
        Csr cs;
        cs.z = n;
        cs.arcs = ptr[n];
        cs.in_ptr = static_cast<uint64_t *>(malloc((n + 1) * sizeof(uint64_t)));
        cs.in_col = static_cast<uint32_t *>(malloc(std::max<uint64_t>(cs.arcs, 1) * sizeof(uint32_t)));
        cs.outdeg = static_cast<uint32_t *>(malloc(n * sizeof(uint32_t)));
        if (!cs.in_ptr || !cs.in_col || !cs.outdeg)
            throw std::bad_alloc();
        std::copy(ptr.begin(), ptr.end(), cs.in_ptr);
        std::copy(col.begin(), col.end(), cs.in_col);
        for (uint64_t v = 0; v < n; ++v)
            cs.outdeg[v] = static_cast<uint32_t>(ptr[v + 1] - ptr[v]);
        export_csr(cs, out);
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

// `count` hyperbolic graphs (graph i: ns[i] nodes, seed + i) as one
// block-diagonal in-CSR: graph i holds the nodes [node_offsets[i],
// node_offsets[i+1]) (caller array of count+1). Graphs are generated in
// parallel, largest first; the output does not depend on the thread count.
int nkgen_hyperbolic_batch(uint64_t count, const uint64_t *ns, double avg_deg, double exponent,
                           uint64_t seed, int nthreads, nkgen_csr *out, uint64_t *node_offsets) {
    try {
        if (count < 1 || !ns || !node_offsets)
            throw std::runtime_error("need count >= 1, ns and node_offsets");
        if (nthreads > 0)
            omp_set_num_threads(nthreads);
        node_offsets[0] = 0;
        for (uint64_t i = 0; i < count; ++i) {
            if (ns[i] < 2 || !(avg_deg < static_cast<double>(ns[i] - 1)))
                throw std::runtime_error("every graph needs n >= 2 and avg_deg < n - 1");
            node_offsets[i + 1] = node_offsets[i] + ns[i];
        }
        const uint64_t z = node_offsets[count];
        if (z >= 0xffffffffull)
            throw std::runtime_error("total node count must be < 2^32");
        if (!(exponent > 2.0))
            throw std::runtime_error("exponent must be > 2");
        std::vector<uint64_t> order(count);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return ns[a] > ns[b]; });
        std::vector<std::vector<uint64_t>> ptrs(count);
        std::vector<std::vector<uint32_t>> cols(count);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t k = 0; k < static_cast<int64_t>(count); ++k) {
            const uint64_t i = order[k];
            rhg_rows(ns[i], avg_deg, exponent, seed + i, ptrs[i], cols[i]);
        }
        std::vector<uint64_t> arc_off(count + 1, 0);
        for (uint64_t i = 0; i < count; ++i)
            arc_off[i + 1] = arc_off[i] + cols[i].size();
        Csr cs;
        cs.z = z;
        cs.arcs = arc_off[count];
        cs.in_ptr = static_cast<uint64_t *>(malloc((z + 1) * sizeof(uint64_t)));
        cs.in_col = static_cast<uint32_t *>(malloc(std::max<uint64_t>(cs.arcs, 1) * sizeof(uint32_t)));
        cs.outdeg = static_cast<uint32_t *>(malloc(z * sizeof(uint32_t)));
        if (!cs.in_ptr || !cs.in_col || !cs.outdeg)
            throw std::bad_alloc();
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t i = 0; i < static_cast<int64_t>(count); ++i) {
            const uint64_t base = node_offsets[i], ab = arc_off[i], n = ns[i];
            for (uint64_t v = 0; v < n; ++v) {
                cs.in_ptr[base + v] = ab + ptrs[i][v];
                cs.outdeg[base + v] = static_cast<uint32_t>(ptrs[i][v + 1] - ptrs[i][v]);
            }
            for (size_t k = 0; k < cols[i].size(); ++k)
                cs.in_col[ab + k] = static_cast<uint32_t>(base + cols[i][k]);
            std::vector<uint64_t>().swap(ptrs[i]);
            std::vector<uint32_t>().swap(cols[i]);
        }
        cs.in_ptr[z] = cs.arcs;
        export_csr(cs, out);
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    }
}

} // extern "C"
