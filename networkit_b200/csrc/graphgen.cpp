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

} // namespace

extern "C" {

struct nkgen_csr {
    uint64_t z;
    uint64_t arcs;
    uint64_t *in_ptr;
    uint32_t *in_col;
    uint32_t *outdeg;
    double *w;
};

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

} // extern "C"
