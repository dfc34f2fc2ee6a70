// Local (seeded) PageRank: ApproximatePageRank (scd/ApproximatePageRank.cpp:18-55)
// and PageRankNibble (scd/PageRankNibble.cpp:28-89), many seed sets per call.
//
// The reference's push loop is a FIFO queue, and its order fixes every bit of
// the result: which neighbour crosses the threshold first, and in which order
// mass is added to each residual. That order is kept exactly. One warp runs
// one problem (a seed set) in the reference's order, its 32 lanes taking 32
// neighbours of the pushed node at a time. Problems run side by side, one per
// warp, so a batch of seeds fills the GPU where the reference's
// SelectiveCommunityDetector::run takes the seeds one after another
// (SelectiveCommunityDetector.cpp:15-23).
//
// Per-problem state is a hash map per warp, the reference's unordered_map
// made compact: open addressing with linear probing, 32-byte entries (node
// tagged with the problem's epoch, residual, value), taken from a
// bump-allocated pool and doubled whenever it is half full. Its
// footprint follows the support, not the graph, so the maps of thousands of
// problems in flight stay in L2. Tags carry the problem's epoch, so a warp
// reuses its table for the next problem without clearing it. The FIFO queue
// is a ring of entry indices beside the table.
//
// PageRankNibble's sweep (bestSweepSet) then runs as:
//   (1) per support node, in the push kernel while the map is live: its key
//       p/vol as an order-preserving integer, and its cut change
//       dcut = sum over its row of (+w, or -w for a neighbour that precedes it
//       in the sweep order), summed in row order;
//   (2) two stable segmented radix sorts of the supports: ascending node id,
//       then descending key. Ties in p/vol therefore go to the smaller id; the
//       reference's unstable std::sort leaves tie order open;
//   (3) one warp per problem scans dcut and the row weight sums in sweep
//       order and keeps the first strict minimum of the conductance.
// Cut and volume are sums of integers on unweighted graphs (the graphs
// PageRankNibble is documented for), so the scan is exact in any order. On
// weighted graphs they are rounded in a different order than the reference's
// one running sum.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <climits>
#include <memory>
#include <vector>

#include "host.hpp"

using namespace nkg;

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kLocalThreads = 256;  // 8 warps (8 problems) per CTA

// Order-preserving map of a double onto uint64 (sign-magnitude to offset
// binary): numeric order, -0 before +0, NaNs at the ends. Sorting these
// integers sorts the doubles.
__device__ __forceinline__ uint64_t order_bits(double d) {
    const uint64_t u = static_cast<uint64_t>(__double_as_longlong(d));
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// weightedDegree(u, true) and the plain row weight sum of every row, each
// summed sequentially in row order (Graph.cpp:427-453; PageRankNibble.cpp:58-65).
template <bool WEIGHTED>
__global__ void local_volumes(uint64_t z, const uint64_t *__restrict__ ptr,
                              const uint32_t *__restrict__ col, const double *__restrict__ w,
                              double *__restrict__ vol, double *__restrict__ wsum) {
    const uint64_t u = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (u >= z)
        return;
    const uint64_t b = ptr[u], e = ptr[u + 1];
    if (WEIGHTED) {
        double s = 0.0, t = 0.0;
        for (uint64_t k = b; k < e; ++k) {
            const double wk = w[k];
            s = __dadd_rn(s, (col[k] == u) ? __dmul_rn(2.0, wk) : wk);
            t = __dadd_rn(t, wk);
        }
        vol[u] = s;
        wsum[u] = t;
    } else {
        uint64_t loops = 0;
        for (uint64_t k = b; k < e; ++k)
            loops += (col[k] == u);
        vol[u] = static_cast<double>(e - b + loops);
        wsum[u] = static_cast<double>(e - b);
    }
}

// One entry of a problem's map (the reference's unordered_map<node,
// pair<double, double>>), 32 bytes: the node tagged with the problem's epoch
// (an entry with another epoch is empty for this problem), residual r, value
// p and, during a rehash, the entry's index in the new table.
struct __align__(32) MapEntry {
    unsigned long long tag;
    double r, p;
    uint32_t fwd, pad;
};

struct PushArgs {
    const uint64_t *ptr;
    const uint32_t *col;
    const double *w;
    const double *vol;
    uint64_t z;
    double alpha, eps;
    uint64_t max_pushes;
    uint64_t problems;
    const uint64_t *seed_ptr;
    const uint32_t *seeds;
    uint32_t epoch_base;  // problem k runs with epoch epoch_base + k + 1
    uint32_t init_cap;    // first table size of a warp (power of two)
    // Table pool: a region of `cap` entries, `cap` support indices and a FIFO
    // ring of `cap` entry indices, handed out by a bump counter; a warp keeps
    // its last region for its next problem and takes a twice larger one when
    // the table is half full or the ring is full.
    MapEntry *ent_pool;
    uint32_t *idx_pool, *ring_pool;
    uint64_t pool_cap;
    unsigned long long *pool_used;
    unsigned long long *next;
    // results
    uint64_t out_cap;
    unsigned long long *out_used;
    uint32_t *out_node;
    double *out_p;
    uint64_t *out_key;
    double *out_dcut;
    uint64_t *sup_off, *sup_cnt, *pushes, *visits;
    int *err;  // 2: push limit reached, 3: table pool exhausted, 4: table too large
    int nibble;
};

__device__ __forceinline__ uint32_t map_home(uint32_t v, uint32_t bits) {
    return (v * 2654435769u) >> (32 - bits);  // Fibonacci hashing
}

// Index of v's entry in the table, or kNone if v has none and !insert.
// With insert, an absent v gets an entry (r = p = 0) and
// `fresh` is set. Lanes of one warp may insert distinct nodes at once: the
// claim of an empty entry is a compare-and-swap of its tag. Returns kNone - 1
// if the table is full (never at the load factor kept, 1/2). The tag and the
// residual come in one 16-byte load from L2 (r_out: v's residual, 0 when
// fresh).
__device__ __forceinline__ uint32_t map_find(MapEntry *tab, uint32_t cap, uint32_t bits,
                                             uint32_t epoch, uint32_t v, bool insert,
                                             bool &fresh, double &r_out) {
    const unsigned long long tag = (static_cast<unsigned long long>(epoch) << 32) | v;
    uint32_t h = map_home(v, bits);
    fresh = false;
    r_out = 0.0;
    for (uint32_t i = 0; i < cap; ++i) {
        const double2 tr = __ldcg(reinterpret_cast<const double2 *>(&tab[h]));
        const unsigned long long t = static_cast<unsigned long long>(__double_as_longlong(tr.x));
        if (t == tag) {
            r_out = tr.y;
            return h;
        }
        if (static_cast<uint32_t>(t >> 32) != epoch) {
            if (!insert)
                return kNone;
            const unsigned long long old = atomicCAS(&tab[h].tag, t, tag);
            if (old == t) {
                tab[h].r = 0.0;
                tab[h].p = 0.0;
                fresh = true;
                return h;
            }
            if (old == tag) {
                r_out = __ldcg(&tab[h].r);
                return h;
            }
        }
        h = (h + 1) & (cap - 1);
    }
    return kNone - 1;
}

// The warp's table: entries, support list (entry indices in first-touch
// order), FIFO ring (entry indices; positions are counters modulo cap), size.
// The FIFO is a ring, not a list through the entries: a node can be queued
// twice, as in the reference, because the test that queues a node again
// after its push (r / vol >= eps) and the test that queues a neighbour
// (r < vol * eps) round differently.
struct WarpMap {
    MapEntry *tab;
    uint32_t *tl, *ring;
    uint32_t cap, bits;
};

// Move the warp's table into a fresh region of at least `need_cap` entries
// (a power of two): every entry of this epoch is inserted anew, the support
// list rewritten, the queued entries [qh, qt) copied in order to the new
// ring's front and `cur` translated through `fwd`. Returns 0, 3 if the pool
// is exhausted, 4 if the table would pass 2^31 entries.
__device__ int map_grow(const PushArgs &a, WarpMap &m, uint64_t need_cap, uint32_t epoch,
                        uint64_t T, uint64_t &qh, uint64_t &qt, uint32_t &cur, unsigned lane) {
    if (need_cap > (1ull << 31))
        return 4;
    uint32_t ncap = m.cap, nbits = m.bits;
    while (ncap < need_cap) {
        ncap <<= 1;
        ++nbits;
    }
    unsigned long long off = 0;
    if (lane == 0)
        off = atomicAdd(a.pool_used, static_cast<unsigned long long>(ncap));
    off = __shfl_sync(kFull, off, 0);
    if (off + ncap > a.pool_cap)
        return 3;
    WarpMap n{a.ent_pool + off, a.idx_pool + off, a.ring_pool + off, ncap, nbits};
    if (T) {
        for (uint64_t i = lane; i < T; i += 32) {
            const uint32_t oi = m.tl[i];
            const MapEntry e = m.tab[oi];
            bool fresh;
            double rr;
            const uint32_t nh = map_find(n.tab, n.cap, n.bits, epoch,
                                         static_cast<uint32_t>(e.tag), true, fresh, rr);
            n.tab[nh].r = e.r;
            n.tab[nh].p = e.p;
            m.tab[oi].fwd = nh;
            n.tl[i] = nh;
        }
        __syncwarp();
        const uint64_t len = qt - qh;
        for (uint64_t i = lane; i < len; i += 32)
            n.ring[i] = m.tab[m.ring[(qh + i) & (m.cap - 1)]].fwd;
        if (cur != kNone)
            cur = m.tab[cur].fwd;
        qh = 0;
        qt = len;
        __syncwarp();
    }
    m = n;
    return 0;
}

// Rows longer than this have their nibble cut change counted by the whole
// warp (unweighted graphs).
constexpr uint64_t kCutWarpRow = 64;

// One warp runs one problem at a time, taking problems from a global counter
// until none are left.
template <bool WEIGHTED>
__global__ void __launch_bounds__(kLocalThreads) local_push(PushArgs a) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t *__restrict__ ptr = a.ptr;
    const uint32_t *__restrict__ col = a.col;
    const double *__restrict__ vol = a.vol;
    const double oma = 1.0 - a.alpha;
    const double eps = a.eps;
    const unsigned lt = lanemask_lt();
    WarpMap m{nullptr, nullptr, nullptr, 0, 0};

    for (;;) {
        unsigned long long k = 0;
        if (lane == 0)
            k = atomicAdd(a.next, 1ull);
        k = __shfl_sync(kFull, k, 0);
        if (k >= a.problems)
            break;
        const uint32_t epoch = a.epoch_base + static_cast<uint32_t>(k) + 1;
        const uint64_t s0 = a.seed_ptr[k], s1 = a.seed_ptr[k + 1], ns = s1 - s0;
        uint64_t T = 0, npush = 0, qh = 0, qt = 0, nvisit = 0;
        uint32_t uidx = kNone;
        int fail = 0;
        // A table of at least init_cap entries, at least 4 per seed.
        const uint64_t want = max(static_cast<uint64_t>(a.init_cap), 4 * ns);
        if (m.cap < want) {
            if (m.tab == nullptr) {
                m.cap = 1;
                m.bits = 0;
            }
            fail = map_grow(a, m, want, epoch, 0, qh, qt, uidx, lane);
        }
        if (!fail) {
            // Seeds: ascending, residual 1/|seeds| each, queued in order.
            const double init = 1.0 / static_cast<double>(ns);
            for (uint64_t i = lane; i < ns; i += 32) {
                bool fresh;
                double rr;
                const uint32_t h = map_find(m.tab, m.cap, m.bits, epoch, a.seeds[s0 + i], true,
                                            fresh, rr);
                m.tab[h].r = init;
                m.tl[i] = h;
                m.ring[i] = h;
            }
            T = ns;
            qt = ns;
            __syncwarp();
        }

        while (!fail && qh < qt) {
            if (npush >= a.max_pushes) {
                fail = 2;
                break;
            }
            uidx = m.ring[qh & (m.cap - 1)];
            ++qh;
            const MapEntry ue = m.tab[uidx];
            const uint32_t u = static_cast<uint32_t>(ue.tag);
            const double volume = vol[u];
            const uint64_t b = ptr[u], e = ptr[u + 1];
            const double res = ue.r;
            const double a1 = __dmul_rn(oma, res);  // (1.0 - alpha) * res
            const double d2 = __dmul_rn(2.0, volume);
            nvisit += e - b;
            for (uint64_t base = b; base < e; base += 32) {
                // Room for 32 new entries at load <= 1/2 and 32 queued ones.
                if (T + 32 > m.cap / 2 || qt - qh + 32 > m.cap) {
                    fail = map_grow(a, m, 2ull * m.cap, epoch, T, qh, qt, uidx, lane);
                    if (fail)
                        break;
                }
                const uint64_t q = base + lane;
                const bool act = q < e;
                uint32_t v = kNone, h = 0;
                double mass = 0.0, volv = 0.0, rv = 0.0;
                bool fresh = false;
                if (act) {
                    v = col[q];
                    const double wk = WEIGHTED ? a.w[q] : 1.0;
                    mass = __ddiv_rn(__dmul_rn(a1, wk), d2);
                    volv = vol[v];
                }
                const unsigned peers = __match_any_sync(kFull, v);
                const bool dup = act && __popc(peers) > 1;
                if (__any_sync(kFull, dup)) {
                    // A node twice in this chunk (a multi-edge): lane 0 takes
                    // the chunk in row order.
                    if (lane == 0) {
                        const uint64_t qe = min(e, base + 32);
                        for (uint64_t qq = base; qq < qe; ++qq) {
                            const uint32_t v2 = col[qq];
                            const double w2 = WEIGHTED ? a.w[qq] : 1.0;
                            const double m2 = __ddiv_rn(__dmul_rn(a1, w2), d2);
                            const double vv = vol[v2];
                            bool fr;
                            double old;
                            const uint32_t h2 = map_find(m.tab, m.cap, m.bits, epoch, v2, true, fr,
                                                         old);
                            if (h2 >= kNone - 1) {
                                fail = 4;
                                break;
                            }
                            if (fr)
                                m.tl[T++] = h2;
                            if (old < __dmul_rn(vv, eps) && __dadd_rn(old, m2) >= __dmul_rn(eps, vv))
                                m.ring[qt++ & (m.cap - 1)] = h2;
                            m.tab[h2].r = __dadd_rn(old, m2);
                        }
                    }
                    T = __shfl_sync(kFull, T, 0);
                    qt = __shfl_sync(kFull, qt, 0);
                    fail = __shfl_sync(kFull, fail, 0);
                    __syncwarp();
                    if (fail)
                        break;
                    continue;
                }
                if (act) {
                    h = map_find(m.tab, m.cap, m.bits, epoch, v, true, fresh, rv);
                    if (h >= kNone - 1)
                        fail = 4;
                }
                if (__any_sync(kFull, fail != 0)) {
                    fail = 4;
                    break;
                }
                bool cond = false;
                if (act) {
                    cond = (rv < __dmul_rn(volv, eps)) &&
                           (__dadd_rn(rv, mass) >= __dmul_rn(eps, volv));
                    m.tab[h].r = __dadd_rn(rv, mass);
                }
                const unsigned fm = __ballot_sync(kFull, fresh);
                if (fresh)
                    m.tl[T + __popc(fm & lt)] = h;
                T += __popc(fm);
                // Queue the crossing lanes in lane (= row) order.
                const unsigned cm = __ballot_sync(kFull, cond);
                if (cond)
                    m.ring[(qt + __popc(cm & lt)) & (m.cap - 1)] = h;
                qt += __popc(cm);
                __syncwarp();
            }
            if (fail)
                break;
            // prRes[u] = (p + alpha*res, (1-alpha)*res/2); queue u again while
            // r/vol >= eps. A self-loop's share added above is overwritten.
            const double ru = __ddiv_rn(__dmul_rn(oma, res), 2.0);
            const bool again = __ddiv_rn(ru, volume) >= eps;
            if (again && qt - qh + 1 > m.cap) {
                fail = map_grow(a, m, 2ull * m.cap, epoch, T, qh, qt, uidx, lane);
                if (fail)
                    break;
            }
            if (lane == 0) {
                m.tab[uidx].p = __dadd_rn(ue.p, __dmul_rn(a.alpha, res));
                m.tab[uidx].r = ru;
                if (again)
                    m.ring[qt & (m.cap - 1)] = uidx;
            }
            qt += again;
            ++npush;
            __syncwarp();
        }
        __syncwarp();

        unsigned long long off = 0;
        if (lane == 0) {
            off = atomicAdd(a.out_used, static_cast<unsigned long long>(T));
            a.sup_off[k] = off;
            a.sup_cnt[k] = T;
            a.pushes[k] = npush;
            a.visits[k] = nvisit;
            if (fail)
                atomicMax(a.err, fail);
        }
        off = __shfl_sync(kFull, off, 0);
        if (fail == 3)
            break;  // no region for this warp; the host grows the pool and re-runs
        if (fail || off + T > a.out_cap)
            continue;  // the host sees the error or the shortfall
        for (uint64_t i = lane; i < T; i += 32) {
            const MapEntry ev = m.tab[m.tl[i]];
            const uint32_t v = static_cast<uint32_t>(ev.tag);
            a.out_node[off + i] = v;
            a.out_p[off + i] = ev.p;
            if (a.nibble) {
                const uint64_t kv = order_bits(__ddiv_rn(ev.p, vol[v]));
                a.out_key[off + i] = kv;
                // Cut change of v: +w for a neighbour outside the prefix that
                // ends before v (v itself included), -w inside; row order.
                // Unweighted rows longer than kCutWarpRow are counted by the
                // whole warp below.
                double acc = 0.0;
                const uint64_t eb = ptr[v], ee = ptr[v + 1];
                if (!WEIGHTED && ee - eb > kCutWarpRow)
                    continue;
                for (uint64_t qq = eb; qq < ee; ++qq) {
                    const uint32_t x = col[qq];
                    const double wq = WEIGHTED ? a.w[qq] : 1.0;
                    bool before = false;
                    if (x != v) {
                        bool fr;
                        double rx;
                        const uint32_t hx = map_find(m.tab, m.cap, m.bits, epoch, x, false, fr, rx);
                        if (hx < kNone - 1) {
                            const uint64_t kx = order_bits(__ddiv_rn(m.tab[hx].p, vol[x]));
                            before = kx > kv || (kx == kv && x < v);
                        }
                    }
                    acc = before ? __dsub_rn(acc, wq) : __dadd_rn(acc, wq);
                }
                a.out_dcut[off + i] = acc;
            }
        }
        __syncwarp();
        if (a.nibble && !WEIGHTED) {
            // The long rows' cut changes, one row at a time across the warp:
            // with unit weights the row-order sum of +-1 is the exact integer
            // (neighbours) - 2 (neighbours before v), whatever the order.
            for (uint64_t base = 0; base < T; base += 32) {
                const uint64_t i = base + lane;
                uint32_t v = 0;
                bool longrow = false;
                if (i < T) {
                    v = static_cast<uint32_t>(m.tab[m.tl[i]].tag);
                    longrow = ptr[v + 1] - ptr[v] > kCutWarpRow;
                }
                unsigned lm = __ballot_sync(kFull, longrow);
                while (lm) {
                    const int src = __ffs(lm) - 1;
                    lm &= lm - 1;
                    const uint32_t vv = __shfl_sync(kFull, v, src);
                    const uint64_t ii = base + static_cast<uint64_t>(src);
                    const uint64_t kv = order_bits(__ddiv_rn(m.tab[m.tl[ii]].p, vol[vv]));
                    const uint64_t eb = ptr[vv], ee = ptr[vv + 1];
                    uint32_t before_cnt = 0;
                    for (uint64_t qq = eb + lane; qq < ee; qq += 32) {
                        const uint32_t x = col[qq];
                        if (x == vv)
                            continue;
                        bool fr;
                        double rx;
                        const uint32_t hx = map_find(m.tab, m.cap, m.bits, epoch, x, false, fr, rx);
                        if (hx < kNone - 1) {
                            const uint64_t kx = order_bits(__ddiv_rn(m.tab[hx].p, vol[x]));
                            before_cnt += (kx > kv || (kx == kv && x < vv)) ? 1u : 0u;
                        }
                    }
                    for (int o = 16; o > 0; o >>= 1)
                        before_cnt += __shfl_xor_sync(kFull, before_cnt, o);
                    if (lane == 0)
                        a.out_dcut[off + ii] =
                            static_cast<double>(ee - eb) - 2.0 * static_cast<double>(before_cnt);
                }
            }
            __syncwarp();
        }
    }
}

// bestSweepSet (PageRankNibble.cpp:48-79) per problem over the support in
// sweep order (ord: pool indices, descending key, ties ascending id):
// cut_i, vol_i = inclusive sums; cond_i = cut_i / min(vol_i, total - vol_i);
// the first strict minimum below DBL_MAX over prefixes smaller than n_nodes.
// Writes the chosen prefix (unsorted) to set_node at the support's offset.
__global__ void __launch_bounds__(kLocalThreads) local_sweep(
    uint64_t problems, const uint64_t *__restrict__ sup_off, const uint64_t *__restrict__ sup_cnt,
    const uint32_t *__restrict__ ord, const uint32_t *__restrict__ out_node,
    const double *__restrict__ out_dcut, const double *__restrict__ wsum, double total_volume,
    uint64_t n_nodes, uint32_t *__restrict__ set_node, uint64_t *__restrict__ set_cnt) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t k = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    if (k >= problems)
        return;
    const uint64_t off = sup_off[k], cnt = sup_cnt[k];
    double cut = 0.0, volume = 0.0;
    double best = 1.79769313486231570815e+308;  // DBL_MAX
    uint64_t best_i = 0;
    for (uint64_t base = 0; base < cnt; base += 32) {
        const uint64_t i = base + lane;
        double d = 0.0, wd = 0.0;
        uint32_t node = 0;
        if (i < cnt) {
            const uint32_t j = ord[off + i];
            node = out_node[j];
            d = out_dcut[j];
            wd = wsum[node];
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double dd = __shfl_up_sync(kFull, d, o);
            const double ww = __shfl_up_sync(kFull, wd, o);
            if (lane >= static_cast<unsigned>(o)) {
                d = __dadd_rn(d, dd);
                wd = __dadd_rn(wd, ww);
            }
        }
        const double c = __dadd_rn(cut, d);
        const double vv = __dadd_rn(volume, wd);
        const double other = __dsub_rn(total_volume, vv);
        const double cond = __ddiv_rn(c, (other < vv) ? other : vv);
        const bool ok = i < cnt && i + 1 < n_nodes && cond < best;
        // First lane holding the smallest qualifying cond.
        double m = ok ? cond : best;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            m = fmin(m, __shfl_xor_sync(kFull, m, o));
        const unsigned hit = __ballot_sync(kFull, ok && cond == m);
        if (hit) {
            best = m;
            best_i = base + __ffs(hit);  // prefix length = index + 1
        }
        cut = __shfl_sync(kFull, c, 31);
        volume = __shfl_sync(kFull, vv, 31);
    }
    for (uint64_t i = lane; i < best_i; i += 32)
        set_node[off + i] = out_node[ord[off + i]];
    if (lane == 0)
        set_cnt[k] = best_i;
}

// Gather per-problem segments (pool order) into problem order.
__global__ void local_gather(uint64_t problems, const uint64_t *__restrict__ seg_off,
                             const uint64_t *__restrict__ seg_cnt, const uint64_t *__restrict__ dst_off,
                             const uint32_t *__restrict__ ord, const uint32_t *__restrict__ node_in,
                             const double *__restrict__ val_in, uint32_t *__restrict__ node_out,
                             double *__restrict__ val_out) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t k = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    if (k >= problems)
        return;
    const uint64_t so = seg_off[k], c = seg_cnt[k], d = dst_off[k];
    for (uint64_t i = lane; i < c; i += 32) {
        const uint32_t j = ord ? ord[so + i] : static_cast<uint32_t>(so + i);
        node_out[d + i] = node_in[j];
        if (val_out)
            val_out[d + i] = val_in[j];
    }
}

__global__ void local_iota(uint32_t *__restrict__ a, uint64_t n) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        a[i] = static_cast<uint32_t>(i);
}

__global__ void local_seg_ends(uint64_t n, const uint64_t *__restrict__ off,
                               const uint64_t *__restrict__ cnt, uint64_t *__restrict__ end) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        end[i] = off[i] + cnt[i];
}

__global__ void local_gather_u64(const uint32_t *__restrict__ idx, const uint64_t *__restrict__ src,
                                 uint64_t *__restrict__ dst, uint64_t n) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        dst[i] = src[idx[i]];
}

}  // namespace

struct nkg_local {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
    uint64_t z = 0, arcs = 0, n_nodes = 0;
    bool weighted = false;
    double total_volume = 0.0;  // 2 * totalEdgeWeight() (PageRankNibble.cpp:46)
    std::vector<uint8_t> exists;
    DeviceArray<uint64_t> ptr;
    DeviceArray<uint32_t> col;
    DeviceArray<double> w, vol, wsum;
    // per-problem maps: the table pool and the epoch counter
    uint64_t budget = 0;
    uint64_t table_cap = 0;       // entries of the table pool
    uint32_t epoch_base = 0;      // epochs below this one are spent
    DeviceArray<MapEntry> ent_pool;
    DeviceArray<uint32_t> idx_pool, ring_pool;
    // result pool
    uint64_t out_cap = 0, nibble_cap = 0;
    DeviceArray<uint32_t> out_node, node_sorted, ord_node, ord_sweep, set_node, set_sorted, iota;
    DeviceArray<double> out_p, out_dcut;
    DeviceArray<uint64_t> out_key, key_sorted;
    DeviceArray<unsigned long long> counters;  // out_used, next problem, table pool used
    DeviceArray<int> err;
    DeviceArray<uint8_t> sort_tmp;
    // last run
    uint64_t problems = 0;
    bool nibble = false;
    std::vector<uint64_t> sup_off, sup_cnt, set_cnt;
    DeviceArray<uint64_t> d_sup_off, d_sup_cnt, d_sup_end, d_set_cnt, d_set_end, d_pushes, d_visits;
    uint64_t table_need = 0;  // table entries the last launch asked for
};

namespace {

constexpr uint32_t kInitCap = 1024;    // first table of a warp: 40 KB

// Table pool of at least `cap` entries (40 bytes each with the support index
// and the ring slot). A new pool holds only zero tags, which match no epoch.
void ensure_tables(nkg_local *h, uint64_t cap) {
    if (h->table_cap >= cap)
        return;
    h->ent_pool.reset();
    h->idx_pool.reset();
    h->ring_pool.reset();
    h->table_cap = 0;
    h->ent_pool.alloc(cap);
    h->idx_pool.alloc(cap);
    h->ring_pool.alloc(cap);
    NKG_CUDA(cudaMemsetAsync(h->ent_pool.get(), 0, cap * sizeof(MapEntry), h->stream));
    h->table_cap = cap;
    h->epoch_base = 0;
}

// Result pool of `cap` entries; the sweep arrays only when `nibble`.
void ensure_out(nkg_local *h, uint64_t cap, bool nibble) {
    if (h->out_cap < cap) {
        h->out_node.alloc(cap);
        h->node_sorted.alloc(cap);
        h->ord_node.alloc(cap);
        h->iota.alloc(cap);
        h->out_p.alloc(cap);
        local_iota<<<ceil_div(cap, 256), 256, 0, h->stream>>>(h->iota.get(), cap);
        NKG_CUDA(cudaGetLastError());
        h->out_cap = cap;
    }
    if (nibble && h->nibble_cap < h->out_cap) {
        const uint64_t c = h->out_cap;
        h->set_node.alloc(c);
        h->set_sorted.alloc(c);
        h->out_key.alloc(c);
        h->key_sorted.alloc(c);
        h->ord_sweep.alloc(c);
        h->out_dcut.alloc(c);
        h->nibble_cap = c;
    }
}

template <typename Fn>
void with_sort_tmp(nkg_local *h, Fn &&fn) {
    size_t bytes = 0;
    NKG_CUDA(fn(nullptr, bytes));
    if (h->sort_tmp.size() < bytes)
        h->sort_tmp.alloc(bytes);
    NKG_CUDA(fn(h->sort_tmp.get(), bytes));
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    NKG_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
}

void run_local(nkg_local *h, double alpha, double eps, uint64_t problems, const uint64_t *seed_ptr,
               const uint32_t *seeds, bool nibble, uint64_t max_pushes, nkg_local_stats *st) {
    cudaStream_t s = h->stream;
    require(problems <= static_cast<uint64_t>(INT_MAX), "too many problems in one call");
    const uint64_t nseeds = seed_ptr[problems];
    require(seed_ptr[0] == 0, "seed_ptr must start at 0");
    for (uint64_t k = 0; k < problems; ++k) {
        require(seed_ptr[k + 1] > seed_ptr[k], "every problem needs at least one seed");
        for (uint64_t i = seed_ptr[k]; i < seed_ptr[k + 1]; ++i) {
            require(seeds[i] < h->z, "seed id >= z");
            require(h->exists.empty() || h->exists[seeds[i]], "seed is a non-existent node");
            require(i == seed_ptr[k] || seeds[i] > seeds[i - 1],
                    "the seeds of a problem must be ascending without duplicates");
        }
    }
    const unsigned sms = num_sms(h->device);
    // Problems in flight: one per resident warp, and as many as the memory
    // budget gives first tables (with room to double twice).
    int ctas_per_sm = 0;
    if (h->weighted)
        NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas_per_sm, local_push<true>,
                                                               kLocalThreads, 0));
    else
        NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas_per_sm, local_push<false>,
                                                               kLocalThreads, 0));
    const uint64_t resident = static_cast<uint64_t>(sms) * std::max(ctas_per_sm, 1) *
                              (kLocalThreads / 32);
    const uint64_t by_budget = h->budget / (4ull * kInitCap * (sizeof(MapEntry) + 8));
    const uint64_t warps =
        std::max<uint64_t>(1, std::min<uint64_t>({problems, resident, by_budget}));
    DeviceArray<uint64_t> d_seed_ptr(problems + 1);
    DeviceArray<uint32_t> d_seeds(nseeds);
    NKG_CUDA(cudaMemcpyAsync(d_seed_ptr.get(), seed_ptr, (problems + 1) * 8, cudaMemcpyHostToDevice, s));
    NKG_CUDA(cudaMemcpyAsync(d_seeds.get(), seeds, nseeds * 4, cudaMemcpyHostToDevice, s));
    h->d_sup_off.alloc(problems);
    h->d_sup_cnt.alloc(problems);
    h->d_sup_end.alloc(problems);
    h->d_set_cnt.alloc(problems);
    h->d_set_end.alloc(problems);
    h->d_pushes.alloc(problems);
    h->d_visits.alloc(problems);
    if (!h->counters)
        h->counters.alloc(3);
    if (!h->err)
        h->err.alloc(1);
    // Tables: what the last call asked for, at least 16 first tables a warp.
    ensure_tables(h, std::max<uint64_t>(warps * kInitCap * 16, h->table_need));
    ensure_out(h, std::max<uint64_t>(h->out_cap, std::max<uint64_t>(1 << 20, problems * 256)),
               nibble);

    uint64_t launches = 0, reruns = 0, used = 0;
    NKG_CUDA(cudaEventRecord(h->ev0, s));
    for (;;) {
        // Every launch takes fresh epochs (a re-run must not see the tags
        // of the failed launch); restart the tags before they could wrap.
        if (static_cast<uint64_t>(h->epoch_base) + problems + 1 >= 0xffffffffull) {
            NKG_CUDA(cudaMemsetAsync(h->ent_pool.get(), 0, h->table_cap * sizeof(MapEntry), s));
            h->epoch_base = 0;
        }
        NKG_CUDA(cudaMemsetAsync(h->counters.get(), 0, 3 * sizeof(unsigned long long), s));
        NKG_CUDA(cudaMemsetAsync(h->err.get(), 0, sizeof(int), s));
        PushArgs a{};
        a.ptr = h->ptr.get();
        a.col = h->col.get();
        a.w = h->w.get();
        a.vol = h->vol.get();
        a.z = h->z;
        a.alpha = alpha;
        a.eps = eps;
        a.max_pushes = max_pushes;
        a.problems = problems;
        a.seed_ptr = d_seed_ptr.get();
        a.seeds = d_seeds.get();
        a.epoch_base = h->epoch_base;
        a.init_cap = kInitCap;
        a.ent_pool = h->ent_pool.get();
        a.idx_pool = h->idx_pool.get();
        a.ring_pool = h->ring_pool.get();
        a.pool_cap = h->table_cap;
        a.pool_used = h->counters.get() + 2;
        a.next = h->counters.get() + 1;
        a.out_cap = h->out_cap;
        a.out_used = h->counters.get();
        a.out_node = h->out_node.get();
        a.out_p = h->out_p.get();
        a.out_key = h->out_key.get();
        a.out_dcut = h->out_dcut.get();
        a.sup_off = h->d_sup_off.get();
        a.sup_cnt = h->d_sup_cnt.get();
        a.pushes = h->d_pushes.get();
        a.visits = h->d_visits.get();
        a.err = h->err.get();
        a.nibble = nibble ? 1 : 0;
        h->epoch_base += static_cast<uint32_t>(problems);
        NKG_CUDA(cudaEventRecord(h->ev3, s));
        const unsigned blocks = ceil_div(warps * 32, kLocalThreads);
        if (h->weighted)
            local_push<true><<<blocks, kLocalThreads, 0, s>>>(a);
        else
            local_push<false><<<blocks, kLocalThreads, 0, s>>>(a);
        NKG_CUDA(cudaGetLastError());
        ++launches;
        const int e = read_scalar(h->err.get(), s);
        if (e == 2)
            throw Error(NKG_ERR_TIMEOUT, "push limit reached before the residuals fell below epsilon");
        if (e == 4)
            throw Error(NKG_ERR_INVALID_ARG, "a problem's support passed 2^30 nodes");
        // The pool counter keeps the entries every warp asked for, granted or
        // not: the next pool holds them all.
        h->table_need = read_scalar(h->counters.get() + 2, s);
        if (e == 3) {
            ensure_tables(h, std::max<uint64_t>(2 * h->table_cap,
                                                h->table_need + h->table_need / 4));
            ++reruns;
            continue;
        }
        used = read_scalar(h->counters.get(), s);
        if (used <= h->out_cap)
            break;
        ensure_out(h, used + used / 8, nibble);
        ++reruns;
    }
    NKG_CUDA(cudaEventRecord(h->ev1, s));
    require(used <= static_cast<uint64_t>(INT_MAX),
            "the supports of one call exceed 2^31 entries; pass fewer seed sets per call");
    const int items = static_cast<int>(used);
    const int segs = static_cast<int>(problems);
    local_seg_ends<<<ceil_div(problems, 256), 256, 0, s>>>(problems, h->d_sup_off.get(),
                                                          h->d_sup_cnt.get(), h->d_sup_end.get());
    ++launches;
    // Support ascending by node id (pool indices in ord_node).
    with_sort_tmp(h, [&](void *tmp, size_t &bytes) {
        return cub::DeviceSegmentedRadixSort::SortPairs(
            tmp, bytes, h->out_node.get(), h->node_sorted.get(), h->iota.get(), h->ord_node.get(),
            items, segs, h->d_sup_off.get(), h->d_sup_end.get(), 0, 32, s);
    });
    launches += 2;
    if (nibble) {
        local_gather_u64<<<ceil_div(used, 256), 256, 0, s>>>(h->ord_node.get(), h->out_key.get(),
                                                             h->key_sorted.get(), used);
        // Stable: equal keys keep ascending node order.
        with_sort_tmp(h, [&](void *tmp, size_t &bytes) {
            return cub::DeviceSegmentedRadixSort::SortPairsDescending(
                tmp, bytes, h->key_sorted.get(), h->out_key.get(), h->ord_node.get(),
                h->ord_sweep.get(), items, segs, h->d_sup_off.get(), h->d_sup_end.get(), 0, 64, s);
        });
        local_sweep<<<ceil_div(problems * 32, kLocalThreads), kLocalThreads, 0, s>>>(
            problems, h->d_sup_off.get(), h->d_sup_cnt.get(), h->ord_sweep.get(),
            h->out_node.get(), h->out_dcut.get(), h->wsum.get(), h->total_volume, h->n_nodes,
            h->set_node.get(), h->d_set_cnt.get());
        local_seg_ends<<<ceil_div(problems, 256), 256, 0, s>>>(
            problems, h->d_sup_off.get(), h->d_set_cnt.get(), h->d_set_end.get());
        with_sort_tmp(h, [&](void *tmp, size_t &bytes) {
            return cub::DeviceSegmentedRadixSort::SortKeys(
                tmp, bytes, h->set_node.get(), h->set_sorted.get(), items, segs,
                h->d_sup_off.get(), h->d_set_end.get(), 0, 32, s);
        });
        NKG_CUDA(cudaGetLastError());
        launches += 7;
    }
    NKG_CUDA(cudaEventRecord(h->ev2, s));
    h->sup_off.resize(problems);
    h->sup_cnt.resize(problems);
    std::vector<uint64_t> pushes(problems), visits(problems);
    NKG_CUDA(cudaMemcpyAsync(h->sup_off.data(), h->d_sup_off.get(), problems * 8,
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaMemcpyAsync(h->sup_cnt.data(), h->d_sup_cnt.get(), problems * 8,
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaMemcpyAsync(pushes.data(), h->d_pushes.get(), problems * 8,
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaMemcpyAsync(visits.data(), h->d_visits.get(), problems * 8,
                             cudaMemcpyDeviceToHost, s));
    if (nibble) {
        h->set_cnt.resize(problems);
        NKG_CUDA(cudaMemcpyAsync(h->set_cnt.data(), h->d_set_cnt.get(), problems * 8,
                                 cudaMemcpyDeviceToHost, s));
    }
    NKG_CUDA(cudaStreamSynchronize(s));
    h->problems = problems;
    h->nibble = nibble;
    if (st) {
        st->pushes = 0;
        st->arc_visits = 0;
        for (uint64_t x : pushes)
            st->pushes += x;
        for (uint64_t x : visits)
            st->arc_visits += x;
        st->table_entries = h->table_need;
        st->support = used;
        st->slots = warps;
        st->reruns = reruns;
        st->ms_push = elapsed(h->ev3, h->ev1);  // the last push launch
        st->ms_total = elapsed(h->ev0, h->ev2);
        st->ms_sweep = st->ms_total - st->ms_push;
        st->kernel_launches = launches;
    }
}

void gather_out(nkg_local *h, const std::vector<uint64_t> &cnt, const uint64_t *d_cnt,
                const uint32_t *ord, const uint32_t *node_in, const double *val_in,
                uint32_t *nodes_out, double *values_out) {
    cudaStream_t s = h->stream;
    std::vector<uint64_t> dst(h->problems);
    uint64_t total = 0;
    for (uint64_t k = 0; k < h->problems; ++k) {
        dst[k] = total;
        total += cnt[k];
    }
    if (total == 0)
        return;
    DeviceArray<uint64_t> d_dst(h->problems);
    DeviceArray<uint32_t> d_nodes(total);
    DeviceArray<double> d_vals(values_out ? total : 0);
    NKG_CUDA(cudaMemcpyAsync(d_dst.get(), dst.data(), h->problems * 8, cudaMemcpyHostToDevice, s));
    local_gather<<<ceil_div(h->problems * 32, 256), 256, 0, s>>>(
        h->problems, h->d_sup_off.get(), d_cnt, d_dst.get(), ord, node_in, val_in, d_nodes.get(),
        values_out ? d_vals.get() : nullptr);
    NKG_CUDA(cudaGetLastError());
    NKG_CUDA(cudaMemcpyAsync(nodes_out, d_nodes.get(), total * 4, cudaMemcpyDeviceToHost, s));
    if (values_out)
        NKG_CUDA(cudaMemcpyAsync(values_out, d_vals.get(), total * 8, cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

extern "C" {

int nkg_local_create(nkg_local **out, uint64_t z, const uint64_t *row_ptr, const uint32_t *col,
                     const double *w, const uint8_t *exists, int directed, int device,
                     uint64_t memory_budget) {
    return guarded([&] {
        require(out != nullptr && row_ptr != nullptr, "NULL argument");
        *out = nullptr;
        require(z >= 1 && z < 0xffffffffull, "z must be in [1, 2^32 - 1)");
        require(row_ptr[0] == 0, "row_ptr must start at 0");
        const uint64_t arcs = row_ptr[z];
        require(arcs < 0xffffffffull, "arc count must be < 2^32 - 1");
        require(arcs == 0 || col != nullptr, "col is NULL");
        uint64_t loops = 0, n_nodes = 0;
        double wsum_edges = 0.0;
        for (uint64_t u = 0; u < z; ++u) {
            require(row_ptr[u + 1] >= row_ptr[u], "row_ptr must be non-decreasing");
            const bool ex = exists == nullptr || exists[u];
            n_nodes += ex;
            require(ex || row_ptr[u + 1] == row_ptr[u], "a non-existent node has arcs");
            for (uint64_t k = row_ptr[u]; k < row_ptr[u + 1]; ++k) {
                const uint32_t v = col[k];
                require(v < z, "neighbour id >= z");
                // With alpha in (0, 1], epsilon > 0 and weights >= 0 the push
                // loop ends: each push moves alpha * r_u >= alpha * eps * vol_u
                // into p, whose total stays <= 1 (Andersen-Chung-Lang).
                require(w == nullptr || w[k] >= 0.0, "weights must be non-negative numbers");
                require(exists == nullptr || exists[v], "an arc ends at a non-existent node");
                loops += (v == u);
                // totalEdgeWeight(): forEdges order (Graph.cpp:860-868,
                // Graph.hpp:1895-1911): rows ascending, arcs in row order,
                // undirected graphs take each edge at its larger endpoint.
                if (w && (directed || u >= v))
                    wsum_edges += w[k];
            }
        }
        const double edges = directed ? static_cast<double>(arcs)
                                      : static_cast<double>((arcs - loops) / 2 + loops);
        int dev = device;
        if (dev < 0)
            NKG_CUDA(cudaGetDevice(&dev));
        DeviceGuard guard(dev);
        std::unique_ptr<nkg_local> h(new nkg_local());
        h->device = dev;
        h->z = z;
        h->arcs = arcs;
        h->n_nodes = n_nodes;
        h->weighted = w != nullptr;
        h->total_volume = (w ? wsum_edges : edges) * 2;
        if (exists)
            h->exists.assign(exists, exists + z);
        h->stream = stream_acquire(h->device);
        NKG_CUDA(cudaEventCreate(&h->ev0));
        NKG_CUDA(cudaEventCreate(&h->ev1));
        NKG_CUDA(cudaEventCreate(&h->ev2));
        NKG_CUDA(cudaEventCreate(&h->ev3));
        cudaStream_t s = h->stream;
        h->ptr.alloc(z + 1);
        h->col.alloc(std::max<uint64_t>(arcs, 1));
        h->vol.alloc(z);
        h->wsum.alloc(z);
        NKG_CUDA(cudaMemcpyAsync(h->ptr.get(), row_ptr, (z + 1) * 8, cudaMemcpyHostToDevice, s));
        if (arcs)
            NKG_CUDA(cudaMemcpyAsync(h->col.get(), col, arcs * 4, cudaMemcpyHostToDevice, s));
        if (w) {
            h->w.alloc(std::max<uint64_t>(arcs, 1));
            if (arcs)
                NKG_CUDA(cudaMemcpyAsync(h->w.get(), w, arcs * 8, cudaMemcpyHostToDevice, s));
            local_volumes<true><<<ceil_div(z, 256), 256, 0, s>>>(z, h->ptr.get(), h->col.get(),
                                                                 h->w.get(), h->vol.get(),
                                                                 h->wsum.get());
        } else {
            local_volumes<false><<<ceil_div(z, 256), 256, 0, s>>>(z, h->ptr.get(), h->col.get(),
                                                                  nullptr, h->vol.get(),
                                                                  h->wsum.get());
        }
        NKG_CUDA(cudaGetLastError());
        size_t free_b = 0, total_b = 0;
        NKG_CUDA(cudaMemGetInfo(&free_b, &total_b));
        h->budget = memory_budget ? memory_budget
                                  : std::min<uint64_t>(free_b / 2, 48ull << 30);
        NKG_CUDA(cudaStreamSynchronize(s));
        *out = h.release();
    });
}

void nkg_local_destroy(nkg_local *h) {
    if (!h)
        return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    if (h->ev0)
        cudaEventDestroy(h->ev0);
    if (h->ev1)
        cudaEventDestroy(h->ev1);
    if (h->ev2)
        cudaEventDestroy(h->ev2);
    if (h->ev3)
        cudaEventDestroy(h->ev3);
    cudaStream_t s = h->stream;
    const int dev = h->device;
    delete h;
    nkg::stream_release(dev, s);
    if (prev >= 0)
        cudaSetDevice(prev);
}

int nkg_local_run(nkg_local *h, double alpha, double epsilon, uint64_t problems,
                  const uint64_t *seed_ptr, const uint32_t *seeds, int flags, uint64_t max_pushes,
                  uint64_t *support_sizes_out, uint64_t *set_sizes_out, nkg_local_stats *stats) {
    return guarded([&] {
        require(h != nullptr && seed_ptr != nullptr, "NULL argument");
        require(problems >= 1, "no problems");
        require(seeds != nullptr, "seeds is NULL");
        require(epsilon > 0.0, "epsilon must be > 0 (the push loop does not end otherwise)");
        require(alpha > 0.0 && alpha <= 1.0,
                "alpha must be in (0, 1] (the push loop need not end otherwise)");
        require((flags & ~NKG_LOCAL_NIBBLE) == 0, "unknown flags");
        DeviceGuard guard(h->device);
        const bool nibble = (flags & NKG_LOCAL_NIBBLE) != 0;
        run_local(h, alpha, epsilon, problems, seed_ptr, seeds, nibble, max_pushes, stats);
        if (support_sizes_out)
            std::copy(h->sup_cnt.begin(), h->sup_cnt.end(), support_sizes_out);
        if (set_sizes_out) {
            require(nibble, "set sizes need NKG_LOCAL_NIBBLE");
            std::copy(h->set_cnt.begin(), h->set_cnt.end(), set_sizes_out);
        }
    });
}

int nkg_local_support(nkg_local *h, uint32_t *nodes_out, double *values_out) {
    return guarded([&] {
        require(h != nullptr && nodes_out != nullptr, "NULL argument");
        if (h->problems == 0)
            throw Error(NKG_ERR_NOT_RUN, "nkg_local_run has not been called");
        DeviceGuard guard(h->device);
        gather_out(h, h->sup_cnt, h->d_sup_cnt.get(), h->ord_node.get(), h->out_node.get(),
                   h->out_p.get(), nodes_out, values_out);
    });
}

int nkg_local_sets(nkg_local *h, uint32_t *nodes_out) {
    return guarded([&] {
        require(h != nullptr && nodes_out != nullptr, "NULL argument");
        if (h->problems == 0 || !h->nibble)
            throw Error(NKG_ERR_NOT_RUN, "no nkg_local_run with NKG_LOCAL_NIBBLE yet");
        DeviceGuard guard(h->device);
        gather_out(h, h->set_cnt, h->d_set_cnt.get(), nullptr, h->set_sorted.get(), nullptr,
                   nodes_out, nullptr);
    });
}

}  // extern "C"
