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
// Per-problem state is dense: one slot of z entries per resident warp, holding
//   r, p     residual and value (the reference's unordered_map pair),
//   stamp    the problem's epoch. An entry is in the map iff its stamp equals
//            the epoch, so slots are never cleared between problems,
//   touched  the support in first-touch order,
//   queue    the FIFO ring (z entries: with non-negative weights a node is
//            queued at most once at a time).
// That is 28 bytes per node per slot; the number of slots follows a memory
// budget.
//
// PageRankNibble's sweep (bestSweepSet) then runs as:
//   (1) per support node, in the push kernel while the slot is live: its key
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
    // slots
    uint64_t slots;
    double *r, *p;
    uint32_t *stamp, *touched, *queue, *epoch;
    // results
    uint64_t pool_cap;
    unsigned long long *pool_used;
    unsigned long long *next;
    uint32_t *out_node;
    double *out_p;
    uint64_t *out_key;
    double *out_dcut;
    uint64_t *sup_off, *sup_cnt, *pushes;
    int *err;  // 1: queue overflow (negative weights), 2: push limit reached
    int nibble;
};

// One warp = one slot; the warp takes problems from a global counter until
// none are left.
template <bool WEIGHTED>
__global__ void __launch_bounds__(kLocalThreads) local_push(PushArgs a) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t slot = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    if (slot >= a.slots)
        return;
    const uint64_t z = a.z;
    double *__restrict__ r = a.r + slot * z;
    double *__restrict__ p = a.p + slot * z;
    uint32_t *__restrict__ stamp = a.stamp + slot * z;
    uint32_t *__restrict__ touched = a.touched + slot * z;
    uint32_t *__restrict__ queue = a.queue + slot * z;
    const uint64_t *__restrict__ ptr = a.ptr;
    const uint32_t *__restrict__ col = a.col;
    const double *__restrict__ vol = a.vol;
    uint32_t epoch = a.epoch[slot];
    const double oma = 1.0 - a.alpha;
    const double eps = a.eps;
    const unsigned lt = lanemask_lt();

    for (;;) {
        unsigned long long k = 0;
        if (lane == 0)
            k = atomicAdd(a.next, 1ull);
        k = __shfl_sync(kFull, k, 0);
        if (k >= a.problems)
            break;
        ++epoch;
        // Seeds: ascending, each with residual 1/|seeds|, queued in order.
        const uint64_t s0 = a.seed_ptr[k], s1 = a.seed_ptr[k + 1];
        const double init = 1.0 / static_cast<double>(s1 - s0);
        for (uint64_t i = s0 + lane; i < s1; i += 32) {
            const uint32_t v = a.seeds[i];
            stamp[v] = epoch;
            r[v] = init;
            p[v] = 0.0;
            touched[i - s0] = v;
            queue[i - s0] = v;
        }
        uint64_t T = s1 - s0, head = 0, tail = s1 - s0, npush = 0;
        int fail = 0;
        __syncwarp();

        while (head < tail) {
            if (npush >= a.max_pushes) {
                fail = 2;
                break;
            }
            const uint32_t u = queue[head % z];
            ++head;
            const double res = r[u];
            const double pu = p[u];
            const double volume = vol[u];
            const uint64_t b = ptr[u], e = ptr[u + 1];
            const double a1 = __dmul_rn(oma, res);  // (1.0 - alpha) * res
            const double d2 = __dmul_rn(2.0, volume);
            for (uint64_t base = b; base < e; base += 32) {
                const uint64_t q = base + lane;
                const bool act = q < e;
                uint32_t v = kNone;
                double mass = 0.0, volv = 0.0, rv = 0.0;
                bool fresh = false;
                if (act) {
                    v = col[q];
                    const double wk = WEIGHTED ? a.w[q] : 1.0;
                    mass = __ddiv_rn(__dmul_rn(a1, wk), d2);
                    volv = vol[v];
                    const uint32_t st = stamp[v];
                    const double rraw = r[v];
                    fresh = st != epoch;
                    rv = fresh ? 0.0 : rraw;
                }
                const unsigned peers = __match_any_sync(kFull, v);
                const bool dup = act && __popc(peers) > 1;
                if (__any_sync(kFull, dup)) {
                    // A node twice in this chunk (a multi-edge): lane 0 takes
                    // the chunk in row order.
                    __syncwarp();
                    if (lane == 0) {
                        const uint64_t qe = min(e, base + 32);
                        for (uint64_t qq = base; qq < qe; ++qq) {
                            const uint32_t v2 = col[qq];
                            const double w2 = WEIGHTED ? a.w[qq] : 1.0;
                            const double m2 = __ddiv_rn(__dmul_rn(a1, w2), d2);
                            const double vv = vol[v2];
                            const bool fr = stamp[v2] != epoch;
                            const double old = fr ? 0.0 : r[v2];
                            if (fr) {
                                stamp[v2] = epoch;
                                p[v2] = 0.0;
                                touched[T++] = v2;
                            }
                            if (old < __dmul_rn(vv, eps) && __dadd_rn(old, m2) >= __dmul_rn(eps, vv)) {
                                queue[tail % z] = v2;
                                ++tail;
                            }
                            r[v2] = __dadd_rn(old, m2);
                        }
                    }
                    T = __shfl_sync(kFull, T, 0);
                    tail = __shfl_sync(kFull, tail, 0);
                } else {
                    bool cond = false;
                    if (act) {
                        cond = (rv < __dmul_rn(volv, eps)) &&
                               (__dadd_rn(rv, mass) >= __dmul_rn(eps, volv));
                        r[v] = __dadd_rn(rv, mass);
                    }
                    const unsigned fm = __ballot_sync(kFull, act && fresh);
                    if (act && fresh) {
                        stamp[v] = epoch;
                        p[v] = 0.0;
                        touched[T + __popc(fm & lt)] = v;
                    }
                    T += __popc(fm);
                    const unsigned cm = __ballot_sync(kFull, cond);
                    if (cond)
                        queue[(tail + __popc(cm & lt)) % z] = v;
                    tail += __popc(cm);
                }
                __syncwarp();
            }
            // prRes[u] = (p + alpha*res, (1-alpha)*res/2); queue u again while
            // r/vol >= eps. A self-loop's share added above is overwritten.
            const double ru = __ddiv_rn(__dmul_rn(oma, res), 2.0);
            if (lane == 0) {
                p[u] = __dadd_rn(pu, __dmul_rn(a.alpha, res));
                r[u] = ru;
            }
            if (__ddiv_rn(ru, volume) >= eps) {
                if (lane == 0)
                    queue[tail % z] = u;
                ++tail;
            }
            ++npush;
            if (tail - head > z) {
                fail = 1;
                break;
            }
            __syncwarp();
        }
        __syncwarp();

        unsigned long long off = 0;
        if (lane == 0) {
            off = atomicAdd(a.pool_used, static_cast<unsigned long long>(T));
            a.sup_off[k] = off;
            a.sup_cnt[k] = T;
            a.pushes[k] = npush;
            if (fail)
                atomicMax(a.err, fail);
        }
        off = __shfl_sync(kFull, off, 0);
        if (fail || off + T > a.pool_cap)
            continue;  // the host sees the error or the shortfall and re-runs
        for (uint64_t i = lane; i < T; i += 32) {
            const uint32_t v = touched[i];
            const double pv = p[v];
            a.out_node[off + i] = v;
            a.out_p[off + i] = pv;
            if (a.nibble) {
                const uint64_t kv = order_bits(pv / vol[v]);
                a.out_key[off + i] = kv;
                // Cut change of v: +w for a neighbour outside the prefix that
                // ends before v (v itself included), -w inside; row order.
                double acc = 0.0;
                const uint64_t eb = ptr[v], ee = ptr[v + 1];
                for (uint64_t qq = eb; qq < ee; ++qq) {
                    const uint32_t x = col[qq];
                    const double wq = WEIGHTED ? a.w[qq] : 1.0;
                    bool before = false;
                    if (x != v && stamp[x] == epoch) {
                        const uint64_t kx = order_bits(p[x] / vol[x]);
                        before = kx > kv || (kx == kv && x < v);
                    }
                    acc = before ? __dsub_rn(acc, wq) : __dadd_rn(acc, wq);
                }
                a.out_dcut[off + i] = acc;
            }
        }
        __syncwarp();
    }
    if (lane == 0)
        a.epoch[slot] = epoch;
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
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    uint64_t z = 0, arcs = 0, n_nodes = 0;
    bool weighted = false;
    double total_volume = 0.0;  // 2 * totalEdgeWeight() (PageRankNibble.cpp:46)
    std::vector<uint8_t> exists;
    DeviceArray<uint64_t> ptr;
    DeviceArray<uint32_t> col;
    DeviceArray<double> w, vol, wsum;
    // per-problem slots
    uint64_t budget = 0, slots = 0, epochs_used = 0;
    DeviceArray<double> r, p;
    DeviceArray<uint32_t> stamp, touched, queue, epoch;
    // result pool
    uint64_t pool_cap = 0, nibble_cap = 0;
    DeviceArray<uint32_t> out_node, node_sorted, ord_node, ord_sweep, set_node, set_sorted, iota;
    DeviceArray<double> out_p, out_dcut;
    DeviceArray<uint64_t> out_key, key_sorted;
    DeviceArray<unsigned long long> counters;  // pool_used, next
    DeviceArray<int> err;
    DeviceArray<uint8_t> sort_tmp;
    // last run
    uint64_t problems = 0;
    bool nibble = false;
    std::vector<uint64_t> sup_off, sup_cnt, set_cnt;
    DeviceArray<uint64_t> d_sup_off, d_sup_cnt, d_sup_end, d_set_cnt, d_set_end, d_pushes;
};

namespace {

constexpr uint64_t kSlotBytesPerNode = 8 + 8 + 4 + 4 + 4;

void ensure_slots(nkg_local *h, uint64_t want) {
    uint64_t fit = std::max<uint64_t>(1, h->budget / (kSlotBytesPerNode * h->z));
    want = std::max<uint64_t>(1, std::min(want, fit));
    if (h->slots >= want)
        return;
    const size_t n = static_cast<size_t>(want * h->z);
    h->r.reset(), h->p.reset(), h->stamp.reset(), h->touched.reset(), h->queue.reset();
    h->slots = 0;
    h->r.alloc(n);
    h->p.alloc(n);
    h->stamp.alloc(n);
    h->touched.alloc(n);
    h->queue.alloc(n);
    h->epoch.alloc(want);
    NKG_CUDA(cudaMemsetAsync(h->stamp.get(), 0, n * 4, h->stream));
    NKG_CUDA(cudaMemsetAsync(h->epoch.get(), 0, want * 4, h->stream));
    h->slots = want;
    h->epochs_used = 0;
}

// Result pool of `cap` entries; the sweep arrays only when `nibble`.
void ensure_pool(nkg_local *h, uint64_t cap, bool nibble) {
    if (h->pool_cap < cap) {
        h->out_node.alloc(cap);
        h->node_sorted.alloc(cap);
        h->ord_node.alloc(cap);
        h->iota.alloc(cap);
        h->out_p.alloc(cap);
        local_iota<<<ceil_div(cap, 256), 256, 0, h->stream>>>(h->iota.get(), cap);
        NKG_CUDA(cudaGetLastError());
        h->pool_cap = cap;
    }
    if (nibble && h->nibble_cap < h->pool_cap) {
        const uint64_t c = h->pool_cap;
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
    ensure_slots(h, std::min<uint64_t>(problems, static_cast<uint64_t>(sms) * 16));
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
    if (!h->counters)
        h->counters.alloc(2);
    if (!h->err)
        h->err.alloc(1);
    ensure_pool(h, std::max<uint64_t>(h->pool_cap, std::max<uint64_t>(1 << 20, problems * 256)),
                nibble);

    uint64_t launches = 0, reruns = 0, used = 0;
    NKG_CUDA(cudaEventRecord(h->ev0, s));
    for (;;) {
        // A slot's epoch grows by one per problem it takes; restart the
        // stamps before any could wrap.
        if (h->epochs_used + problems >= 0xfffffff0ull) {
            NKG_CUDA(cudaMemsetAsync(h->stamp.get(), 0, h->slots * h->z * 4, s));
            NKG_CUDA(cudaMemsetAsync(h->epoch.get(), 0, h->slots * 4, s));
            h->epochs_used = 0;
        }
        h->epochs_used += problems;
        NKG_CUDA(cudaMemsetAsync(h->counters.get(), 0, 2 * sizeof(unsigned long long), s));
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
        a.slots = h->slots;
        a.r = h->r.get();
        a.p = h->p.get();
        a.stamp = h->stamp.get();
        a.touched = h->touched.get();
        a.queue = h->queue.get();
        a.epoch = h->epoch.get();
        a.pool_cap = h->pool_cap;
        a.pool_used = h->counters.get();
        a.next = h->counters.get() + 1;
        a.out_node = h->out_node.get();
        a.out_p = h->out_p.get();
        a.out_key = h->out_key.get();
        a.out_dcut = h->out_dcut.get();
        a.sup_off = h->d_sup_off.get();
        a.sup_cnt = h->d_sup_cnt.get();
        a.pushes = h->d_pushes.get();
        a.err = h->err.get();
        a.nibble = nibble ? 1 : 0;
        const unsigned blocks = ceil_div(h->slots * 32, kLocalThreads);
        if (h->weighted)
            local_push<true><<<blocks, kLocalThreads, 0, s>>>(a);
        else
            local_push<false><<<blocks, kLocalThreads, 0, s>>>(a);
        NKG_CUDA(cudaGetLastError());
        ++launches;
        const int e = read_scalar(h->err.get(), s);
        if (e == 1)
            throw Error(NKG_ERR_INVALID_ARG,
                        "push queue overflow: a node was queued twice (negative weights?)");
        if (e == 2)
            throw Error(NKG_ERR_TIMEOUT, "push limit reached before the residuals fell below epsilon");
        used = read_scalar(h->counters.get(), s);
        if (used <= h->pool_cap)
            break;
        ensure_pool(h, used + used / 8, nibble);
        ++reruns;
    }
    NKG_CUDA(cudaEventRecord(h->ev1, s));
    require(used <= static_cast<uint64_t>(INT_MAX),
            "the supports of one call exceed 2^31 entries; pass fewer seed sets per call");
    const int items = static_cast<int>(used);
    const int segs = static_cast<int>(problems);
    require(problems <= static_cast<uint64_t>(INT_MAX), "too many problems in one call");
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
    std::vector<uint64_t> pushes(problems);
    NKG_CUDA(cudaMemcpyAsync(h->sup_off.data(), h->d_sup_off.get(), problems * 8,
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaMemcpyAsync(h->sup_cnt.data(), h->d_sup_cnt.get(), problems * 8,
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaMemcpyAsync(pushes.data(), h->d_pushes.get(), problems * 8,
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
        for (uint64_t x : pushes)
            st->pushes += x;
        st->support = used;
        st->slots = h->slots;
        st->reruns = reruns;
        st->ms_push = elapsed(h->ev0, h->ev1);
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
        NKG_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        NKG_CUDA(cudaEventCreate(&h->ev0));
        NKG_CUDA(cudaEventCreate(&h->ev1));
        NKG_CUDA(cudaEventCreate(&h->ev2));
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
    cudaStream_t s = h->stream;
    delete h;
    if (s)
        cudaStreamDestroy(s);
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
