// Many-graph PageRank: a batch of independent, uneven graphs solved in one
// persistent launch (no reference counterpart; every graph's iteration is
// PageRank.cpp:54-71 with its own n, teleport, residual and stopping test).
//
// The graphs are given as one block-diagonal in-CSR (graph i owns the node
// ids [node_offsets[i], node_offsets[i+1])). Each graph is relabelled by
// in-degree bucket (half-octaves), descending, inside its own id range,
// keeping the id order inside a bucket. With a row-split threshold T, its
// rows longer than T ("long rows", a prefix) are summed by a whole warp
// each; the others sit in SELL-32 slices (32 rows, column-major slots, one
// row per lane; slice length = its longest row's length).
//
// The kernel is persistent and cluster-based: every thread-block cluster of
// C CTAs takes the next graph from a queue ordered by arc count, descending,
// and iterates it to convergence on its own. The cluster's warps take the
// graph's long rows and slices round-robin; one cluster barrier per
// iteration orders the iterate buffers, and the CTAs exchange their residual,
// sum and sink partials through distributed shared memory (double-buffered,
// so every CTA reads all partials and takes the same decision). No grid-wide
// synchronisation exists: clusters never wait on one another. The gathered
// iterate is written during the kernel, so it is read with coherent loads
// after the barrier's acquire (never through the non-coherent path). The
// structure arrays are read through the read-only path with the default L2
// policy: a graph is swept many times in a row, so its arcs stay in L2 when
// it fits.
//
// FP32 iterates stop at tol, at max_iterations, or at the FP32 rounding
// floor: the exact iteration contracts the L1 residual by at least damp per
// sweep (the iteration matrix is column-substochastic), so a residual that
// shrinks by less than 0.9x is rounding noise. FP64 iterates stop like the
// reference (tol or max_iterations only).
//
// The cluster size C, the CTA size and T are chosen by an autotuner that
// times a few fixed sweeps of the whole batch for every candidate.
#include <cooperative_groups.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "host.hpp"
#include "sweep.cuh"

namespace cg = cooperative_groups;

namespace nkg {
namespace {

constexpr unsigned kMaxCluster = 16;  // 16 is above the portable 8: opted in per kernel
// nkg_batch_tuning.variant bits
constexpr uint32_t kVariantUnroll16 = 1;  // 16 slots per batch of gathers (else 8)
constexpr uint32_t kVariantL2Only = 2;    // iterate loads bypass L1

struct BatchParams {
    double damp;
    double tol;
    unsigned long long max_iterations;
    int l2;
    int distribute;
    int normalized;
    int pad;
};

// Per-graph layout for one threshold T.
struct GraphMeta {
    uint32_t base;        // first (relabelled) node id
    uint32_t n;           // nodes
    uint32_t n_long;      // rows longer than T (the first n_long rows)
    uint32_t slice0;      // first slice
    uint32_t slices;      // slices of the other rows
    uint32_t sinks;       // rows without out-arcs
    uint32_t pad[2];
};

template <typename T>
struct BatchArgs {
    const GraphMeta *__restrict__ meta;
    const uint32_t *__restrict__ order;      // queue position -> graph
    const uint32_t *__restrict__ row_ptr;    // relabelled in-CSR (long rows)
    const uint32_t *__restrict__ col;
    const uint32_t *__restrict__ slice_off;  // slots / 32, per slice (+1)
    const uint32_t *__restrict__ col_sell;   // padding -> zero entry `total`
    const uint32_t *__restrict__ degc;       // out-degree count
    const uint32_t *__restrict__ perm;       // relabelled -> caller id
    T *y0;                                    // iterate buffers (total + 1 each)
    T *y1;
    double *out;                              // scores, caller ids
    unsigned long long *iterations;           // per graph
    double *residual;                         // per graph
    unsigned long long *times;                // per graph: start and end (global timer, ns)
    unsigned int *queue;                      // next queue position
    unsigned int *floor_stops;                // graphs stopped at the FP32 floor
    const BatchParams *prm;
    uint32_t count;
    uint32_t total;
};

struct ClusterShared {
    double part[2][3];     // this CTA's residual / sum / sink partials (double-buffered)
    double s_red[32];
    uint32_t graph;
    int done;
    double sink_coef, sumx, sink, res;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Coherent loads of the iterate (it is written during the kernel): through
// L1 (CG = false) or L2 only (CG = true).
template <bool CG>
__device__ __forceinline__ float ld_iter(const float *p) {
    if (CG)
        return __ldcg(p);
    return *p;
}
template <bool CG>
__device__ __forceinline__ double ld_iter(const double *p) {
    if (CG)
        return __ldcg(p);
    return *p;
}

// Row r of graph (tele, sink_coef): the update of PageRank.cpp:64-65 in gather
// form (y = x/deg for rows with out-arcs, x for sinks), accumulating the
// residual, the sum and the sink mass of the new iterate.
template <typename T, bool CG>
__device__ __forceinline__ void batch_finish(const BatchArgs<T> &a, const T *yin, T *yout,
                                             uint32_t r, T acc, T damp, T tele, T sink_coef,
                                             bool distribute, bool l2, double &res, double &sumx,
                                             double &sink) {
    const uint32_t dc = a.degc[r];
    if (distribute)
        acc = t_add(acc, sink_coef);
    const T x = t_add(t_mul(acc, damp), tele);
    const T yo = ld_iter<CG>(yin + r);
    const T xo = dc ? t_mul(yo, static_cast<T>(dc)) : yo;
    const double d = static_cast<double>(xo) - static_cast<double>(x);
    res += l2 ? d * d : fabs(d);
    sumx += static_cast<double>(x);
    if (dc) {
        yout[r] = x / static_cast<T>(dc);
    } else {
        sink += static_cast<double>(x);
        yout[r] = x;
    }
}

template <typename T, int THREADS, int UNROLL, bool CG>
__global__ void __launch_bounds__(THREADS, UNROLL > 8 ? 512 / THREADS : sizeof(T) > 4 ? 1024 / THREADS : 1280 / THREADS)
    batch_kernel(BatchArgs<T> a) {
    __shared__ ClusterShared sh;
    cg::cluster_group cluster = cg::this_cluster();
    const unsigned crank = cluster.block_rank();
    const unsigned csize = cluster.num_blocks();
    const int lane = threadIdx.x & 31;
    const uint32_t wpc = THREADS / 32;
    const uint32_t cw = crank * wpc + (threadIdx.x >> 5);  // warp index in the cluster
    const uint32_t nw = csize * wpc;
    const BatchParams prm = *a.prm;
    const T damp = static_cast<T>(prm.damp);
    const bool fp32 = sizeof(T) == 4;

    for (;;) {
        if (crank == 0 && threadIdx.x == 0)
            sh.graph = atomicAdd(a.queue, 1u);
        cluster.sync();
        const uint32_t q = *cluster.map_shared_rank(&sh.graph, 0);
        if (q >= a.count) {
            cluster.sync();  // no CTA exits while another still reads its shared memory
            break;
        }
        const uint32_t gi = a.order[q];
        const GraphMeta m = a.meta[gi];
        if (crank == 0 && threadIdx.x == 0)
            a.times[2 * gi] = global_ns();
        const T tele = static_cast<T>((1.0 - prm.damp) / static_cast<double>(m.n));
        // x = 1/n in gather form (PageRank.cpp:26)
        const T x0 = static_cast<T>(1.0 / static_cast<double>(m.n));
        for (uint32_t i = crank * THREADS + threadIdx.x; i < m.n; i += csize * THREADS) {
            const uint32_t r = m.base + i, dc = a.degc[r];
            a.y0[r] = dc ? x0 / static_cast<T>(dc) : x0;
        }
        // sink term of the first sweep: S0 = sinks / n spread over n rows
        T sink_coef = static_cast<T>(
            prm.distribute ? static_cast<double>(m.sinks) * (1.0 / static_cast<double>(m.n)) /
                                 static_cast<double>(m.n)
                           : 0.0);
        double res_prev = 0.0;
        unsigned long long it = 0;
        cluster.sync();
        for (;;) {
            const T *yin = (it & 1) ? a.y1 : a.y0;
            T *yout = (it & 1) ? a.y0 : a.y1;
            double res = 0.0, sumx = 0.0, sink = 0.0;
            const uint32_t items = m.n_long + m.slices;
            for (uint32_t item = cw; item < items; item += nw) {
                if (item < m.n_long) {
                    const uint32_t r = m.base + item;
                    const uint32_t b = a.row_ptr[r], e = a.row_ptr[r + 1];
                    T acc = T(0);
                    uint32_t k = b + lane;
                    for (; k + 96 < e; k += 128) {
                        uint32_t c[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            c[u] = __ldg(a.col + k + 32 * u);
                        T v[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            v[u] = ld_iter<CG>(yin + c[u]);
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            acc += v[u];
                    }
                    for (; k < e; k += 32)
                        acc += ld_iter<CG>(yin + __ldg(a.col + k));
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1)
                        acc += __shfl_xor_sync(0xffffffffu, acc, o);
                    if (lane == 0)
                        batch_finish<T, CG>(a, yin, yout, r, acc, damp, tele, sink_coef,
                                        prm.distribute, prm.l2, res, sumx, sink);
                } else {
                    const uint32_t s = m.slice0 + (item - m.n_long);
                    const uint32_t off = a.slice_off[s], len = a.slice_off[s + 1] - off;
                    const uint32_t *cp = a.col_sell + static_cast<size_t>(off) * 32 + lane;
                    T acc = T(0);
                    uint32_t j = 0;
                    for (; j + UNROLL <= len; j += UNROLL) {
                        uint32_t c[UNROLL];
#pragma unroll
                        for (int u = 0; u < UNROLL; ++u)
                            c[u] = __ldg(cp + static_cast<size_t>(j + u) * 32);
                        T v[UNROLL];
#pragma unroll
                        for (int u = 0; u < UNROLL; ++u)
                            v[u] = ld_iter<CG>(yin + c[u]);
#pragma unroll
                        for (int u = 0; u < UNROLL; ++u)
                            acc += v[u];
                    }
                    if (j < len) {
                        // the last len - j < UNROLL steps as one predicated batch (same order)
                        uint32_t c[UNROLL];
#pragma unroll
                        for (int u = 0; u < UNROLL; ++u)
                            c[u] = j + u < len ? __ldg(cp + static_cast<size_t>(j + u) * 32) : 0u;
                        T v[UNROLL];
#pragma unroll
                        for (int u = 0; u < UNROLL; ++u)
                            v[u] = j + u < len ? ld_iter<CG>(yin + c[u]) : T(0);
#pragma unroll
                        for (int u = 0; u < UNROLL; ++u)
                            if (j + u < len)
                                acc += v[u];
                    }
                    const uint32_t i = m.n_long + (item - m.n_long) * 32 + lane;
                    if (i < m.n)
                        batch_finish<T, CG>(a, yin, yout, m.base + i, acc, damp, tele, sink_coef,
                                        prm.distribute, prm.l2, res, sumx, sink);
                }
            }
            res = block_sum<THREADS>(res, sh.s_red);
            sumx = block_sum<THREADS>(sumx, sh.s_red);
            sink = block_sum<THREADS>(sink, sh.s_red);
            const int slot = static_cast<int>(it & 1);
            if (threadIdx.x == 0) {
                sh.part[slot][0] = res;
                sh.part[slot][1] = sumx;
                sh.part[slot][2] = sink;
            }
            cluster.sync();
            // Every CTA sums the partials in rank order and takes the same decision.
            if (threadIdx.x == 0) {
                double t0 = 0.0, t1 = 0.0, t2 = 0.0;
                for (unsigned rk = 0; rk < csize; ++rk) {
                    const double *pp = cluster.map_shared_rank(&sh.part[slot][0], rk);
                    t0 += pp[0];
                    t1 += pp[1];
                    t2 += pp[2];
                }
                const double norm = prm.l2 ? sqrt(t0) : t0;
                const unsigned long long done_it = it + 1;
                int done = (done_it >= prm.max_iterations || norm <= prm.tol) ? 1 : 0;
                int at_floor = 0;
                if (fp32 && !done && it >= 1 && norm > 0.9 * res_prev) {
                    done = 1;
                    at_floor = 1;
                }
                sh.done = done;
                sh.res = norm;
                sh.sumx = t1;
                sh.sink = t2;
                sh.sink_coef = prm.distribute ? t2 / static_cast<double>(m.n) : 0.0;
                if (done && crank == 0) {
                    a.times[2 * gi + 1] = global_ns();
                    a.iterations[gi] = done_it;
                    a.residual[gi] = norm;
                    if (at_floor)
                        atomicAdd(a.floor_stops, 1u);
                }
            }
            __syncthreads();
            res_prev = sh.res;
            sink_coef = static_cast<T>(sh.sink_coef);
            ++it;
            if (sh.done)
                break;
        }
        // Scores of the final iterate (PageRank.cpp:75-92), in caller ids.
        const double factor =
            prm.normalized ? (1.0 / static_cast<double>(m.n)) * ((1.0 - prm.damp) + prm.damp * sh.sink)
                           : sh.sumx;
        const T *yfin = (it & 1) ? a.y1 : a.y0;
        for (uint32_t i = crank * THREADS + threadIdx.x; i < m.n; i += csize * THREADS) {
            const uint32_t r = m.base + i, dc = a.degc[r];
            const T yv = ld_iter<CG>(yfin + r);
            const double x = dc ? static_cast<double>(t_mul(yv, static_cast<T>(dc)))
                                : static_cast<double>(yv);
            a.out[a.perm[r]] = x / factor;
        }
    }
}

// ---------------------------------------------------------------------------
// Layout build kernels

// Graph id of every node; the arcs' validity (sources inside the row's own
// graph); the out-degree count; the relabelling key (graph, in-degree desc).
__global__ void bt_node_graph(const uint64_t *__restrict__ node_off, uint32_t count,
                              uint32_t *__restrict__ node_graph) {
    for (uint32_t i = blockIdx.x; i < count; i += gridDim.x)
        for (uint64_t v = node_off[i] + threadIdx.x; v < node_off[i + 1]; v += blockDim.x)
            node_graph[v] = i;
}

// Graphs are relabelled by degree_bucket (common.cuh): inside a bucket rows
// keep their id order, so on graphs whose ids follow geometry (hyperbolic
// graphs number nodes by angle) neighbouring rows gather from neighbouring
// ids and the lanes of a warp share sectors.
__global__ void bt_validate(const uint64_t *__restrict__ in_ptr, const uint32_t *__restrict__ in_col,
                            const uint32_t *__restrict__ node_graph, uint32_t total, uint64_t arcs,
                            uint32_t *__restrict__ outdeg, uint64_t *__restrict__ keys,
                            uint32_t *__restrict__ ids, int *__restrict__ err) {
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint64_t v = warp; v < total; v += nwarps) {
        const uint64_t b = in_ptr[v], e = in_ptr[v + 1];
        if (e < b || e > arcs) {
            if (lane == 0)
                atomicCAS(err, 0, 1);
            continue;
        }
        const uint32_t gv = node_graph[v];
        if (lane == 0) {
            keys[v] = (static_cast<uint64_t>(gv) << 32) |
                      (0xffffffffu - degree_bucket(static_cast<uint32_t>(e - b)));
            ids[v] = static_cast<uint32_t>(v);
        }
        for (uint64_t k = b + lane; k < e; k += 32) {
            const uint32_t c = in_col[k];
            if (c >= total) {
                atomicCAS(err, 0, 2);
                continue;
            }
            if (node_graph[c] != gv) {
                atomicCAS(err, 0, 3);
                continue;
            }
            atomicAdd(outdeg + c, 1u);
        }
    }
}

__global__ void bt_perm(const uint32_t *__restrict__ sorted_ids, const uint64_t *__restrict__ in_ptr,
                        const uint32_t *__restrict__ outdeg, uint32_t total,
                        uint32_t *__restrict__ perm, uint32_t *__restrict__ inv,
                        uint32_t *__restrict__ rowlen, uint32_t *__restrict__ degc) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= total)
        return;
    const uint32_t o = sorted_ids[r];
    perm[r] = o;
    inv[o] = r;
    rowlen[r] = static_cast<uint32_t>(in_ptr[o + 1] - in_ptr[o]);
    degc[r] = outdeg[o];
}

__global__ void bt_relabel(const uint32_t *__restrict__ perm, const uint64_t *__restrict__ in_ptr,
                           const uint32_t *__restrict__ in_col, const uint32_t *__restrict__ inv,
                           const uint32_t *__restrict__ row_ptr, uint32_t total,
                           uint32_t *__restrict__ col) {
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint64_t r = warp; r < total; r += nwarps) {
        const uint64_t src = in_ptr[perm[r]];
        const uint32_t dst = row_ptr[r], len = row_ptr[r + 1] - dst;
        for (uint32_t j = lane; j < len; j += 32)
            col[dst + j] = inv[in_col[src + j]];
    }
}

// Per graph (one thread each): rows longer than T, a prefix of the graph's
// rows when T is a power of two (rows are ordered by degree bucket,
// descending; any other T gives a correct split with more padding).
__global__ void bt_split(GraphMeta *__restrict__ meta, uint32_t count,
                         const uint32_t *__restrict__ rowlen, uint32_t split) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count)
        return;
    GraphMeta m = meta[i];
    uint32_t lo = 0, hi = m.n;  // first row with length <= split
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (rowlen[m.base + mid] > split)
            lo = mid + 1;
        else
            hi = mid;
    }
    m.n_long = lo;
    m.slices = (m.n - lo + 31) / 32;
    meta[i] = m;
}

__global__ void bt_sinks(const uint32_t *__restrict__ degc, const uint32_t *__restrict__ node_graph,
                         uint32_t total, uint32_t *__restrict__ sinks) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < total && degc[r] == 0)
        atomicAdd(sinks + node_graph[r], 1u);
}

// Slice lengths (the longest of the slice's rows) and the graph of every
// slice.
__global__ void bt_slice_len(const GraphMeta *__restrict__ meta, uint32_t count,
                             const uint32_t *__restrict__ rowlen, uint32_t *__restrict__ slen,
                             uint32_t *__restrict__ slice_graph) {
    for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
        const GraphMeta m = meta[i];
        for (uint32_t k = threadIdx.x; k < m.slices; k += blockDim.x) {
            const uint32_t r0 = m.n_long + 32 * k, r1 = min(m.n, r0 + 32);
            uint32_t len = 0;
            for (uint32_t r = r0; r < r1; ++r)
                len = max(len, rowlen[m.base + r]);
            slen[m.slice0 + k] = len;
            slice_graph[m.slice0 + k] = i;
        }
    }
}

__global__ void bt_fill(const GraphMeta *__restrict__ meta, const uint32_t *__restrict__ slice_graph,
                        uint32_t slices, const uint32_t *__restrict__ slice_off,
                        const uint32_t *__restrict__ row_ptr, const uint32_t *__restrict__ col,
                        uint32_t pad, uint32_t *__restrict__ col_sell) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint32_t s = warp; s < slices; s += nwarps) {
        const GraphMeta m = meta[slice_graph[s]];
        const uint32_t i = m.n_long + (s - m.slice0) * 32 + lane;
        uint32_t start = 0, len = 0;
        if (i < m.n) {
            start = row_ptr[m.base + i];
            len = row_ptr[m.base + i + 1] - start;
        }
        const uint32_t off = slice_off[s], slen = slice_off[s + 1] - off;
        for (uint32_t j = 0; j < slen; ++j)
            col_sell[(static_cast<size_t>(off) + j) * 32 + lane] = j < len ? col[start + j] : pad;
    }
}

} // namespace
} // namespace nkg

using namespace nkg;

struct BatchGraph {
    cudaGraphExec_t exec = nullptr;
    uint32_t cluster = 0, threads = 0, split = 0, variant = 0;
    uint64_t layout_gen = 0;
};

struct nkg_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t count = 0, total = 0;
    uint64_t arcs = 0;
    std::vector<uint64_t> node_off;            // host copy (count+1)
    std::vector<GraphMeta> meta_h;
    DeviceArray<GraphMeta> meta;
    DeviceArray<uint32_t> order;               // queue -> graph (arcs, descending)
    DeviceArray<uint32_t> perm, degc, rowlen, row_ptr, col;
    DeviceArray<uint32_t> slice_off, col_sell;
    uint32_t slices = 0, layout_split = 0;
    uint64_t layout_gen = 0;
    BatchGraph graphs[2];  // [FP32, FP64]
    uint64_t slots = 0;
    DeviceArray<float> y32[2];
    DeviceArray<double> y64[2];
    DeviceArray<double> out_buf, residual;
    DeviceArray<unsigned long long> iterations;
    DeviceArray<unsigned long long> times;     // per graph: start, end (ns)
    DeviceArray<unsigned int> counters;        // queue, floor stops
    DeviceArray<BatchParams> prm;
    PinnedHost<BatchParams> prm_h;
    nkg_batch_tuning tuning{};
};

namespace nkg {
namespace {

void batch_layout(nkg_batch *b, uint32_t split) {
    if (b->col_sell && b->layout_split == split)
        return;
    cudaStream_t s = b->stream;
    const uint32_t count = b->count;
    bt_split<<<ceil_div(count, 128), 128, 0, s>>>(b->meta.get(), count, b->rowlen.get(), split);
    NKG_CUDA(cudaGetLastError());
    NKG_CUDA(cudaMemcpyAsync(b->meta_h.data(), b->meta.get(), count * sizeof(GraphMeta),
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    uint64_t slices = 0;
    for (auto &m : b->meta_h) {
        m.slice0 = static_cast<uint32_t>(slices);
        slices += m.slices;
    }
    require(slices < 0xffffffffull, "too many slices");
    b->slices = static_cast<uint32_t>(slices);
    NKG_CUDA(cudaMemcpyAsync(b->meta.get(), b->meta_h.data(), count * sizeof(GraphMeta),
                             cudaMemcpyHostToDevice, s));
    DeviceArray<uint32_t> slen(std::max<uint64_t>(slices, 1)), sgraph(std::max<uint64_t>(slices, 1));
    bt_slice_len<<<std::min<uint32_t>(count, 4096), 256, 0, s>>>(b->meta.get(), count,
                                                                 b->rowlen.get(), slen.get(),
                                                                 sgraph.get());
    NKG_CUDA(cudaGetLastError());
    b->slice_off.alloc(slices + 1);
    NKG_CUDA(cudaMemsetAsync(b->slice_off.get(), 0, sizeof(uint32_t), s));
    if (slices) {
        size_t tb = 0;
        NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, slen.get(), b->slice_off.get() + 1,
                                               static_cast<int64_t>(slices), s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb, slen.get(), b->slice_off.get() + 1,
                                               static_cast<int64_t>(slices), s));
    }
    const uint32_t cols = read_scalar(b->slice_off.get() + slices, s);
    b->slots = static_cast<uint64_t>(cols) * 32;
    b->col_sell.alloc(std::max<uint64_t>(b->slots, 1));
    if (slices)
        bt_fill<<<num_sms(b->device) * 16, 256, 0, s>>>(b->meta.get(), sgraph.get(), b->slices,
                                                        b->slice_off.get(), b->row_ptr.get(),
                                                        b->col.get(), b->total, b->col_sell.get());
    NKG_CUDA(cudaGetLastError());
    NKG_CUDA(cudaStreamSynchronize(s));
    b->layout_split = split;
    ++b->layout_gen;
}

template <typename T, int TH, typename F>
void with_batch_variant(uint32_t variant, F &&f) {
    const std::integral_constant<int, TH> th{};
    switch (variant & 3u) {
    case kVariantUnroll16: f(batch_kernel<T, TH, 16, false>, th); break;
    case kVariantL2Only: f(batch_kernel<T, TH, 8, true>, th); break;
    case kVariantUnroll16 | kVariantL2Only: f(batch_kernel<T, TH, 16, true>, th); break;
    default: f(batch_kernel<T, TH, 8, false>, th); break;
    }
}

// Calls f(kernel, threads) for the kernel of a tuning.
template <typename T, typename F>
void with_batch_kernel(const nkg_batch_tuning &t, F &&f) {
    switch (t.threads) {
    case 128: with_batch_variant<T, 128>(t.variant, f); break;
    case 512: with_batch_variant<T, 512>(t.variant, f); break;
    default: with_batch_variant<T, 256>(t.variant, f); break;
    }
}


// Launch the persistent kernel (queue reset first). Returns false when the
// cluster shape does not fit.
template <typename T>
bool batch_launch(nkg_batch *b, const nkg_batch_tuning &t, T *y0, T *y1, double *out,
                  bool check_only = false) {
    cudaStream_t s = b->stream;
    bool ok = true;
    with_batch_kernel<T>(t, [&](auto kfn, auto TH) {
        constexpr int threads = decltype(TH)::value;
        if (t.cluster > 8 &&
            cudaFuncSetAttribute(kfn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                cudaSuccess) {
            cudaGetLastError();
            ok = false;
            return;
        }
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = t.cluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.blockDim = dim3(threads);
        cfg.gridDim = dim3(t.cluster);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, kfn, &cfg) != cudaSuccess || clusters < 1) {
            cudaGetLastError();
            ok = false;
            return;
        }
        if (check_only)
            return;
        cfg.gridDim = dim3(static_cast<unsigned>(clusters) * t.cluster);
        BatchArgs<T> a{};
        a.meta = b->meta.get();
        a.order = b->order.get();
        a.row_ptr = b->row_ptr.get();
        a.col = b->col.get();
        a.slice_off = b->slice_off.get();
        a.col_sell = b->col_sell.get();
        a.degc = b->degc.get();
        a.perm = b->perm.get();
        a.y0 = y0;
        a.y1 = y1;
        a.out = out;
        a.iterations = b->iterations.get();
        a.residual = b->residual.get();
        a.times = b->times.get();
        a.queue = b->counters.get();
        a.floor_stops = b->counters.get() + 1;
        a.prm = b->prm.get();
        a.count = b->count;
        a.total = b->total;
        NKG_CUDA(cudaMemsetAsync(b->counters.get(), 0, 2 * sizeof(unsigned int), s));
        NKG_CUDA(cudaLaunchKernelEx(&cfg, kfn, a));
    });
    return ok;
}

void upload_params(nkg_batch *b, const nkg_pr_params &p) {
    BatchParams *h = b->prm_h.get();
    std::memset(h, 0, sizeof(*h));
    h->damp = p.damp;
    h->tol = p.tol;
    h->max_iterations = p.max_iterations;
    h->l2 = p.norm == NKG_NORM_L2;
    h->distribute = p.distribute_sinks ? 1 : 0;
    h->normalized = p.normalized ? 1 : 0;
    NKG_CUDA(cudaMemcpyAsync(b->prm.get(), h, sizeof(BatchParams), cudaMemcpyHostToDevice,
                             b->stream));
}

template <typename T>
void ensure_iterates(nkg_batch *b);
template <>
void ensure_iterates<float>(nkg_batch *b) {
    for (auto &y : b->y32)
        if (!y) {
            y.alloc(static_cast<size_t>(b->total) + 1);
            NKG_CUDA(cudaMemsetAsync(y.get(), 0, (static_cast<size_t>(b->total) + 1) * 4, b->stream));
        }
}
template <>
void ensure_iterates<double>(nkg_batch *b) {
    for (auto &y : b->y64)
        if (!y) {
            y.alloc(static_cast<size_t>(b->total) + 1);
            NKG_CUDA(cudaMemsetAsync(y.get(), 0, (static_cast<size_t>(b->total) + 1) * 8, b->stream));
        }
}

template <typename T>
T *iter_buf(nkg_batch *b, int k);
template <>
float *iter_buf<float>(nkg_batch *b, int k) { return b->y32[k].get(); }
template <>
double *iter_buf<double>(nkg_batch *b, int k) { return b->y64[k].get(); }

} // namespace
} // namespace nkg

namespace nkg {
namespace {

nkg_batch *batch_create(uint32_t count, const uint64_t *node_off, const uint64_t *in_ptr,
                        const uint32_t *in_col, int device) {
    require(count >= 1, "count must be >= 1");
    require(node_off != nullptr && in_ptr != nullptr, "node_offsets / in_row_ptr is NULL");
    require(node_off[0] == 0, "node_offsets[0] must be 0");
    for (uint32_t i = 0; i < count; ++i)
        require(node_off[i + 1] > node_off[i], "every graph needs at least one node");
    const uint64_t total = node_off[count];
    require(total < 0xffffffffull, "total node count must be < 2^32 - 1");
    const uint64_t arcs = in_ptr[total];
    require(in_ptr[0] == 0, "in_row_ptr must start at 0");
    require(arcs < 0xffffffffull, "total arc count must be < 2^32 - 1");
    require(arcs == 0 || in_col != nullptr, "in_col is NULL");
    int dev = device;
    if (dev < 0)
        NKG_CUDA(cudaGetDevice(&dev));
    DeviceGuard guard(dev);
    std::unique_ptr<nkg_batch> b(new nkg_batch());
    b->device = dev;
    b->count = count;
    b->total = static_cast<uint32_t>(total);
    b->arcs = arcs;
    b->node_off.assign(node_off, node_off + count + 1);
    b->stream = stream_acquire(dev);
    NKG_CUDA(cudaEventCreate(&b->ev0));
    NKG_CUDA(cudaEventCreate(&b->ev1));
    cudaStream_t s = b->stream;
    const unsigned sms = num_sms(dev);

    DeviceArray<uint64_t> d_ptr(total + 1), d_off(count + 1);
    DeviceArray<uint32_t> d_col(std::max<uint64_t>(arcs, 1));
    NKG_CUDA(cudaMemcpyAsync(d_ptr.get(), in_ptr, (total + 1) * 8, cudaMemcpyHostToDevice, s));
    NKG_CUDA(cudaMemcpyAsync(d_off.get(), node_off, (count + 1) * 8, cudaMemcpyHostToDevice, s));
    if (arcs)
        NKG_CUDA(cudaMemcpyAsync(d_col.get(), in_col, arcs * 4, cudaMemcpyHostToDevice, s));
    DeviceArray<uint32_t> node_graph(total), outdeg(total), ids(total), ids_s(total);
    DeviceArray<uint64_t> keys(total), keys_s(total);
    DeviceArray<int> err(1);
    NKG_CUDA(cudaMemsetAsync(outdeg.get(), 0, total * 4, s));
    NKG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
    bt_node_graph<<<std::min<uint32_t>(count, 8192), 256, 0, s>>>(d_off.get(), count,
                                                                  node_graph.get());
    bt_validate<<<sms * 16, 256, 0, s>>>(d_ptr.get(), d_col.get(), node_graph.get(),
                                         static_cast<uint32_t>(total), arcs, outdeg.get(),
                                         keys.get(), ids.get(), err.get());
    NKG_CUDA(cudaGetLastError());
    switch (read_scalar(err.get(), s)) {
    case 0: break;
    case 1: throw Error(NKG_ERR_INVALID_ARG, "in_row_ptr is not non-decreasing within [0, arcs]");
    case 2: throw Error(NKG_ERR_INVALID_ARG, "in_col holds a node id >= the total node count");
    default: throw Error(NKG_ERR_INVALID_ARG, "an arc joins two different graphs of the batch");
    }
    int gbits = 1;
    while (gbits < 32 && (1ull << gbits) <= count)
        ++gbits;
    {
        size_t tb = 0;
        NKG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.get(), keys_s.get(), ids.get(),
                                                 ids_s.get(), static_cast<int64_t>(total), 0,
                                                 32 + gbits, s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, keys.get(), keys_s.get(), ids.get(),
                                                 ids_s.get(), static_cast<int64_t>(total), 0,
                                                 32 + gbits, s));
    }
    DeviceArray<uint32_t> inv(total);
    b->perm.alloc(total);
    b->degc.alloc(total);
    b->rowlen.alloc(total);
    bt_perm<<<ceil_div(total, 256), 256, 0, s>>>(ids_s.get(), d_ptr.get(), outdeg.get(),
                                                 static_cast<uint32_t>(total), b->perm.get(),
                                                 inv.get(), b->rowlen.get(), b->degc.get());
    b->row_ptr.alloc(total + 1);
    NKG_CUDA(cudaMemsetAsync(b->row_ptr.get(), 0, sizeof(uint32_t), s));
    {
        size_t tb = 0;
        NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, b->rowlen.get(), b->row_ptr.get() + 1,
                                               static_cast<int64_t>(total), s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb, b->rowlen.get(), b->row_ptr.get() + 1,
                                               static_cast<int64_t>(total), s));
    }
    b->col.alloc(std::max<uint64_t>(arcs, 1));
    if (arcs)
        bt_relabel<<<sms * 16, 256, 0, s>>>(b->perm.get(), d_ptr.get(), d_col.get(), inv.get(),
                                            b->row_ptr.get(), static_cast<uint32_t>(total),
                                            b->col.get());
    DeviceArray<uint32_t> sinks(count);
    NKG_CUDA(cudaMemsetAsync(sinks.get(), 0, count * 4, s));
    bt_sinks<<<ceil_div(total, 256), 256, 0, s>>>(b->degc.get(), node_graph.get(),
                                                  static_cast<uint32_t>(total), sinks.get());
    NKG_CUDA(cudaGetLastError());
    std::vector<uint32_t> hs(count);
    NKG_CUDA(cudaMemcpyAsync(hs.data(), sinks.get(), count * 4, cudaMemcpyDeviceToHost, s));
    // graph arc counts for the queue order
    std::vector<uint64_t> garcs(count);
    for (uint32_t i = 0; i < count; ++i)
        garcs[i] = in_ptr[node_off[i + 1]] - in_ptr[node_off[i]];
    NKG_CUDA(cudaStreamSynchronize(s));
    b->meta_h.resize(count);
    for (uint32_t i = 0; i < count; ++i) {
        GraphMeta &m = b->meta_h[i];
        std::memset(&m, 0, sizeof(m));
        m.base = static_cast<uint32_t>(node_off[i]);
        m.n = static_cast<uint32_t>(node_off[i + 1] - node_off[i]);
        m.sinks = hs[i];
    }
    b->meta.alloc(count);
    NKG_CUDA(cudaMemcpyAsync(b->meta.get(), b->meta_h.data(), count * sizeof(GraphMeta),
                             cudaMemcpyHostToDevice, s));
    std::vector<uint32_t> order(count);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t x, uint32_t y) { return garcs[x] > garcs[y]; });
    b->order.alloc(count);
    NKG_CUDA(cudaMemcpyAsync(b->order.get(), order.data(), count * 4, cudaMemcpyHostToDevice, s));
    b->out_buf.alloc(total);
    b->residual.alloc(count);
    b->iterations.alloc(count);
    b->times.alloc(2 * static_cast<size_t>(count));
    b->counters.alloc(2);
    b->prm.alloc(1);
    b->prm_h.alloc(1);
    b->tuning.cluster = 4;
    b->tuning.threads = 256;
    b->tuning.split = 128;
    NKG_CUDA(cudaStreamSynchronize(s));
    return b.release();
}

void check_batch_params(const nkg_pr_params *p) {
    require(p != nullptr, "params is NULL");
    require(p->norm == NKG_NORM_L1 || p->norm == NKG_NORM_L2, "norm must be L1 (0) or L2 (1)");
    require(p->precision == NKG_PREC_FP64 || p->precision == NKG_PREC_FP32,
            "the batch runs in FP64 or FP32");
    require(std::isfinite(p->damp), "damp must be finite");
    require(!std::isnan(p->tol), "tol must not be NaN");
}

void check_tuning(const nkg_batch_tuning &t) {
    require(t.cluster == 1 || t.cluster == 2 || t.cluster == 4 || t.cluster == 8 ||
                t.cluster == kMaxCluster,
            "cluster must be 1, 2, 4, 8 or 16");
    require(t.threads == 128 || t.threads == 256 || t.threads == 512,
            "threads must be 128, 256 or 512");
    require(t.split >= 1, "split must be >= 1");
    require((t.variant & ~3u) == 0, "unknown variant bits");
}

// The queue reset and the persistent kernel, captured as one CUDA graph per
// precision (re-captured when the tuning or the layout changes).
template <typename T>
cudaGraphExec_t batch_graph(nkg_batch *b, const nkg_batch_tuning &t) {
    BatchGraph &G = b->graphs[sizeof(T) == 8 ? 1 : 0];
    if (G.exec && G.cluster == t.cluster && G.threads == t.threads && G.split == t.split &&
        G.variant == t.variant && G.layout_gen == b->layout_gen)
        return G.exec;
    if (G.exec)
        cudaGraphExecDestroy(G.exec);
    G.exec = nullptr;
    cudaStream_t s = b->stream;
    cudaGraph_t graph = nullptr;
    NKG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const bool ok = batch_launch<T>(b, t, iter_buf<T>(b, 0), iter_buf<T>(b, 1), b->out_buf.get());
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    require(ok, "the chosen cluster shape does not fit on this GPU");
    NKG_CUDA(e);
    e = cudaGraphInstantiate(&G.exec, graph, 0);
    cudaGraphDestroy(graph);
    NKG_CUDA(e);
    G.cluster = t.cluster;
    G.threads = t.threads;
    G.split = t.split;
    G.variant = t.variant;
    G.layout_gen = b->layout_gen;
    return G.exec;
}

// One run of the captured batch graph with the given tuning; device ms.
template <typename T>
float batch_timed(nkg_batch *b, const nkg_batch_tuning &t) {
    batch_layout(b, t.split);
    ensure_iterates<T>(b);
    cudaGraphExec_t exec = batch_graph<T>(b, t);
    NKG_CUDA(cudaEventRecord(b->ev0, b->stream));
    NKG_CUDA(cudaGraphLaunch(exec, b->stream));
    NKG_CUDA(cudaEventRecord(b->ev1, b->stream));
    NKG_CUDA(cudaEventSynchronize(b->ev1));
    NKG_CUDA(cudaGetLastError());
    float ms = 0.f;
    NKG_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    return ms;
}

} // namespace
} // namespace nkg

extern "C" {

int nkg_batch_create(nkg_batch **out, uint32_t count, const uint64_t *node_offsets,
                     const uint64_t *in_row_ptr, const uint32_t *in_col, int device) {
    return guarded([&] {
        require(out != nullptr, "out is NULL");
        *out = nullptr;
        *out = batch_create(count, node_offsets, in_row_ptr, in_col, device);
    });
}

void nkg_batch_destroy(nkg_batch *b) {
    if (!b)
        return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    for (auto &G : b->graphs)
        if (G.exec)
            cudaGraphExecDestroy(G.exec);
    if (b->ev0)
        cudaEventDestroy(b->ev0);
    if (b->ev1)
        cudaEventDestroy(b->ev1);
    cudaStream_t s = b->stream;
    const int dev = b->device;
    delete b;
    nkg::stream_release(dev, s);
    if (prev >= 0)
        cudaSetDevice(prev);
}

int nkg_batch_get_tuning(const nkg_batch *b, nkg_batch_tuning *t) {
    return guarded([&] {
        require(b != nullptr && t != nullptr, "NULL argument");
        *t = b->tuning;
    });
}

int nkg_batch_set_tuning(nkg_batch *b, const nkg_batch_tuning *t) {
    return guarded([&] {
        require(b != nullptr && t != nullptr, "NULL argument");
        check_tuning(*t);
        DeviceGuard guard(b->device);
        nkg_batch_tuning c = *t;
        c.ms = 0.0;
        require(batch_launch<float>(b, c, nullptr, nullptr, nullptr, true) &&
                    batch_launch<double>(b, c, nullptr, nullptr, nullptr, true),
                "the cluster shape does not fit on this GPU");
        b->tuning = c;
    });
}

int nkg_batch_tune(nkg_batch *b, const nkg_pr_params *p, uint32_t sweeps,
                   nkg_batch_tuning *results, uint32_t capacity, uint32_t *n_results,
                   nkg_batch_tuning *best_out) {
    return guarded([&] {
        require(b != nullptr, "batch is NULL");
        check_batch_params(p);
        require(sweeps <= 1000, "sweeps must be in [0, 1000]");
        DeviceGuard guard(b->device);
        nkg_pr_params tp = *p;
        if (sweeps) {
            tp.tol = -1.0;  // no stopping test: every graph runs `sweeps` sweeps
            tp.max_iterations = sweeps;
        }  // else every candidate runs the batch to convergence, as a real run does
        upload_params(b, tp);
        const uint32_t splits[] = {32, 64, 128, 256, 1024};
        const uint32_t threads[] = {256, 512};
        const uint32_t clusters[] = {1, 2, 4, 8, 16};
        nkg_batch_tuning best{};
        best.ms = 1e300;
        uint32_t nres = 0;
        for (uint32_t sp : splits)
            for (uint32_t th : threads)
                for (uint32_t cl : clusters) {
                    nkg_batch_tuning t{};
                    t.cluster = cl;
                    t.threads = th;
                    t.split = sp;
                    const bool fits =
                        p->precision == NKG_PREC_FP64
                            ? batch_launch<double>(b, t, nullptr, nullptr, nullptr, true)
                            : batch_launch<float>(b, t, nullptr, nullptr, nullptr, true);
                    if (!fits)
                        continue;
                    float ms;
                    if (p->precision == NKG_PREC_FP64) {
                        batch_timed<double>(b, t);  // warm-up (layout, caches)
                        ms = batch_timed<double>(b, t);
                    } else {
                        batch_timed<float>(b, t);
                        ms = batch_timed<float>(b, t);
                    }
                    t.ms = ms;
                    if (results && nres < capacity)
                        results[nres] = t;
                    ++nres;
                    if (ms < best.ms)
                        best = t;
                }
        require(nres > 0, "no cluster shape fits on this GPU");
        // Second stage: the kernel variants on the best shape.
        for (uint32_t var = 1; var <= 3; ++var) {
            nkg_batch_tuning t = best;
            t.variant = var;
            t.ms = 0.0;
            const bool fits =
                p->precision == NKG_PREC_FP64
                    ? batch_launch<double>(b, t, nullptr, nullptr, nullptr, true)
                    : batch_launch<float>(b, t, nullptr, nullptr, nullptr, true);
            if (!fits)
                continue;
            float ms;
            if (p->precision == NKG_PREC_FP64) {
                batch_timed<double>(b, t);
                ms = batch_timed<double>(b, t);
            } else {
                batch_timed<float>(b, t);
                ms = batch_timed<float>(b, t);
            }
            t.ms = ms;
            if (results && nres < capacity)
                results[nres] = t;
            ++nres;
            if (ms < best.ms)
                best = t;
        }
        b->tuning = best;
        batch_layout(b, best.split);
        if (n_results)
            *n_results = nres;
        if (best_out)
            *best_out = best;
    });
}

int nkg_batch_graph_times(nkg_batch *b, double *start_ms, double *end_ms) {
    return guarded([&] {
        require(b != nullptr && start_ms != nullptr && end_ms != nullptr, "NULL argument");
        DeviceGuard guard(b->device);
        std::vector<unsigned long long> t(2 * static_cast<size_t>(b->count));
        NKG_CUDA(cudaMemcpyAsync(t.data(), b->times.get(), t.size() * 8, cudaMemcpyDeviceToHost,
                                 b->stream));
        NKG_CUDA(cudaStreamSynchronize(b->stream));
        unsigned long long t0 = ~0ull;
        for (uint32_t i = 0; i < b->count; ++i)
            t0 = std::min(t0, t[2 * i]);
        for (uint32_t i = 0; i < b->count; ++i) {
            start_ms[i] = static_cast<double>(t[2 * i] - t0) * 1e-6;
            end_ms[i] = static_cast<double>(t[2 * i + 1] - t0) * 1e-6;
        }
    });
}

int nkg_batch_run(nkg_batch *b, const nkg_pr_params *p, double *scores_out, int flags,
                  uint64_t *iterations_out, uint32_t *floor_stops_out, nkg_stats *stats) {
    return guarded([&] {
        require(b != nullptr && scores_out != nullptr, "NULL argument");
        require((flags & ~NKG_DEVICE_PTRS) == 0, "unknown flags");
        check_batch_params(p);
        DeviceGuard guard(b->device);
        cudaStream_t s = b->stream;
        upload_params(b, *p);
        const float ms = p->precision == NKG_PREC_FP64 ? batch_timed<double>(b, b->tuning)
                                                       : batch_timed<float>(b, b->tuning);
        const bool dev = (flags & NKG_DEVICE_PTRS) != 0;
        NKG_CUDA(cudaMemcpyAsync(scores_out, b->out_buf.get(), static_cast<size_t>(b->total) * 8,
                                 dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
        std::vector<unsigned long long> its(b->count);
        std::vector<double> res(b->count);
        unsigned int counters[2];
        NKG_CUDA(cudaMemcpyAsync(its.data(), b->iterations.get(), b->count * 8,
                                 cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaMemcpyAsync(res.data(), b->residual.get(), b->count * 8,
                                 cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaMemcpyAsync(counters, b->counters.get(), sizeof(counters),
                                 cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        uint64_t sweeps = 0;
        double maxres = 0.0;
        for (uint32_t i = 0; i < b->count; ++i) {
            sweeps += its[i];
            maxres = std::max(maxres, res[i]);
            if (iterations_out)
                iterations_out[i] = its[i];
        }
        if (floor_stops_out)
            *floor_stops_out = counters[1];
        if (stats) {
            clear_stats(stats);
            stats->iterations = sweeps;
            stats->residual = maxres;
            stats->ms_total = ms;
            stats->ms_iterations = ms;
            stats->kernel_launches = 1;
            if (p->precision == NKG_PREC_FP64)
                stats->fp64_sweeps = sweeps;
            else
                stats->fp32_sweeps = sweeps;
        }
    });
}

} // extern "C"
