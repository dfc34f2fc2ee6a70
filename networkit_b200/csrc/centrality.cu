// EigenvectorCentrality and KatzCentrality on the sliced in-layout (the
// ranked-next rows of the PageRank path: the same pull SpMV, other
// epilogues).
//
//   EigenvectorCentrality::run (EigenvectorCentrality.cpp:20-60):
//     values[u] = sum over in-arcs (arc order) of w * x[v];
//     length = sqrt(sum values^2); x = values / length;
//     until |length - oldLength| <= tol (NumericTools::equal); |x| if x[0] < 0.
//   KatzCentrality::run (KatzCentrality.cpp:28-72):
//     values[u] = sum of w * alpha * (1 + x[v]) + beta; length as above;
//     x = values (no scaling inside the loop); until the length settles;
//     finally x / length.
// Deleted ids keep the initial 1 in both (they are never updated).
//
// Per iteration: one sweep over the slices (each lane sums its row in arc
// order, products rounded separately like the reference, no FMA
// contraction; warps take cost-balanced units of slices from a device
// counter and store each unit's sum of squares in a slot of its own), one
// fix-up for rows split into chunks whose last CTA reduces
// sum(values^2) in a fixed order and takes the stopping test. The eigenvector's
// division by the length is folded into the next sweep: x holds the values
// before scaling, every row divides its sum by the previous length once (the
// first sweep reads the initial 1s and divides by nothing), and the output
// pass divides by the last length. Padding slots gather the extra entry x[n],
// set to 0 (eigenvector) or -1 (Katz: alpha * (1 + -1) = 0), so they add 0.
// KatzCentrality with EdgeDirection::OutEdges runs over the out-layout of the
// adjoint (rows = nodes by out-degree).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "graph.hpp"
#include "host.hpp"
#include "sweep.cuh"

namespace nkg {
namespace {

constexpr int kCentThreads = 512;
constexpr int kCentUnroll = 8;
constexpr int kCentFix = 256;

struct CentState {
    double length;        // length of the last iteration's values
    unsigned long long iteration;
    int done;
    unsigned int ticket;
    unsigned int queue;   // next work unit of the sweep (reset by cent_fix)
};

struct CentArgs {
    const uint32_t *__restrict__ col_sell;
    const double *__restrict__ w_sell;       // weighted graphs
    const uint32_t *__restrict__ slice_off;
    const uint32_t *__restrict__ unit_start;
    const uint32_t *__restrict__ chunk_begin;
    const double *__restrict__ x_in;         // n+1 (x_in[n] = pad)
    double *__restrict__ x_out;              // n+1 (rows < n written)
    double *__restrict__ chunk_val;
    double *__restrict__ part;               // per work unit of the sweep
    double *__restrict__ fix_part;           // per fix-up CTA
    CentState *st;
    double alpha, beta, tol;
    unsigned long long max_iter;
    uint32_t n, n_long, n_vlong, s_chunk, units, sweep_ctas;
};

// One arc's term: w * x (eigenvector) or (w * alpha) * (1 + x) (Katz).
template <int MODE, bool WEIGHTED>
__device__ __forceinline__ double cent_term(const CentArgs &a, double x, double w) {
    if (MODE == 0)
        return WEIGHTED ? __dmul_rn(w, x) : x;
    const double wa = WEIGHTED ? __dmul_rn(w, a.alpha) : a.alpha;
    return __dmul_rn(wa, __dadd_rn(1.0, x));
}

// The previous iteration's length that eigenvector rows divide their sums by
// (0: the first iteration, whose input is the unscaled initial vector).
__device__ __forceinline__ double cent_prev_length(const CentArgs &a) {
    return a.st->iteration ? a.st->length : 0.0;
}

template <int MODE>
__device__ __forceinline__ void cent_row(const CentArgs &a, uint32_t r, double acc, double len_prev,
                                         double &sq) {
    const double v = MODE == 0 ? (len_prev > 0.0 ? acc / len_prev : acc) : __dadd_rn(acc, a.beta);
    a.x_out[r] = v;
    sq += v * v;
}

template <int MODE, bool WEIGHTED, int THREADS, int UNROLL>
__global__ void __launch_bounds__(THREADS, WEIGHTED || UNROLL > 8 ? 1024 / THREADS : 1536 / THREADS)
    cent_sweep(CentArgs a) {
    if (*(volatile int *)&a.st->done)
        return;
    const double len_prev = MODE == 0 ? cent_prev_length(a) : 0.0;
    const int lane = threadIdx.x & 31;
    // Warps take units from a device counter in order (as the queued
    // PageRank sweep); every unit's sum of squares goes to its own slot.
    const uint32_t nw = gridDim.x * (THREADS / 32);
    for (uint32_t u = blockIdx.x * (THREADS / 32) + (threadIdx.x >> 5); u < a.units;
         u = next_unit(&a.st->queue, a.units, nw, lane)) {
        double sq = 0.0;
        const uint32_t s_end = a.unit_start[u + 1];
        for (uint32_t s = a.unit_start[u]; s < s_end; ++s) {
            const uint32_t off = a.slice_off[s];
            const uint32_t len = a.slice_off[s + 1] - off;
            const size_t base = static_cast<size_t>(off) * 32 + lane;
            const uint32_t *cp = a.col_sell + base;
            double acc = 0.0;
            uint32_t j = 0;
            for (; j + UNROLL <= len; j += UNROLL) {
                uint32_t c[UNROLL];
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    c[k] = ld_stream(cp + static_cast<size_t>(j + k) * 32);
                double x[UNROLL], w[UNROLL];
#pragma unroll
                for (int k = 0; k < UNROLL; ++k) {
                    x[k] = __ldg(a.x_in + c[k]);
                    w[k] = WEIGHTED ? ld_stream(a.w_sell + base + static_cast<size_t>(j + k) * 32)
                                    : 1.0;
                }
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    acc = __dadd_rn(acc, cent_term<MODE, WEIGHTED>(a, x[k], w[k]));
            }
            if (j < len) {
                // the last len - j < UNROLL steps as one predicated batch (same order)
                uint32_t c[UNROLL];
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    c[k] = j + k < len ? ld_stream(cp + static_cast<size_t>(j + k) * 32) : 0u;
                double x[UNROLL], w[UNROLL];
#pragma unroll
                for (int k = 0; k < UNROLL; ++k) {
                    x[k] = j + k < len ? __ldg(a.x_in + c[k]) : 0.0;
                    w[k] = WEIGHTED && j + k < len
                               ? ld_stream(a.w_sell + base + static_cast<size_t>(j + k) * 32)
                               : 1.0;
                }
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    if (j + k < len)
                        acc = __dadd_rn(acc, cent_term<MODE, WEIGHTED>(a, x[k], w[k]));
            }
            if (s < a.s_chunk) {
                a.chunk_val[static_cast<size_t>(s) * 32 + lane] = acc;
            } else {
                const uint32_t r = a.n_long + (s - a.s_chunk) * 32 + lane;
                if (r < a.n)
                    cent_row<MODE>(a, r, acc, len_prev, sq);
            }
        }
        sq = warp_sum(sq);
        if (lane == 0)
            a.part[u] = sq;
    }
}

// Split rows (a warp for each row of many chunks, one thread for each other
// row; split_row_sum), then the last CTA sums
// the squares in a fixed order and takes NumericTools::equal(length, old, tol).
template <int MODE>
__global__ void __launch_bounds__(kCentFix) cent_fix(CentArgs a) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    if (*(volatile int *)&a.st->done)
        return;
    const double len_prev = MODE == 0 ? cent_prev_length(a) : 0.0;
    double sq = 0.0;
    // The sweep's unit partials: a fixed share of the units per thread.
    for (uint32_t i = blockIdx.x * kCentFix + threadIdx.x; i < a.units; i += gridDim.x * kCentFix)
        sq += a.part[i];
    uint32_t r;
    double acc;
    if (split_row_sum<kCentFix>(a.chunk_begin, a.chunk_val, a.n_long, a.n_vlong, r, acc))
        cent_row<MODE>(a, r, acc, len_prev, sq);
    sq = block_sum<kCentFix>(sq, s_red);
    if (threadIdx.x == 0) {
        a.fix_part[blockIdx.x] = sq;
        __threadfence();
        s_last = atomicAdd(&a.st->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    double t = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kCentFix)
        t += ((volatile double *)a.fix_part)[i];
    t = block_sum<kCentFix>(t, s_red);
    if (threadIdx.x == 0) {
        CentState *st = a.st;
        const double length = sqrt(t);
        const double old = st->length;
        const unsigned long long it = st->iteration + 1;
        st->length = length;
        st->iteration = it;
        st->ticket = 0;
        st->queue = 0;
        __threadfence();
        st->done = ((length <= old + a.tol && length >= old - a.tol) || it >= a.max_iter) ? 1 : 0;
    }
}

// Scores in the caller's ids: row of caller id o (via map, kNone = deleted)
// divided by the last length (both measures: the eigenvector's values are
// kept unscaled between sweeps), deleted ids 1; sign_fix makes
// every score |x| when x of caller id 0 is negative (EigenvectorCentrality.cpp:53-57).
__global__ void cent_output(const double *__restrict__ x, const uint32_t *__restrict__ row_of,
                            uint64_t z, const CentState *st, int divide, int sign_fix,
                            double *__restrict__ out) {
    const uint64_t o = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (o >= z)
        return;
    const uint32_t r = row_of[o];
    if (r == kNone) {
        out[o] = 1.0;
        return;
    }
    double v = x[r];
    if (divide)
        v = v / st->length;
    if (sign_fix) {
        const uint32_t r0 = row_of[0];
        if (r0 != kNone && x[r0] < 0.0)
            v = fabs(v);
    }
    out[o] = v;
}

__global__ void cent_init(double *__restrict__ x0, double *__restrict__ x1, uint32_t n,
                          double pad) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) {
        x0[r] = 1.0;
    } else if (r == n) {
        x0[n] = pad;
        x1[n] = pad;
    }
}

// caller id -> row of the out-layout (through the relabelling)
__global__ void out_row_of(const uint32_t *__restrict__ inv, const uint32_t *__restrict__ tinv,
                           uint64_t z, uint32_t *__restrict__ row_of) {
    const uint64_t o = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (o < z) {
        const uint32_t r = inv[o];
        row_of[o] = r == kNone ? kNone : tinv[r];
    }
}

struct CentResult {
    uint64_t iterations = 0, launches = 0;
    double length = 0.0, ms = 0.0;
};

template <int MODE, bool WEIGHTED>
CentResult cent_run(nkg_graph *g, const SellLayout &L, const double *w_sell, double alpha,
                    double beta, double tol, uint64_t max_iter, const uint32_t *row_of,
                    double *d_out) {
    cudaStream_t s = g->stream;
    const uint32_t n = static_cast<uint32_t>(g->n);
    const unsigned sms = num_sms(g->device);
    auto kfn = cent_sweep<MODE, WEIGHTED, kCentThreads, kCentUnroll>;
    NKG_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, 0));
    int occ = 0;
    NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, kCentThreads, 0));
    require(occ >= 1, "centrality kernel does not fit on an SM");
    const uint64_t slices = L.slices;
    const unsigned ctas = static_cast<unsigned>(std::max<uint64_t>(
        1, std::min<uint64_t>(static_cast<uint64_t>(occ) * sms,
                              (slices * 32 + kCentThreads - 1) / kCentThreads)));
    const uint32_t units = static_cast<uint32_t>(std::max<uint64_t>(
        1, std::min<uint64_t>(static_cast<uint64_t>(ctas) * (kCentThreads / 32) * kQueueUnitsPerWarp,
                              std::max<uint64_t>(slices, 1))));
    const unsigned fix_ctas =
        fix_ctas_with_units(split_fix_ctas<kCentFix>(L.n_long, L.n_vlong), units, kCentFix);
    DeviceArray<uint32_t> unit_start(static_cast<size_t>(units) + 1);
    sell_units(L, units, unit_start.get(), s);
    DeviceArray<double> x[2] = {DeviceArray<double>(n + 1), DeviceArray<double>(n + 1)};
    DeviceArray<double> chunk_val(static_cast<size_t>(L.s_chunk) * 32 + 1), part(units),
        fix_part(fix_ctas);
    DeviceArray<CentState> st(1);
    CentResult R;
    NKG_CUDA(cudaEventRecord(g->ev0, s));
    NKG_CUDA(cudaMemsetAsync(st.get(), 0, sizeof(CentState), s));
    cent_init<<<ceil_div(static_cast<uint64_t>(n) + 1, 256), 256, 0, s>>>(
        x[0].get(), x[1].get(), n, MODE == 0 ? 0.0 : -1.0);
    NKG_CUDA(cudaGetLastError());
    CentArgs a{};
    a.col_sell = L.col_sell.get();
    a.w_sell = w_sell;
    a.slice_off = L.slice_off.get();
    a.unit_start = unit_start.get();
    a.chunk_begin = L.chunk_begin.get();
    a.chunk_val = chunk_val.get();
    a.part = part.get();
    a.fix_part = fix_part.get();
    a.st = st.get();
    a.alpha = alpha;
    a.beta = beta;
    a.tol = tol;
    a.max_iter = max_iter;
    a.n = n;
    a.n_long = L.n_long;
    a.n_vlong = L.n_vlong;
    a.s_chunk = L.s_chunk;
    a.units = units;
    a.sweep_ctas = ctas;
    CentState *hst = reinterpret_cast<CentState *>(g->scalars_host.get());
    static_assert(sizeof(CentState) <= 16 * sizeof(double), "CentState fits the pinned buffer");
    for (;;) {
        for (int k = 0; k < kSweepsPerGraph; ++k) {
            a.x_in = x[k & 1].get();
            a.x_out = x[(k + 1) & 1].get();
            kfn<<<ctas, kCentThreads, 0, s>>>(a);
            cent_fix<MODE><<<fix_ctas, kCentFix, 0, s>>>(a);
        }
        NKG_CUDA(cudaGetLastError());
        R.launches += kSweepsPerGraph * 2;
        NKG_CUDA(cudaMemcpyAsync(hst, st.get(), sizeof(CentState), cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        if (hst->done)
            break;
        check_cancel(g, "centrality run cancelled");
    }
    R.iterations = hst->iteration;
    R.length = hst->length;
    const double *xfin = x[R.iterations & 1].get();
    cent_output<<<ceil_div(g->z, 256), 256, 0, s>>>(xfin, row_of, g->z, st.get(), 1,
                                                    MODE == 0 ? 1 : 0, d_out);
    NKG_CUDA(cudaGetLastError());
    R.launches += 2;
    NKG_CUDA(cudaEventRecord(g->ev1, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    NKG_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    R.ms = ms;
    return R;
}

__global__ void max_u32(const uint32_t *__restrict__ v, uint32_t n, unsigned int *__restrict__ out) {
    unsigned int m = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = max(m, v[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(out, m);
}

void finish_output(nkg_graph *g, double *d_out, double *out, bool on_device) {
    if (!on_device) {
        NKG_CUDA(cudaMemcpyAsync(out, d_out, g->z * sizeof(double), cudaMemcpyDeviceToHost,
                                 g->stream));
        NKG_CUDA(cudaStreamSynchronize(g->stream));
    }
}

void fill_stats(const CentResult &R, uint64_t *iterations_out, nkg_stats *stats) {
    if (iterations_out)
        *iterations_out = R.iterations;
    if (stats) {
        clear_stats(stats);
        stats->iterations = R.iterations;
        stats->residual = R.length;
        stats->ms_total = R.ms;
        stats->ms_iterations = R.ms;
        stats->kernel_launches = R.launches;
        stats->fp64_sweeps = R.iterations;
    }
}

} // namespace
} // namespace nkg

using namespace nkg;

extern "C" {

int nkg_eigenvector_run(nkg_graph *g, double tol, uint64_t max_iterations, double *scores_out,
                        int flags, uint64_t *iterations_out, nkg_stats *stats) {
    return guarded([&] {
        require(g != nullptr && scores_out != nullptr, "NULL argument");
        require((flags & ~NKG_DEVICE_PTRS) == 0, "unknown flags");
        require(!std::isnan(tol), "tol must not be NaN");
        DeviceGuard guard(g->device);
        RunScope scope(g);
        const bool dev = (flags & NKG_DEVICE_PTRS) != 0;
        DeviceArray<double> tmp;
        double *d_out = scores_out;
        if (!dev) {
            tmp.alloc(g->z);
            d_out = tmp.get();
        }
        const CentResult R =
            g->weighted ? cent_run<0, true>(g, g->fw, g->fw.w_sell64.get(), 0.0, 0.0, tol,
                                            max_iterations, g->inv.get(), d_out)
                        : cent_run<0, false>(g, g->fw, nullptr, 0.0, 0.0, tol, max_iterations,
                                             g->inv.get(), d_out);
        finish_output(g, d_out, scores_out, dev);
        fill_stats(R, iterations_out, stats);
    });
}

int nkg_katz_run(nkg_graph *g, double alpha, double beta, double tol, int edge_direction,
                 uint64_t max_iterations, double *scores_out, int flags, uint64_t *iterations_out,
                 nkg_stats *stats) {
    return guarded([&] {
        require(g != nullptr && scores_out != nullptr, "NULL argument");
        require((flags & ~NKG_DEVICE_PTRS) == 0, "unknown flags");
        require(edge_direction == 0 || edge_direction == 1,
                "edge_direction must be 0 (InEdges) or 1 (OutEdges)");
        require(!(alpha < 0), "Alpha must be non negative.");
        require(!std::isnan(tol) && std::isfinite(beta), "tol / beta must be numbers");
        DeviceGuard guard(g->device);
        RunScope scope(g);
        cudaStream_t s = g->stream;
        if (alpha == 0) {
            // KatzCentrality::defaultAlpha: 1 / (1 + maxDegree(G)), maxDegree = out-degree count
            DeviceArray<unsigned int> m(1);
            NKG_CUDA(cudaMemsetAsync(m.get(), 0, sizeof(unsigned int), s));
            max_u32<<<num_sms(g->device) * 4, 256, 0, s>>>(g->degc.get(),
                                                           static_cast<uint32_t>(g->n), m.get());
            NKG_CUDA(cudaGetLastError());
            alpha = 1.0 / (1.0 + static_cast<double>(read_scalar(m.get(), s)));
        }
        const bool dev = (flags & NKG_DEVICE_PTRS) != 0;
        DeviceArray<double> tmp;
        double *d_out = scores_out;
        if (!dev) {
            tmp.alloc(g->z);
            d_out = tmp.get();
        }
        CentResult R;
        if (edge_direction == 0) {
            R = g->weighted ? cent_run<1, true>(g, g->fw, g->fw.w_sell64.get(), alpha, beta, tol,
                                                max_iterations, g->inv.get(), d_out)
                            : cent_run<1, false>(g, g->fw, nullptr, alpha, beta, tol,
                                                 max_iterations, g->inv.get(), d_out);
        } else {
            const OutLayoutView ol = adjoint_out_layout(g);
            DeviceArray<uint32_t> row_of(g->z);
            out_row_of<<<ceil_div(g->z, 256), 256, 0, s>>>(g->inv.get(), ol.tinv, g->z,
                                                           row_of.get());
            NKG_CUDA(cudaGetLastError());
            R = g->weighted ? cent_run<1, true>(g, *ol.tl, ol.tl->w_sell64.get(), alpha, beta,
                                                tol, max_iterations, row_of.get(), d_out)
                            : cent_run<1, false>(g, *ol.tl, nullptr, alpha, beta, tol,
                                                 max_iterations, row_of.get(), d_out);
        }
        finish_output(g, d_out, scores_out, dev);
        fill_stats(R, iterations_out, stats);
    });
}

} // extern "C"
