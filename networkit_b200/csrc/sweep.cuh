// One Jacobi sweep of PageRank (PageRank.cpp:56-70) as a merge-path pull SpMV
// over the in-CSR plus a fix-up kernel that finishes rows cut by tile
// boundaries and closes the iteration (residual, sink mass, convergence).
//
// Storage: the iterate is kept in "gather form" y[r] = x[r] / deg[r] for nodes
// with out-arcs and y[r] = x[r] for sinks, so that a sweep gathers exactly the
// per-arc term x[v]*w/deg[v] of PageRank.cpp:62 (bit-identical for unweighted
// graphs, where w = 1). The previous x[r] needed by the stopping test
// (PageRank.cpp:41-51) is recovered as y[r]*deg[r].
//
// Work split (Merrill & Garland, "Merge-based Parallel Sparse Matrix-Vector
// Multiplication", SC'16): the sequence of n row-ends and `arcs` arcs is cut
// into tiles of TILE = THREADS*IPT items; a persistent CTA walks tiles
// blockIdx.x, blockIdx.x+gridDim.x, ... Every thread consumes IPT consecutive
// items, so power-law rows cost the same per item as short ones. Rows that
// straddle a tile boundary leave a head/tail partial for the fix-up kernel.
// All sums use fixed trees, so a run is bit-reproducible.
#pragma once

#include "common.cuh"

namespace nkg {

// Constant per run, read from device memory so that captured CUDA graphs
// stay valid across runs with different parameters.
struct RunParams {
    double damp;
    double tele_uniform;  // (1 - damp) / n  (PageRank.cpp:25)
    double one_minus_damp;
    double inv_n;
    int distribute;       // distributeSinks
    int personal;         // teleport vector present
    int l2;               // norm == L2
    int pad;
    double tol;
    unsigned long long max_iterations;
};

// Mutable per-run state, advanced by the last CTA of every fix-up launch.
struct IterState {
    unsigned long long iteration;  // completed sweeps
    double residual;               // norm of the last sweep
    double sink_mass;              // sum of x over sinks of the last iterate
    double sink_coef;              // sink term applied by the next sweep
    int done;                      // converged / max reached
    unsigned int ticket;           // last-block detection in the fix-up
    int pad[2];
};

template <typename T>
struct SweepArgs {
    const uint32_t *__restrict__ row_ptr;  // n+1
    const uint32_t *__restrict__ col;      // arcs (node ids after relabelling)
    const T *__restrict__ w;               // arc weights (weighted graphs)
    const uint32_t *__restrict__ degc;     // out-degree count (unweighted)
    const T *__restrict__ degw;            // weighted out-degree (weighted)
    const T *__restrict__ tele;            // personalised teleport (n) or null
    const T *__restrict__ y_in;
    T *__restrict__ y_out;
    const uint32_t *__restrict__ tile_row; // ntiles+1 merge-path coordinates
    const uint32_t *__restrict__ tile_arc;
    T *__restrict__ head_val;              // per tile: partial of its first row
    T *__restrict__ tail_val;              // per tile: partial of its last row
    double *__restrict__ cta_res;          // per sweep CTA
    double *__restrict__ cta_sink;
    double *__restrict__ fix_res;          // per fix-up CTA
    double *__restrict__ fix_sink;
    const RunParams *__restrict__ rp;
    IterState *st;
    uint32_t ntiles;
    uint32_t n;
    uint32_t n_nonsink;  // rows [n_nonsink, n) are sinks (out-degree 0)
    uint32_t sweep_ctas;
};

template <typename T>
__device__ __forceinline__ T t_mul(T a, T b);
template <>
__device__ __forceinline__ double t_mul<double>(double a, double b) { return __dmul_rn(a, b); }
template <>
__device__ __forceinline__ float t_mul<float>(float a, float b) { return __fmul_rn(a, b); }
template <typename T>
__device__ __forceinline__ T t_add(T a, T b);
template <>
__device__ __forceinline__ double t_add<double>(double a, double b) { return __dadd_rn(a, b); }
template <>
__device__ __forceinline__ float t_add<float>(float a, float b) { return __fadd_rn(a, b); }

// Finish row r from its in-arc sum `acc`: PageRank.cpp:64-65 (plus the sink
// term of distributeSinks), the residual term of PageRank.cpp:34-39 and the
// new gather-form value. No FMA contraction: the reference rounds the
// multiply and the add separately.
template <typename T, bool WEIGHTED>
__device__ __forceinline__ void finish_row(const SweepArgs<T> &a, const RunParams &rp, T sink_coef,
                                           uint32_t r, T acc, double &res, double &sink) {
    if (rp.distribute)
        acc = t_add(acc, rp.personal ? t_mul(sink_coef, a.tele[r]) : sink_coef);
    T x = t_mul(acc, static_cast<T>(rp.damp));
    x = t_add(x, rp.personal ? t_mul(static_cast<T>(rp.one_minus_damp), a.tele[r])
                             : static_cast<T>(rp.tele_uniform));
    const bool is_sink = r >= a.n_nonsink;
    const T yo = a.y_in[r];
    T deg;
    if (WEIGHTED)
        deg = ld_stream(a.degw + r);
    else
        deg = static_cast<T>(ld_stream(a.degc + r));
    const T xo = is_sink ? yo : t_mul(yo, deg);
    const double d = static_cast<double>(xo) - static_cast<double>(x);
    res += rp.l2 ? __dmul_rn(d, d) : fabs(d);
    if (is_sink) {
        sink += static_cast<double>(x);
        a.y_out[r] = x;
    } else {
        a.y_out[r] = x / deg;
    }
}

// Segmented inclusive scan of (row, value) pairs over the block in thread
// order: (r1,v1) + (r2,v2) = (r2, r1 == r2 ? v1 + v2 : v2). Rows are
// non-decreasing in thread order, which makes the operator associative.
// Returns the exclusive prefix in (ex_row, ex_val) (ex_row = kNone for thread
// 0) and the inclusive value in inc_val.
template <typename T, int THREADS>
__device__ __forceinline__ void seg_scan(uint32_t row, T val, uint32_t &ex_row, T &ex_val,
                                         T &inc_val, uint32_t *s_wrow, T *s_wval) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T v = val;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T vu = __shfl_up_sync(0xffffffffu, v, o);
        const uint32_t ru = __shfl_up_sync(0xffffffffu, row, o);
        if (lane >= o && ru == row)
            v = vu + v;
    }
    if (lane == 31) {
        s_wrow[wid] = row;
        s_wval[wid] = v;
    }
    __syncthreads();
    uint32_t pr = kNone;
    T pv = T(0);
    for (int j = 0; j < wid; ++j) {
        const uint32_t rj = s_wrow[j];
        const T vj = s_wval[j];
        pv = (pr == rj) ? pv + vj : vj;
        pr = rj;
    }
    if (wid > 0 && pr == row)
        v = pv + v;
    inc_val = v;
    const T vprev = __shfl_up_sync(0xffffffffu, v, 1);
    const uint32_t rprev = __shfl_up_sync(0xffffffffu, row, 1);
    if (lane > 0) {
        ex_row = rprev;
        ex_val = vprev;
    } else {
        ex_row = wid > 0 ? pr : kNone;
        ex_val = pv;
    }
}

template <typename T, bool WEIGHTED, int THREADS, int IPT>
struct SweepSmem {
    static constexpr int TILE = THREADS * IPT;
    static constexpr size_t bytes = sizeof(T) * TILE * 2 + sizeof(uint32_t) * TILE;
};

template <typename T, bool WEIGHTED, int THREADS, int IPT>
__global__ void __launch_bounds__(THREADS) sweep_kernel(SweepArgs<T> a) {
    constexpr int TILE = THREADS * IPT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *s_val = reinterpret_cast<T *>(smem_raw);
    T *s_rowsum = s_val + TILE;
    uint32_t *s_rowend = reinterpret_cast<uint32_t *>(s_rowsum + TILE);
    __shared__ uint32_t s_wrow[THREADS / 32];
    __shared__ T s_wval[THREADS / 32];
    __shared__ double s_red[32];
    __shared__ int s_head;

    if (*(volatile int *)&a.st->done)
        return;
    const RunParams rp = *a.rp;
    const T sink_coef = static_cast<T>(a.st->sink_coef);
    double res = 0.0, sink = 0.0;

    for (uint32_t t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const uint32_t row0 = a.tile_row[t], row1 = a.tile_row[t + 1];
        const uint32_t arc0 = a.tile_arc[t], arc1 = a.tile_arc[t + 1];
        const int nr = static_cast<int>(row1 - row0);
        const int na = static_cast<int>(arc1 - arc0);
        __syncthreads();  // smem of the previous tile is no longer read
        for (int i = threadIdx.x; i < nr; i += THREADS)
            s_rowend[i] = ld_stream(a.row_ptr + row0 + i + 1) - arc0;
        if (threadIdx.x == 0)
            s_head = (nr > 0 && a.row_ptr[row0] < arc0) ? 1 : 0;
        // Gather phase: all column loads first, then all gathers, so every
        // thread keeps IPT independent loads in flight.
        uint32_t c[IPT];
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int i = k * THREADS + threadIdx.x;
            c[k] = i < na ? ld_stream(a.col + arc0 + i) : kNone;
        }
        T v[IPT];
#pragma unroll
        for (int k = 0; k < IPT; ++k)
            v[k] = c[k] != kNone ? __ldg(a.y_in + c[k]) : T(0);
        if (WEIGHTED) {
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                const int i = k * THREADS + threadIdx.x;
                if (i < na)
                    v[k] = t_mul(v[k], ld_stream(a.w + arc0 + i));
            }
        }
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int i = k * THREADS + threadIdx.x;
            if (i < na)
                s_val[i] = v[k];
        }
        __syncthreads();

        // Merge-path split of this thread's IPT items.
        const int total = nr + na;
        const int diag = min(static_cast<int>(threadIdx.x) * IPT, total);
        const int diag_end = min(diag + IPT, total);
        int lo = max(diag - na, 0), hi = min(diag, nr);
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (static_cast<int>(s_rowend[mid]) <= diag - mid - 1)
                lo = mid + 1;
            else
                hi = mid;
        }
        int ri = lo, ai = diag - lo;
        T acc = T(0), first_val = T(0);
        int first_row = -1;
        for (int k = diag; k < diag_end; ++k) {
            if (ri < nr && ai >= static_cast<int>(s_rowend[ri])) {
                if (first_row < 0) {
                    first_row = ri;
                    first_val = acc;
                } else {
                    s_rowsum[ri] = acc;
                }
                acc = T(0);
                ++ri;
            } else {
                acc += s_val[ai];
                ++ai;
            }
        }
        // Rows cut between threads: add the partial sums of earlier threads.
        uint32_t ex_row;
        T ex_val, inc_val;
        seg_scan<T, THREADS>(static_cast<uint32_t>(ri), acc, ex_row, ex_val, inc_val, s_wrow,
                             s_wval);
        if (first_row >= 0)
            s_rowsum[first_row] =
                (ex_row == static_cast<uint32_t>(first_row)) ? ex_val + first_val : first_val;
        // The last row has arcs past the last row end: hand its partial on.
        if (threadIdx.x == THREADS - 1) {
            const bool tail = na > 0 && (nr == 0 || static_cast<int>(s_rowend[nr - 1]) < na);
            if (tail)
                a.tail_val[t] = inc_val;
        }
        __syncthreads();
        const int head = s_head;
        for (int i = threadIdx.x; i < nr; i += THREADS) {
            if (i == 0 && head) {
                a.head_val[t] = s_rowsum[0];
                continue;
            }
            finish_row<T, WEIGHTED>(a, rp, sink_coef, row0 + i, s_rowsum[i], res, sink);
        }
    }
    const double bres = block_sum<THREADS>(res, s_red);
    const double bsink = block_sum<THREADS>(sink, s_red);
    if (threadIdx.x == 0) {
        a.cta_res[blockIdx.x] = bres;
        a.cta_sink[blockIdx.x] = bsink;
    }
}

// Finish the rows that start in an earlier tile, then (last CTA) reduce all
// partial sums in index order and close the iteration (PageRank.cpp:68-70).
template <typename T, bool WEIGHTED, int THREADS>
__global__ void __launch_bounds__(THREADS) fixup_kernel(SweepArgs<T> a) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    if (*(volatile int *)&a.st->done)
        return;
    const RunParams rp = *a.rp;
    const T sink_coef = static_cast<T>(a.st->sink_coef);
    double res = 0.0, sink = 0.0;
    const uint32_t t = blockIdx.x * THREADS + threadIdx.x;
    if (t < a.ntiles) {
        const uint32_t row0 = a.tile_row[t];
        const uint32_t rs = a.row_ptr[row0];
        if (a.tile_row[t + 1] > row0 && a.tile_arc[t] > rs) {
            // Tiles t0..t-1 end inside row0; sum their tails in order.
            uint32_t t0 = t - 1;
            while (t0 > 0 && a.tile_row[t0] == row0 && a.tile_arc[t0] > rs)
                --t0;
            T sum = T(0);
            for (uint32_t k = t0; k < t; ++k)
                sum += a.tail_val[k];
            sum += a.head_val[t];
            finish_row<T, WEIGHTED>(a, rp, sink_coef, row0, sum, res, sink);
        }
    }
    const double bres = block_sum<THREADS>(res, s_red);
    const double bsink = block_sum<THREADS>(sink, s_red);
    if (threadIdx.x == 0) {
        a.fix_res[blockIdx.x] = bres;
        a.fix_sink[blockIdx.x] = bsink;
        __threadfence();
        const unsigned prev = atomicAdd(&a.st->ticket, 1u);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    // Fixed-order reduction of sweep-CTA and fix-up-CTA partials.
    double r = 0.0, s = 0.0;
    for (uint32_t i = threadIdx.x; i < a.sweep_ctas; i += THREADS) {
        r += ((volatile double *)a.cta_res)[i];
        s += ((volatile double *)a.cta_sink)[i];
    }
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += THREADS) {
        r += ((volatile double *)a.fix_res)[i];
        s += ((volatile double *)a.fix_sink)[i];
    }
    r = block_sum<THREADS>(r, s_red);
    s = block_sum<THREADS>(s, s_red);
    if (threadIdx.x == 0) {
        IterState *st = a.st;
        const unsigned long long it = st->iteration + 1;
        const double norm = rp.l2 ? sqrt(r) : r;
        st->iteration = it;
        st->residual = norm;
        st->sink_mass = s;
        st->sink_coef = rp.distribute ? (rp.personal ? s : s / static_cast<double>(a.n)) : 0.0;
        st->ticket = 0;
        __threadfence();
        st->done = (it >= rp.max_iterations || norm <= rp.tol) ? 1 : 0;
    }
}

} // namespace nkg
