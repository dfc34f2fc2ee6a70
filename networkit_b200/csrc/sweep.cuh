// One Jacobi sweep of PageRank (PageRank.cpp:56-70) as a sliced-ELLPACK pull
// SpMV over the in-adjacency, plus a fix-up kernel that finishes the rows that
// were split into chunks and closes the iteration (residual, sink mass,
// convergence test).
//
// Storage of the iterate: "gather form" y[r] = x[r] / deg[r] for nodes with
// out-arcs and y[r] = x[r] for sinks, so a sweep gathers exactly the per-arc
// term x[v]*w/deg[v] of PageRank.cpp:62 (bit-identical for unweighted graphs,
// where w = 1). The previous x[r] for the stopping test (PageRank.cpp:41-51)
// is recovered as y[r]*deg[r]. y has one extra zero entry at index n, the
// target of padding slots.
//
// Layout (SELL-C-sigma, Kreutzer et al., SIAM J. Sci. Comput. 36(5), 2014, with
// C = 32 and sigma = n): nodes are relabelled by in-degree, descending, so 32
// consecutive rows have nearly equal length. Rows longer than kChunk arcs are
// cut into chunks of kChunk arcs ("virtual rows", placed first). Slice s holds
// 32 virtual rows column-major: slot (j, lane) at col_sell[(off[s] + j) * 32 +
// lane], so a warp loads 128 contiguous bytes per step and every lane sums its
// own row sequentially, in the reference's arc order. No shared memory and no
// barriers are needed: the whole L1 is left to cache the hot part of y.
// The slices are cut into contiguous, cost-balanced ranges ("units", fixed at
// set-up). Every warp runs one unit of its own first and then takes the next
// unit from a device counter (next_unit), so no warp is left with a share that
// ends late. Each unit's residual and sink partials go to a slot of its own, so
// every sum has a fixed order and a run is bit-reproducible.
#pragma once

#include <algorithm>

#include "common.cuh"

namespace nkg {

// Arcs per chunk of a split row; also the longest sequential loop of a lane.
// Measured with the queued units (same box each): 512-arc chunks made R-MAT 24
// (FP64) runs 0.9% faster (55,455 split rows instead of 190,051, a lighter
// fix-up) but the weighted R-MAT 22 forward + backward 9% slower and the 4M
// hyperbolic graph 1% slower; 128 was slower on R-MAT 24 too.
constexpr uint32_t kChunk = 256;
// A split row with more chunks than this is summed by a whole warp in the fix-up.
constexpr uint32_t kShortChunks = 16;

// Work units of the queued sweeps: warp gw of nw runs unit gw first, with no
// ticket, then units nw + t for the tickets t it takes from `queue`, while
// any are left. A grid that covers all units takes no tickets at all, so small
// graphs pay no atomics. Returns the warp's next unit (>= units: done).
__device__ __forceinline__ uint32_t next_unit(unsigned int *queue, uint32_t units, uint32_t nw,
                                              int lane) {
    if (nw >= units)
        return units;
    uint32_t t = 0;
    if (lane == 0)
        t = atomicAdd(queue, 1u);
    return nw + __shfl_sync(0xffffffffu, t, 0);
}

// Fix-up CTAs of a queued sweep: those its split rows need, and enough that
// no thread adds more than kUnitsPerFixThread of the sweep's unit partials.
constexpr uint32_t kUnitsPerFixThread = 4;
inline unsigned fix_ctas_with_units(unsigned split_ctas, uint64_t units, unsigned threads) {
    const uint64_t per_cta = static_cast<uint64_t>(threads) * kUnitsPerFixThread;
    return static_cast<unsigned>(std::max<uint64_t>(split_ctas, (units + per_cta - 1) / per_cta));
}

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
    double residual_sum;           // its sum before the square root (L2)
    double sink_mass;              // sum of x over sinks of the last iterate
    double sink_coef;              // sink term applied by the next sweep
    int done;                      // converged / max reached
    unsigned int ticket;           // last-block detection in the fix-up
    int error;
    unsigned int queue;            // next work unit of a queued sweep (reset by the fix-up)
};

template <typename T>
struct SweepArgs {
    const uint32_t *__restrict__ col_sell;   // slices, column-major, padded with n
    const T *__restrict__ w_sell;            // matching weights (weighted graphs)
    const uint32_t *__restrict__ slice_off;  // S+1, in units of 32 slots
    const uint32_t *__restrict__ unit_start; // U+1 slice indices
    const uint32_t *__restrict__ chunk_begin;// n_long+1: chunks of split row r
    const uint32_t *__restrict__ degc;       // out-degree count (sink test)
    const T *__restrict__ degw;              // weighted out-degree (weighted graphs)
    const T *__restrict__ tele;              // personalised teleport (n) or null
    const T *__restrict__ y_in;              // n+1 (y_in[n] = 0)
    T *__restrict__ y_out;
    T *__restrict__ chunk_val;               // per chunk slot: partial row sum
    double *__restrict__ cta_res;            // per sweep CTA
    double *__restrict__ cta_sink;
    double *__restrict__ fix_res;            // per fix-up CTA
    double *__restrict__ fix_sink;
    const RunParams *__restrict__ rp;
    IterState *st;
    uint32_t n;
    uint32_t n_long;        // rows [0, n_long) are split into chunks
    uint32_t n_vlong;       // rows [0, n_vlong) have more than kShortChunks chunks
    uint32_t s_chunk;       // slices [0, s_chunk) hold chunks, the rest rows
    uint32_t units;
    uint32_t sweep_ctas;
    uint32_t hot;           // ids [0, hot) are read from the shared-memory tier
    uint32_t trace_cap;     // entries of trace
    double *trace;          // residual of completed sweep i at [i] (i < trace_cap)
    // Row slice of a partitioned run (PART kernels): local row r (in the
    // slice's own relabelled order) is slice row row_map[r]; the slice's
    // iterate entries, degrees, teleport and output are in slice row order,
    // and its previous iterate value sits at y_in[row_base + row_map[r]] of
    // the shared iterate, whose entry `pad` is the zero of padding slots.
    const uint32_t *__restrict__ row_map;
    uint32_t row_base;
    uint32_t pad;
    // Queued sweep: warps take units from IterState::queue and store each
    // unit's residual and sink partial sums here (indexed by unit), so the
    // sums keep a fixed order whichever warp ran the unit. Null: the static
    // round-robin assignment with per-CTA partials in cta_res / cta_sink.
    double *unit_res;
    double *unit_sink;
    // The queued sweep's last CTA closes the iteration itself (graphs with no
    // split rows and few units; no fix-up launch): see close_iteration.
    int close_in_sweep;
    int pad5;
};

// Graphs with no split rows and at most this many units close every
// iteration in the sweep's last CTA instead of a fix-up launch.
constexpr uint32_t kCloseInSweepUnits = 8192;

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
template <typename T, bool WEIGHTED, bool PART = false>
__device__ __forceinline__ void finish_row(const SweepArgs<T> &a, const RunParams &rp, T sink_coef,
                                           uint32_t r0, T acc, double &res, double &sink) {
    const uint32_t r = PART ? a.row_map[r0] : r0;
    const uint32_t dc = ld_stream(a.degc + r);
    const T deg = WEIGHTED ? ld_stream(a.degw + r) : static_cast<T>(dc);
    const T yo = a.y_in[(PART ? a.row_base : 0u) + r];
    if (rp.distribute)
        acc = t_add(acc, rp.personal ? t_mul(sink_coef, a.tele[r]) : sink_coef);
    T x = t_mul(acc, static_cast<T>(rp.damp));
    x = t_add(x, rp.personal ? t_mul(static_cast<T>(rp.one_minus_damp), a.tele[r])
                             : static_cast<T>(rp.tele_uniform));
    const bool is_sink = dc == 0;
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

// Per-run constants read where a row is finished. The volatile asm keeps each
// load at its use, so the values are not hoisted into registers held across
// the gather loop.
__device__ __forceinline__ double ld_keep(const double *p) {
    double v;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ int ld_keep(const int *p) {
    int v;
    asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

template <typename T, bool WEIGHTED, bool PART = false>
__device__ __forceinline__ void finish_row_sweep(const SweepArgs<T> &a, uint32_t r, T acc,
                                                 double &res, double &sink) {
    RunParams rp;
    rp.damp = ld_keep(&a.rp->damp);
    rp.tele_uniform = ld_keep(&a.rp->tele_uniform);
    rp.one_minus_damp = ld_keep(&a.rp->one_minus_damp);
    rp.distribute = ld_keep(&a.rp->distribute);
    rp.personal = ld_keep(&a.rp->personal);
    rp.l2 = ld_keep(&a.rp->l2);
    const T sink_coef = static_cast<T>(ld_keep(&a.st->sink_coef));
    finish_row<T, WEIGHTED, PART>(a, rp, sink_coef, r, acc, res, sink);
}

// Padding slots (column n, whose gathered value is the zero entry y[n]) skip
// the load and add zero, the same sum bit for bit without the L1 lookup.
// Gathers go through L1 with the default policy (__ldg); the kernel uses no
// shared memory, so the whole L1 caches the hot scores. The sweep is bound by
// L1 miss requests to L2 (one sector per scattered lane). Measured
// alternatives that were slower on B200: L2-only loads; holding the hottest
// scores in shared memory (random 8-byte loads hit bank conflicts and
// throttle the MIO queue); per-lane L1 evict-last / no-allocate hints (the
// predicated loads raise register use and cut occupancy).

// Launch shapes of the sweep kernel: threads per CTA and slot steps per batch
// of independent gathers.
template <int TH, int UNROLL_>
struct SweepShape {
    static constexpr int threads = TH, unroll = UNROLL_;
};
constexpr int kNumSweepShapes = 4;

template <typename F>
inline void with_sweep_shape(int v, F &&f) {
    switch (v) {
    case 1: f(SweepShape<256, 8>{}); break;
    case 2: f(SweepShape<256, 4>{}); break;
    case 3: f(SweepShape<256, 16>{}); break;
    default: f(SweepShape<512, 8>{}); break;
    }
}

// Hot-source tier. The rows are relabelled by in-degree, and on power-law
// graphs in- and out-degree go together, so the first ids are also the
// sources that most arcs gather from (on directed R-MAT scale 24 the first
// 28,672 ids are the sources of 34% of the arcs, the first 57,344 of 46%).
// The tier copies y_in[0, hot) into shared memory at the start of every
// sweep, and a gather of such an id is a shared-memory load instead of a
// request through L1. Every other gather goes through L1 as before. Each CTA
// holds its own copy of the tier: two CTAs of 768 threads per SM (48 warps,
// as the regular sweep) where two copies fit, else one CTA of 1024 threads.
// Measured on B200 it is not faster than the whole L1 for the gathers (the
// shared memory it takes is L1 the gathers lose), so it is off by default.
constexpr int kHotThreads = 1024;
constexpr int kHotThreadsPair = 768;
constexpr int kHotUnroll = 8;
// Largest tier: 224 KB of the 227 KB a CTA may opt into (the rest holds the
// block reduction's scratch).
constexpr uint32_t kHotMaxBytes = 224u * 1024u;

template <typename T, bool HOT, bool PART = false>
__device__ __forceinline__ T gather_y(const SweepArgs<T> &a, const T *s_y, uint32_t c) {
    if (HOT && c < a.hot)
        return s_y[c];
    return c != (PART ? a.pad : a.n) ? __ldg(a.y_in + c) : T(0);
}

// 16-byte read-only load that does not allocate in L1 (the tier copy).
__device__ __forceinline__ uint4 ld_na_v4(const uint4 *p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// Closes an iteration from the reduced residual sum r and sink mass s
// (PageRank.cpp:68-70): iteration count, stopping norm, trace, the sink term
// of the next sweep, the convergence flag. One thread, after every partial
// sum of the sweep is in r and s.
template <typename T>
__device__ __forceinline__ void close_iteration(const SweepArgs<T> &a, const RunParams &rp, double r,
                                                double s) {
    IterState *st = a.st;
    const unsigned long long it = st->iteration + 1;
    const double norm = rp.l2 ? sqrt(r) : r;
    st->iteration = it;
    st->residual = norm;
    st->residual_sum = r;
    if (it - 1 < a.trace_cap)
        a.trace[it - 1] = norm;
    st->sink_mass = s;
    st->sink_coef = rp.distribute ? (rp.personal ? s : s / static_cast<double>(a.n)) : 0.0;
    st->ticket = 0;
    st->queue = 0;
    __threadfence();
    st->done = (it >= rp.max_iterations || norm <= rp.tol) ? 1 : 0;
}

// Slices [s_begin, s_end) of one work unit: each lane accumulates one
// virtual row of a slice in arc order. Chunk slices store partial sums; row
// slices finish rows, adding their residual and sink terms to res / sink.
template <typename T, bool WEIGHTED, int UNROLL, bool HOT, bool PART>
__device__ __forceinline__ void sweep_unit(const SweepArgs<T> &a, const T *s_y, uint32_t s_begin,
                                           uint32_t s_end, int lane, double &res, double &sink) {
    for (uint32_t s = s_begin; s < s_end; ++s) {
        const uint32_t off = a.slice_off[s];
        const uint32_t len = a.slice_off[s + 1] - off;
        const size_t base = static_cast<size_t>(off) * 32 + lane;
        const uint32_t *cp = a.col_sell + base;
        T acc = T(0);
        uint32_t j = 0;
        for (; j + UNROLL <= len; j += UNROLL) {
            uint32_t c[UNROLL];
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                c[k] = ld_stream(cp + static_cast<size_t>(j + k) * 32);
            T v[UNROLL];
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                v[k] = gather_y<T, HOT, PART>(a, s_y, c[k]);
            if (WEIGHTED) {
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    v[k] = t_mul(v[k], ld_stream(a.w_sell + base + static_cast<size_t>(j + k) * 32));
            }
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                acc += v[k];
        }
        if (j < len) {
            // The last len - j < UNROLL steps as one predicated batch, so
            // their gathers are in flight together; the sum keeps the same
            // order (absent steps add nothing).
            uint32_t c[UNROLL];
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                c[k] = j + k < len ? ld_stream(cp + static_cast<size_t>(j + k) * 32) : 0u;
            T v[UNROLL];
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                v[k] = j + k < len ? gather_y<T, HOT, PART>(a, s_y, c[k]) : T(0);
            if (WEIGHTED) {
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    if (j + k < len)
                        v[k] = t_mul(v[k], ld_stream(a.w_sell + base + static_cast<size_t>(j + k) * 32));
            }
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                if (j + k < len)
                    acc += v[k];
        }
        if (s < a.s_chunk) {
            a.chunk_val[static_cast<size_t>(s) * 32 + lane] = acc;
        } else {
            const uint32_t r = a.n_long + (s - a.s_chunk) * 32 + lane;
            if (r < a.n)
                finish_row_sweep<T, WEIGHTED, PART>(a, r, acc, res, sink);
        }
    }
}

// The sweep: each warp walks its units (sweep_unit).
// Registers are fitted to 48 warps per SM (more warps do not make the sweep
// faster: it is bound by the rate of L1 miss requests), and to 32 for the
// other batch depths and the weighted FP64 sweep, which would spill at 48.
// HOT: the variant with the shared-memory tier (a.hot * sizeof(T) bytes of
// dynamic shared memory, a multiple of 16). PART: the row slice of a
// partitioned run (see SweepArgs.row_map).
// QUEUED: after a first unit of their own, warps take the next unit from a
// device counter (next_unit) instead of a fixed round-robin share, so warps
// that run faster take more of the graph and the sweep ends when the work
// does, not when the slowest share does (R-MAT 24, FP64: 0.874 ms against
// 0.956 ms with 8 round-robin units per warp, same scores bit for bit). Every unit's residual and sink partials go to their
// own slots (unit_res, unit_sink) after a fixed-order warp sum, and the
// fix-up adds them in a fixed order: the result does not depend on which
// warp ran which unit. The regular PageRank sweep and the row slices of a
// partitioned run are always QUEUED; the shared-memory tier keeps the
// round-robin units.
template <typename T, bool WEIGHTED, int THREADS, int UNROLL, bool HOT = false, bool PART = false,
          bool QUEUED = false>
__global__ void __launch_bounds__(THREADS, UNROLL != 8 || (WEIGHTED && sizeof(T) > 4) ? 1024 / THREADS : 1536 / THREADS)
    sweep_kernel(SweepArgs<T> a) {
    static_assert(!(QUEUED && HOT), "the queued sweep has no shared-memory tier");
    __shared__ double s_red[32];
    extern __shared__ __align__(16) unsigned char s_dyn[];
    T *s_y = reinterpret_cast<T *>(s_dyn);
    if (*(volatile int *)&a.st->done)
        return;
    const int lane = threadIdx.x & 31;
    if (QUEUED) {
        const uint32_t nw = gridDim.x * (THREADS / 32);
        for (uint32_t u = blockIdx.x * (THREADS / 32) + (threadIdx.x >> 5); u < a.units;
             u = next_unit(&a.st->queue, a.units, nw, lane)) {
            double res = 0.0, sink = 0.0;
            sweep_unit<T, WEIGHTED, UNROLL, false, PART>(a, s_y, a.unit_start[u],
                                                          a.unit_start[u + 1], lane, res, sink);
            res = warp_sum(res);
            sink = warp_sum(sink);
            if (lane == 0) {
                a.unit_res[u] = res;
                a.unit_sink[u] = sink;
                if (a.close_in_sweep)
                    __threadfence();  // visible to the CTA that closes the iteration
            }
        }
        if (!a.close_in_sweep)
            return;
        // The last CTA to finish adds the units' partials in unit order (a
        // fixed tree) and closes the iteration; no CTA waits for another.
        __shared__ bool s_last;
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            s_last = atomicAdd(&a.st->ticket, 1u) == gridDim.x - 1;
        }
        __syncthreads();
        if (!s_last)
            return;
        __threadfence();
        double r = 0.0, sk = 0.0;
        for (uint32_t i = threadIdx.x; i < a.units; i += THREADS) {
            r += ((volatile double *)a.unit_res)[i];
            sk += ((volatile double *)a.unit_sink)[i];
        }
        r = block_sum<THREADS>(r, s_red);
        sk = block_sum<THREADS>(sk, s_red);
        if (threadIdx.x == 0)
            close_iteration(a, *a.rp, r, sk);
        return;
    }
    if (HOT) {
        const uint32_t vecs = a.hot * static_cast<uint32_t>(sizeof(T)) / 16u;
        const uint4 *src = reinterpret_cast<const uint4 *>(a.y_in);
        uint4 *dst = reinterpret_cast<uint4 *>(s_dyn);
        for (uint32_t i = threadIdx.x; i < vecs; i += THREADS)
            dst[i] = ld_na_v4(src + i);
        __syncthreads();
    }
    const uint32_t wpc = THREADS / 32;
    const uint32_t gw = blockIdx.x * wpc + (threadIdx.x >> 5);
    const uint32_t nw = gridDim.x * wpc;
    double res = 0.0, sink = 0.0;
    for (uint32_t u = gw; u < a.units; u += nw)
        sweep_unit<T, WEIGHTED, UNROLL, HOT, PART>(a, s_y, a.unit_start[u], a.unit_start[u + 1],
                                                   lane, res, sink);
    const double bres = block_sum<THREADS>(res, s_red);
    const double bsink = block_sum<THREADS>(sink, s_red);
    if (threadIdx.x == 0) {
        a.cta_res[blockIdx.x] = bres;
        a.cta_sink[blockIdx.x] = bsink;
    }
}

// Fix-up: finish the split rows from their chunk sums (in chunk order), then
// (last CTA) reduce all partial sums in index order and close the iteration
// (PageRank.cpp:68-70). The first fix_vlong_ctas() CTAs finish the rows with
// many chunks, one row per warp; the others take one split row per thread.
constexpr int kFixThreads = 256;
constexpr uint32_t kFixWarps = kFixThreads / 32;

__host__ __device__ inline uint32_t fix_vlong_ctas(uint32_t n_vlong) {
    return (n_vlong + kFixWarps - 1) / kFixWarps;
}

// The same layout for the other fix-ups of split rows (FP32 product, adjoint,
// centrality), with THREADS threads per CTA: the first CTAs give each row of
// more than kShortChunks chunks a warp, the rest one thread per split row.
template <int THREADS>
inline unsigned split_fix_ctas(uint32_t n_long, uint32_t n_vlong) {
    constexpr uint32_t w = THREADS / 32;
    const uint64_t short_rows = n_long > n_vlong ? n_long - n_vlong : 0;
    return static_cast<unsigned>(std::max<uint64_t>(
        1, (n_vlong + w - 1) / w + (short_rows + THREADS - 1) / THREADS));
}

// Lane-strided partial sum of one split row's chunk partials
// v[cb + lane], v[cb + lane + 32], ... in ascending order, with 16 loads in
// flight at a time (a row has up to about a thousand chunks). Absent entries
// add zero, so the sum equals the one-at-a-time loop bit for bit.
template <typename V>
__device__ __forceinline__ V lane_chunk_sum(const V *__restrict__ v, uint32_t cb, uint32_t ce,
                                            int lane) {
    constexpr int kBatch = 16;
    V part = V(0);
    for (uint32_t k0 = cb + lane; k0 < ce; k0 += 32 * kBatch) {
        V x[kBatch];
#pragma unroll
        for (int q = 0; q < kBatch; ++q) {
            const uint32_t k = k0 + 32u * q;
            x[q] = k < ce ? v[k] : V(0);
        }
#pragma unroll
        for (int q = 0; q < kBatch; ++q)
            part += x[q];
    }
    return part;
}

// Split row r of this thread in that layout and its chunk sum. Returns true
// for the thread that finishes r (lane 0 of a row's warp, or the row's own
// thread). A warp sums lane-strided partials in V, then across lanes in double
// in a fixed tree; a thread sums the chunks in order. Every thread of a warp
// given a row must call it (the lane sum is warp-wide).
template <int THREADS, typename V>
__device__ __forceinline__ bool split_row_sum(const uint32_t *__restrict__ chunk_begin,
                                              const V *__restrict__ chunk_val, uint32_t n_long,
                                              uint32_t n_vlong, uint32_t &r, V &acc) {
    constexpr uint32_t w = THREADS / 32;
    const uint32_t vctas = (n_vlong + w - 1) / w;
    if (blockIdx.x < vctas) {
        r = blockIdx.x * w + (threadIdx.x >> 5);
        if (r >= n_vlong)
            return false;
        const int lane = threadIdx.x & 31;
        const V part = lane_chunk_sum(chunk_val, chunk_begin[r], chunk_begin[r + 1], lane);
        acc = static_cast<V>(warp_sum(static_cast<double>(part)));
        return lane == 0;
    }
    r = n_vlong + (blockIdx.x - vctas) * THREADS + threadIdx.x;
    if (r >= n_long)
        return false;
    V sum = V(0);
    for (uint32_t k = chunk_begin[r]; k < chunk_begin[r + 1]; ++k)
        sum += chunk_val[k];
    acc = sum;
    return true;
}

template <typename T, bool WEIGHTED, bool PART = false>
__global__ void __launch_bounds__(kFixThreads) fixup_kernel(SweepArgs<T> a) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    if (*(volatile int *)&a.st->done)
        return;
    const RunParams rp = *a.rp;
    const T sink_coef = static_cast<T>(a.st->sink_coef);
    double res = 0.0, sink = 0.0;
    if (a.unit_res) {
        // Partials of a queued sweep: a fixed share of the units per thread.
        for (uint32_t i = blockIdx.x * kFixThreads + threadIdx.x; i < a.units;
             i += gridDim.x * kFixThreads) {
            res += a.unit_res[i];
            sink += a.unit_sink[i];
        }
    }
    const uint32_t vctas = fix_vlong_ctas(a.n_vlong);
    if (blockIdx.x < vctas) {
        const uint32_t r = blockIdx.x * kFixWarps + (threadIdx.x >> 5);
        const int lane = threadIdx.x & 31;
        if (r < a.n_vlong) {
            const T part = lane_chunk_sum<T>(a.chunk_val, a.chunk_begin[r], a.chunk_begin[r + 1], lane);
            const double tot = warp_sum(static_cast<double>(part));
            if (lane == 0)
                finish_row<T, WEIGHTED, PART>(a, rp, sink_coef, r, static_cast<T>(tot), res, sink);
        }
    } else {
        const uint32_t r = a.n_vlong + (blockIdx.x - vctas) * kFixThreads + threadIdx.x;
        if (r < a.n_long) {
            const uint32_t cb = a.chunk_begin[r], ce = a.chunk_begin[r + 1];
            T parts[kShortChunks];
#pragma unroll
            for (uint32_t k = 0; k < kShortChunks; ++k)
                parts[k] = cb + k < ce ? a.chunk_val[cb + k] : T(0);
            T sum = T(0);
#pragma unroll
            for (uint32_t k = 0; k < kShortChunks; ++k)
                sum += parts[k];
            finish_row<T, WEIGHTED, PART>(a, rp, sink_coef, r, sum, res, sink);
        }
    }
    const double bres = block_sum<kFixThreads>(res, s_red);
    const double bsink = block_sum<kFixThreads>(sink, s_red);
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
    const uint32_t sweep_parts = a.unit_res ? 0u : a.sweep_ctas;
    for (uint32_t i = threadIdx.x; i < sweep_parts; i += kFixThreads) {
        r += ((volatile double *)a.cta_res)[i];
        s += ((volatile double *)a.cta_sink)[i];
    }
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kFixThreads) {
        r += ((volatile double *)a.fix_res)[i];
        s += ((volatile double *)a.fix_sink)[i];
    }
    r = block_sum<kFixThreads>(r, s_red);
    s = block_sum<kFixThreads>(s, s_red);
    if (threadIdx.x == 0)
        close_iteration(a, rp, r, s);
}

} // namespace nkg
