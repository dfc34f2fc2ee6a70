// Differentiable PageRank: the adjoint (backward) solve, the gradients with
// respect to the arc weights and the teleport vector, and in-place weight
// updates. No reference counterpart; the forward it differentiates is
// PageRank.cpp:20-104 on a weighted graph (optionally distributeSinks and a
// personalised teleport).
//
// Forward fixed point, with t the teleport distribution (1/n without one), m
// the sink mask and A[u,v] = w(v->u)/wdeg[v]:
//     x = d (A x + [distributeSinks] (m.x) t) + (1-d) t,    p = x / sum(x).
// For a loss L with g = dL/dp, with gbar = g - (g.p) 1, the adjoint lam solves
//     (I - d M^T) lam = gbar,   M^T q = A^T q + [distributeSinks] m (t.q),
// and, with c = A^T lam (c[v] = sum_{v->u} w lam[u] / wdeg[v]),
//     dL/dw(v->u) = d (p[v] / wdeg[v]) (lam[u] - c[v])
//     dL/dt[u]    = (d [distributeSinks] m.p + (1-d) / sum(x)) lam[u]
// where sum(x) follows from p alone at the fixed point (summing the forward
// equation over all nodes, tau = sum(t)):
//     sum(x) = (1-d) tau / (1 - d + d (m.p) (1 - [distributeSinks] tau)).
// (This lam is sum(x) times the lam of the un-normalised system, which is why
// neither gradient needs sum(x) beyond that one factor.)
//
// A^T is a pull over the out-adjacency, so the graph gets a second sliced
// layout: the out-CSR, its rows ("out-rows") the nodes sorted by out-degree,
// descending, each listing its out-arcs in the order they appear in the
// in-CSR, its column ids out-row numbers. Every vector of the adjoint solve
// is indexed by out-row, so rows are written in place and only the gathers
// are scattered. The FP32 solve is the BiCGSTAB of refine.cuh with OP = 1;
// the FP64 Jacobi sweep below gives the refinement's residual, the FP64 solve
// and the final c. dL/dw is then one pass over the in-adjacency's sliced
// layout, written straight into the caller's arc order.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>

#include "graph.hpp"
#include "host.hpp"
#include "refine.cuh"

namespace nkg {

// Work buffers of one backward pass, kept between calls (sized for n).
struct AdjWork {
    DeviceArray<double> p, g, t, gbar, c, part, fix_part, chunk64, lam_f, lam[2];
    DeviceArray<double2> qc;
    DeviceArray<float> t32, chunk32, x, r, rhat, pv, v, sv, tv;
    DeviceArray<unsigned char> scal;  // AdjScalars, BiScalars, AdjState
    bool ready = false;
};

struct AdjointState {
    SellLayout tl;                  // out-adjacency, rows = out-rows
    DeviceArray<uint32_t> trow;     // n: relabelled id of out-row rt
    DeviceArray<uint32_t> tinv;     // n: out-row of relabelled id v
    DeviceArray<uint32_t> tperm;    // n: caller id of out-row rt
    DeviceArray<uint32_t> tdegc;    // n: out-degree of out-row rt
    DeviceArray<uint32_t> tptr;     // n+1: out-CSR offsets
    DeviceArray<uint32_t> tarc;     // arcs: in-CSR entry of every out-CSR entry
    DeviceArray<double> tdegw64;    // n: weighted out-degree (weighted graphs)
    DeviceArray<float> tdegw32;     // n
    DeviceArray<float> w_sell32;    // slots (weighted graphs)
    DeviceArray<uint32_t> units32, units64;
    uint32_t n_units32 = 0, n_units64 = 0;
    unsigned ctas32 = 0, ctas64 = 0;
    int shape = -1;
    // dL/dw pass: source and row (relabelled) of every arc in the caller's
    // order, and the grid of that pass.
    DeviceArray<uint32_t> gw_src, gw_row;
    unsigned gw_ctas = 0;
    // Weight updates: caller arc index of every slot (kNone for padding) of
    // the in-layout and of the out-layout; chunk partial sums of out-degrees.
    DeviceArray<uint32_t> fw_map, t_map;
    DeviceArray<double> tchunk;
    AdjWork work;
};

void destroy_adjoint(AdjointState *a) { delete a; }

namespace {

constexpr int kAdjThreads = 256;

// ---------------------------------------------------------------------------
// Layout build kernels

__global__ void adj_outdeg_keys(const uint32_t *__restrict__ degc, uint32_t n,
                                uint32_t *__restrict__ keys, uint32_t *__restrict__ ids) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) {
        keys[r] = degc[r];
        ids[r] = r;
    }
}

__global__ void adj_row_info(const uint32_t *__restrict__ trow, const uint32_t *__restrict__ degc,
                             const uint32_t *__restrict__ perm, const double *__restrict__ degw,
                             uint32_t n, uint32_t *__restrict__ tdegc, uint32_t *__restrict__ tinv,
                             uint32_t *__restrict__ tperm, double *__restrict__ tdegw) {
    const uint32_t rt = blockIdx.x * blockDim.x + threadIdx.x;
    if (rt < n) {
        const uint32_t v = trow[rt];
        tdegc[rt] = degc[v];
        tinv[v] = rt;
        tperm[rt] = perm[v];
        if (tdegw)
            tdegw[rt] = degw[v];
    }
}

// Per in-arc k (row u, source v): sort key = out-row of v, value = k; and the
// out-row of its target u. One warp per in-row.
__global__ void adj_arc_keys(const uint32_t *__restrict__ row_ptr, const uint32_t *__restrict__ col,
                             const uint32_t *__restrict__ tinv, uint32_t n,
                             uint32_t *__restrict__ key, uint32_t *__restrict__ val,
                             uint32_t *__restrict__ arc_row) {
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint64_t u = warp; u < n; u += nwarps) {
        const uint32_t b = row_ptr[u], e = row_ptr[u + 1];
        const uint32_t ut = tinv[u];
        for (uint32_t k = b + lane; k < e; k += 32) {
            key[k] = tinv[col[k]];
            val[k] = k;
            arc_row[k] = ut;
        }
    }
}

// out[k] = src[idx[k]]
__global__ void adj_gather_u32(const uint32_t *__restrict__ idx, const uint32_t *__restrict__ src,
                               uint64_t m, uint32_t *__restrict__ out) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < m;
         k += stride)
        out[k] = src[idx[k]];
}

// Caller arc index of every in-CSR entry (row r starts at row_src[r] there).
__global__ void adj_caller_index(const uint32_t *__restrict__ row_ptr,
                                 const uint64_t *__restrict__ row_src, uint32_t n,
                                 uint32_t *__restrict__ out) {
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint64_t r = warp; r < n; r += nwarps) {
        const uint32_t b = row_ptr[r], e = row_ptr[r + 1];
        const uint64_t src = row_src[r];
        for (uint32_t k = b + lane; k < e; k += 32)
            out[k] = static_cast<uint32_t>(src + (k - b));
    }
}

// ---------------------------------------------------------------------------
// Weight updates

// w64[slot] = w[map[slot]] (0 for padding), and its FP32 copy.
__global__ void adj_refresh_slots(const uint32_t *__restrict__ map, uint64_t slots,
                                  const double *__restrict__ w, double *__restrict__ w64,
                                  float *__restrict__ w32) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < slots;
         k += stride) {
        const uint32_t m = map[k];
        const double v = m != kNone ? w[m] : 0.0;
        w64[k] = v;
        if (w32)
            w32[k] = static_cast<float>(v);
    }
}

struct DegreeOut {
    const uint32_t *trow;
    double *tdegw64;
    float *tdegw32;
    double *degw64;  // relabelled order (the forward's)
    float *degw32;   // relabelled order, FP32 plane (or null)
};

__device__ __forceinline__ void put_degree(const DegreeOut &o, uint32_t rt, double d) {
    o.tdegw64[rt] = d;
    o.tdegw32[rt] = static_cast<float>(d);
    const uint32_t v = o.trow[rt];
    o.degw64[v] = d;
    if (o.degw32)
        o.degw32[v] = static_cast<float>(d);
}

// Weighted out-degrees from the out-layout's slot weights: every lane sums its
// virtual row in slot order (padding weighs 0); split rows keep chunk sums.
__global__ void adj_degree_sums(const uint32_t *__restrict__ slice_off,
                                const double *__restrict__ w64, uint32_t slices, uint32_t s_chunk,
                                uint32_t n_long, uint32_t n, double *__restrict__ tchunk,
                                DegreeOut o) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint32_t s = warp; s < slices; s += nwarps) {
        const uint32_t off = slice_off[s], len = slice_off[s + 1] - off;
        const double *wp = w64 + static_cast<size_t>(off) * 32 + lane;
        double sum = 0.0;
        uint32_t j = 0;
        for (; j + 8 <= len; j += 8) {
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k)
                v[k] = wp[static_cast<size_t>(j + k) * 32];
#pragma unroll
            for (int k = 0; k < 8; ++k)
                sum += v[k];
        }
        for (; j < len; ++j)
            sum += wp[static_cast<size_t>(j) * 32];
        if (s < s_chunk) {
            tchunk[static_cast<size_t>(s) * 32 + lane] = sum;
        } else {
            const uint32_t r = n_long + (s - s_chunk) * 32 + lane;
            if (r < n)
                put_degree(o, r, sum);
        }
    }
}

__global__ void adj_degree_fix(const uint32_t *__restrict__ chunk_begin, uint32_t n_long,
                               const double *__restrict__ tchunk, DegreeOut o) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_long)
        return;
    double sum = 0.0;
    for (uint32_t k = chunk_begin[r]; k < chunk_begin[r + 1]; ++k)
        sum += tchunk[k];
    put_degree(o, r, sum);
}

// Weighted out-degrees given by the caller (caller ids).
__global__ void adj_degree_given(const double *__restrict__ wdeg, const uint32_t *__restrict__ tperm,
                                 uint32_t n, DegreeOut o) {
    const uint32_t rt = blockIdx.x * blockDim.x + threadIdx.x;
    if (rt < n)
        put_degree(o, rt, wdeg[tperm[rt]]);
}

// ---------------------------------------------------------------------------
// FP64 Jacobi sweep of the adjoint system (out-row order)

struct AdjState {
    double tdot;               // tel.lam_in (uniform teleport: times 1/n)
    double residual;           // L1 norm of lam_out - lam_in
    unsigned long long iteration;
    int done;
    unsigned int ticket;
};

struct AdjArgs {
    const uint32_t *__restrict__ col_sell;
    const double *__restrict__ w_sell;
    const uint32_t *__restrict__ slice_off;
    const uint32_t *__restrict__ unit_start;
    const uint32_t *__restrict__ chunk_begin;
    const uint32_t *__restrict__ degc;
    const double *__restrict__ degw;
    const double *__restrict__ tele;      // teleport or null
    const double *__restrict__ gbar;
    const double *__restrict__ lam_in;    // n+1, lam_in[n] = 0
    double *__restrict__ lam_out;         // n+1 or null (c only)
    double *__restrict__ c_out;           // n or null
    double *__restrict__ chunk_val;
    double *__restrict__ part;            // 2 per work unit of the sweep
    double *__restrict__ fix_part;        // 2 per fix-up CTA
    AdjState *st;
    unsigned int *queue;                  // next work unit of the sweep (reset by adj_fix)
    double damp, inv_n, tol;
    unsigned long long max_iter;
    uint32_t n, n_long, n_vlong, s_chunk, units, sweep_ctas;
    int distribute, personal;
};

template <bool WEIGHTED>
__device__ __forceinline__ void adj_row(const AdjArgs &a, uint32_t v, double acc, double tdot,
                                        double &res, double &td) {
    const uint32_t dc = a.degc[v];
    const double deg = WEIGHTED ? a.degw[v] : static_cast<double>(dc);
    const double c = dc ? acc / deg : 0.0;
    if (a.c_out)
        a.c_out[v] = c;
    if (a.lam_out) {
        const double lnew = a.gbar[v] + a.damp * (c + (a.distribute && !dc ? tdot : 0.0));
        a.lam_out[v] = lnew;
        res += fabs(lnew - a.lam_in[v]);
        td += a.personal ? a.tele[v] * lnew : lnew;
    }
}

template <bool WEIGHTED, int THREADS, int UNROLL>
__global__ void __launch_bounds__(THREADS, UNROLL > 8 ? 512 / THREADS : WEIGHTED ? 1024 / THREADS : 1536 / THREADS)
    adj_sweep(AdjArgs a) {
    if (*(volatile int *)&a.st->done)
        return;
    const double tdot = a.st->tdot;
    const int lane = threadIdx.x & 31;
    // Warps take units from a device counter in order (as the queued
    // PageRank sweep); every unit's two partial sums go to their own slots.
    const uint32_t nw = gridDim.x * (THREADS / 32);
    for (uint32_t u = blockIdx.x * (THREADS / 32) + (threadIdx.x >> 5); u < a.units;
         u = next_unit(a.queue, a.units, nw, lane)) {
        double res = 0.0, td = 0.0;
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
                double v[UNROLL];
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    v[k] = c[k] != a.n ? __ldg(a.lam_in + c[k]) : 0.0;
                if (WEIGHTED) {
#pragma unroll
                    for (int k = 0; k < UNROLL; ++k)
                        v[k] *= ld_stream(a.w_sell + base + static_cast<size_t>(j + k) * 32);
                }
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    acc += v[k];
            }
            if (j < len) {
                // the last len - j < UNROLL steps as one predicated batch (same order)
                uint32_t c[UNROLL];
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    c[k] = j + k < len ? ld_stream(cp + static_cast<size_t>(j + k) * 32) : 0u;
                double v[UNROLL];
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    v[k] = j + k < len && c[k] != a.n ? __ldg(a.lam_in + c[k]) : 0.0;
                if (WEIGHTED) {
#pragma unroll
                    for (int k = 0; k < UNROLL; ++k)
                        if (j + k < len)
                            v[k] *= ld_stream(a.w_sell + base + static_cast<size_t>(j + k) * 32);
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
                    adj_row<WEIGHTED>(a, r, acc, tdot, res, td);
            }
        }
        res = warp_sum(res);
        td = warp_sum(td);
        if (lane == 0) {
            a.part[2 * static_cast<size_t>(u)] = res;
            a.part[2 * static_cast<size_t>(u) + 1] = td;
        }
    }
}

// Split out-rows (one thread each, chunks in order), then the last CTA
// closes the sweep: residual, tel.lam_out for the next sweep, stopping test.
template <bool WEIGHTED>
__global__ void __launch_bounds__(kAdjThreads) adj_fix(AdjArgs a) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    if (*(volatile int *)&a.st->done)
        return;
    const double tdot = a.st->tdot;
    double res = 0.0, td = 0.0;
    // The sweep's unit partials: a fixed share of the units per thread.
    for (uint32_t i = blockIdx.x * kAdjThreads + threadIdx.x; i < a.units;
         i += gridDim.x * kAdjThreads) {
        res += a.part[2 * static_cast<size_t>(i)];
        td += a.part[2 * static_cast<size_t>(i) + 1];
    }
    uint32_t r;
    double acc;
    if (split_row_sum<kAdjThreads>(a.chunk_begin, a.chunk_val, a.n_long, a.n_vlong, r, acc))
        adj_row<WEIGHTED>(a, r, acc, tdot, res, td);
    res = block_sum<kAdjThreads>(res, s_red);
    td = block_sum<kAdjThreads>(td, s_red);
    if (threadIdx.x == 0) {
        a.fix_part[2 * blockIdx.x] = res;
        a.fix_part[2 * blockIdx.x + 1] = td;
    }
    if (!bi_last_block(&a.st->ticket, &s_last))
        return;
    double t1 = 0.0, t2 = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kAdjThreads) {
        t1 += ((volatile double *)a.fix_part)[2 * i];
        t2 += ((volatile double *)a.fix_part)[2 * i + 1];
    }
    t1 = block_sum<kAdjThreads>(t1, s_red);
    t2 = block_sum<kAdjThreads>(t2, s_red);
    if (threadIdx.x == 0) {
        AdjState *st = a.st;
        const unsigned long long it = st->iteration + 1;
        st->iteration = it;
        if (a.lam_out) {
            st->residual = t1;
            st->tdot = a.personal ? t2 : t2 * a.inv_n;
        }
        st->ticket = 0;
        *a.queue = 0;
        __threadfence();
        st->done = (it >= a.max_iter || t1 <= a.tol) ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// Inputs, right-hand side, gradients

// Scalars of one backward pass (FP64, device).
struct AdjScalars {
    double gp;      // g.p
    double sp;      // m.p
    double tau;     // sum of the teleport (1 without one)
    double gnorm;   // |gbar|_1
    double sumx;    // sum(x) of the forward fixed point
    double tfac;    // dL/dt = tfac * lam
    unsigned int ticket;
};

// p, g (and the teleport) into out-row order; g.p, m.p and sum(t); the
// scalars that follow from them.
__global__ void __launch_bounds__(kAdjThreads)
    adj_inputs(const double *__restrict__ scores, const double *__restrict__ grad,
               const double *__restrict__ tele_orig, const uint32_t *__restrict__ tperm,
               const uint32_t *__restrict__ tdegc, uint32_t n, double damp, int distribute,
               double *__restrict__ p_t, double *__restrict__ g_t, double *__restrict__ t_t,
               float *__restrict__ t32, double *__restrict__ part, AdjScalars *sc) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    double gp = 0.0, sp = 0.0, tau = 0.0;
    for (uint32_t r = blockIdx.x * kAdjThreads + threadIdx.x; r < n; r += gridDim.x * kAdjThreads) {
        const uint32_t o = tperm[r];
        const double pv = scores[o], gv = grad[o];
        p_t[r] = pv;
        g_t[r] = gv;
        gp += gv * pv;
        if (tdegc[r] == 0)
            sp += pv;
        if (tele_orig) {
            const double t = tele_orig[o];
            t_t[r] = t;
            t32[r] = static_cast<float>(t);
            tau += t;
        }
    }
    gp = block_sum<kAdjThreads>(gp, s_red);
    sp = block_sum<kAdjThreads>(sp, s_red);
    tau = block_sum<kAdjThreads>(tau, s_red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = gp;
        part[3 * blockIdx.x + 1] = sp;
        part[3 * blockIdx.x + 2] = tau;
    }
    if (!bi_last_block(&sc->ticket, &s_last))
        return;
    double t1 = 0.0, t2 = 0.0, t3 = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kAdjThreads) {
        t1 += ((volatile double *)part)[3 * i];
        t2 += ((volatile double *)part)[3 * i + 1];
        t3 += ((volatile double *)part)[3 * i + 2];
    }
    t1 = block_sum<kAdjThreads>(t1, s_red);
    t2 = block_sum<kAdjThreads>(t2, s_red);
    t3 = block_sum<kAdjThreads>(t3, s_red);
    if (threadIdx.x == 0) {
        sc->gp = t1;
        sc->sp = t2;
        const double tau_v = tele_orig ? t3 : 1.0;
        sc->tau = tau_v;
        const double denom = 1.0 - damp + damp * t2 * (1.0 - (distribute ? tau_v : 0.0));
        const double sumx = (1.0 - damp) * tau_v / denom;
        sc->sumx = sumx;
        sc->tfac = (distribute ? damp * t2 : 0.0) + (1.0 - damp) / sumx;
        sc->ticket = 0;
    }
}

// gbar = g - (g.p) 1 (FP64 and FP32 copies), lam0 = gbar, |gbar|_1 and the
// sweep state of lam0 (tel.gbar, not done).
__global__ void __launch_bounds__(kAdjThreads)
    adj_rhs(const double *__restrict__ g_t, const double *__restrict__ t_t, uint32_t n,
            int personal, double inv_n, double *__restrict__ gbar, float *__restrict__ r32,
            double *__restrict__ lam0, double *__restrict__ part, AdjScalars *sc, AdjState *st) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    const double gp = sc->gp;
    double nrm = 0.0, td = 0.0;
    for (uint32_t r = blockIdx.x * kAdjThreads + threadIdx.x; r < n; r += gridDim.x * kAdjThreads) {
        const double b = g_t[r] - gp;
        gbar[r] = b;
        r32[r] = static_cast<float>(b);
        lam0[r] = b;
        nrm += fabs(b);
        td += personal ? t_t[r] * b : b;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        lam0[n] = 0.0;
    nrm = block_sum<kAdjThreads>(nrm, s_red);
    td = block_sum<kAdjThreads>(td, s_red);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = nrm;
        part[2 * blockIdx.x + 1] = td;
    }
    if (!bi_last_block(&sc->ticket, &s_last))
        return;
    double t1 = 0.0, t2 = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kAdjThreads) {
        t1 += ((volatile double *)part)[2 * i];
        t2 += ((volatile double *)part)[2 * i + 1];
    }
    t1 = block_sum<kAdjThreads>(t1, s_red);
    t2 = block_sum<kAdjThreads>(t2, s_red);
    if (threadIdx.x == 0) {
        sc->gnorm = t1;
        st->tdot = personal ? t2 : t2 * inv_n;
        st->residual = 0.0;
        st->iteration = 0;
        st->done = 0;
        st->ticket = 0;
        sc->ticket = 0;
    }
}

// lam64 = x32 (add = 0) or lam64 += x32 (add = 1), lam64[n] = 0, and the
// sweep state for lam64 (tel.lam64; not done).
__global__ void __launch_bounds__(kAdjThreads)
    adj_to_fp64(const float *__restrict__ x32, double *__restrict__ lam, const double *t_t,
                uint32_t n, int add, int personal, double inv_n, double *__restrict__ part,
                unsigned int *ticket, AdjState *st) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    double td = 0.0;
    for (uint32_t r = blockIdx.x * kAdjThreads + threadIdx.x; r < n; r += gridDim.x * kAdjThreads) {
        const double v = add ? lam[r] + static_cast<double>(x32[r]) : static_cast<double>(x32[r]);
        lam[r] = v;
        td += personal ? t_t[r] * v : v;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        lam[n] = 0.0;
    td = block_sum<kAdjThreads>(td, s_red);
    if (threadIdx.x == 0)
        part[blockIdx.x] = td;
    if (!bi_last_block(ticket, &s_last))
        return;
    double t = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kAdjThreads)
        t += ((volatile double *)part)[i];
    t = block_sum<kAdjThreads>(t, s_red);
    if (threadIdx.x == 0) {
        st->tdot = personal ? t : t * inv_n;
        st->iteration = 0;
        st->done = 0;
        st->ticket = 0;
        *ticket = 0;
    }
}

// Right-hand side of a correction solve: r32 = lam_out - lam_in.
__global__ void adj_residual_rhs(const double *__restrict__ lam_out,
                                 const double *__restrict__ lam_in, uint32_t n,
                                 float *__restrict__ r32) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n)
        r32[r] = static_cast<float>(lam_out[r] - lam_in[r]);
}

// Into the relabelled (in-layout) order: lam_f[v] = lam[tinv[v]] and the pair
// qc[v] = (d p[v] / wdeg[v], c[v]) that every out-arc of v reads; qc[n] = 0
// for the padding slots.
template <bool WEIGHTED>
__global__ void adj_to_forward(const uint32_t *__restrict__ tinv, const double *__restrict__ lam_t,
                               const double *__restrict__ c_t, const double *__restrict__ p_t,
                               const uint32_t *__restrict__ tdegc, const double *__restrict__ tdegw,
                               uint32_t n, double damp, double *__restrict__ lam_f,
                               double2 *__restrict__ qc) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v > n)
        return;
    if (v == n) {
        qc[n] = make_double2(0.0, 0.0);
        return;
    }
    const uint32_t rt = tinv[v];
    lam_f[v] = lam_t[rt];
    const uint32_t dc = tdegc[rt];
    const double deg = WEIGHTED ? tdegw[rt] : static_cast<double>(dc);
    qc[v] = make_double2(dc ? damp * (p_t[rt] / deg) : 0.0, c_t[rt]);
}

constexpr int kGradThreads = 256;

// The arcs in the caller's order: source (relabelled) and row (relabelled)
// of caller arc e, scattered once from the relabelled in-CSR (one warp per row).
__global__ void adj_caller_arcs(const uint32_t *__restrict__ row_ptr,
                                const uint64_t *__restrict__ row_src,
                                const uint32_t *__restrict__ col, uint32_t n,
                                uint32_t *__restrict__ src_c, uint32_t *__restrict__ row_c) {
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint64_t r = warp; r < n; r += nwarps) {
        const uint32_t b = row_ptr[r], e = row_ptr[r + 1];
        const uint64_t dst = row_src[r];
        for (uint32_t k = b + lane; k < e; k += 32) {
            src_c[dst + (k - b)] = col[k];
            row_c[dst + (k - b)] = static_cast<uint32_t>(r);
        }
    }
}


// dL/dw in the caller's arc order: arc e (source v, row u) gets
// qc[v].x (lam[u] - qc[v].y). Index reads and stores are coalesced; the pair
// qc[v] is the one scattered load per arc (lam[u] repeats along a row).
__global__ void __launch_bounds__(kGradThreads)
    adj_grad_w(const uint32_t *__restrict__ src_c, const uint32_t *__restrict__ row_c,
               const double *__restrict__ lam_f, const double2 *__restrict__ qc, uint64_t arcs,
               double *__restrict__ grad_w) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * kGradThreads;
    uint64_t e = blockIdx.x * static_cast<uint64_t>(kGradThreads) + threadIdx.x;
    for (; e + 3 * stride < arcs; e += 4 * stride) {
        uint32_t v[4], u[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = ld_stream(src_c + e + k * stride);
            u[k] = ld_stream(row_c + e + k * stride);
        }
        double2 q[4];
        double l[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            q[k] = __ldg(qc + v[k]);
            l[k] = __ldg(lam_f + u[k]);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
            __stcs(grad_w + e + k * stride, q[k].x * (l[k] - q[k].y));
    }
    for (; e < arcs; e += stride) {
        const double2 q = __ldg(qc + ld_stream(src_c + e));
        __stcs(grad_w + e, q.x * (__ldg(lam_f + ld_stream(row_c + e)) - q.y));
    }
}

// dL/dt in the caller's ids (0 for ids of deleted nodes).
__global__ void adj_grad_t(const uint32_t *__restrict__ inv, const uint32_t *__restrict__ tinv,
                           uint64_t z, const double *__restrict__ lam_t,
                           const AdjScalars *sc, double *__restrict__ grad_t) {
    const uint64_t o = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (o >= z)
        return;
    const uint32_t r = inv[o];
    grad_t[o] = r == kNone ? 0.0 : sc->tfac * lam_t[tinv[r]];
}

} // namespace

// ---------------------------------------------------------------------------
// Host side

AdjointState &adjoint_ensure(nkg_graph *g) {
    if (g->adj)
        return *g->adj;
    require(!g->arc_sorted,
            "the adjoint needs the in-rows in the caller's arc order (arc_order 0)");
    require(!g->w64src_stale, "internal: CSR weights out of date");
    cudaStream_t s = g->stream;
    const uint32_t n = static_cast<uint32_t>(g->n);
    const uint64_t arcs = g->arcs;
    const unsigned sms = num_sms(g->device);
    std::unique_ptr<AdjointState> A(new AdjointState());

    // Out-rows: nodes by out-degree, descending (stable: ties by node).
    {
        DeviceArray<uint32_t> keys(n), ids(n), keys_s(n);
        A->trow.alloc(n);
        adj_outdeg_keys<<<ceil_div(n, 256), 256, 0, s>>>(g->degc.get(), n, keys.get(), ids.get());
        NKG_CUDA(cudaGetLastError());
        size_t tb = 0;
        NKG_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, keys.get(), keys_s.get(),
                                                           ids.get(), A->trow.get(),
                                                           static_cast<int64_t>(n), 0, 32, s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.get(), tb, keys.get(), keys_s.get(),
                                                           ids.get(), A->trow.get(),
                                                           static_cast<int64_t>(n), 0, 32, s));
    }
    A->tinv.alloc(n);
    A->tperm.alloc(n);
    A->tdegc.alloc(n);
    if (g->weighted) {
        A->tdegw64.alloc(n);
        A->tdegw32.alloc(n);
    }
    adj_row_info<<<ceil_div(n, 256), 256, 0, s>>>(A->trow.get(), g->degc.get(), g->perm.get(),
                                                  g->degw64src.get(), n, A->tdegc.get(),
                                                  A->tinv.get(), A->tperm.get(), A->tdegw64.get());
    NKG_CUDA(cudaGetLastError());
    A->tptr.alloc(static_cast<size_t>(n) + 1);
    NKG_CUDA(cudaMemsetAsync(A->tptr.get(), 0, sizeof(uint32_t), s));
    {
        size_t tb = 0;
        NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, A->tdegc.get(), A->tptr.get() + 1,
                                               static_cast<int64_t>(n), s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb, A->tdegc.get(), A->tptr.get() + 1,
                                               static_cast<int64_t>(n), s));
    }

    // Group the in-arcs by out-row (stable: in-CSR order inside a row).
    A->tarc.alloc(std::max<uint64_t>(arcs, 1));
    DeviceArray<uint32_t> tcol(std::max<uint64_t>(arcs, 1));
    if (arcs) {
        DeviceArray<uint32_t> key(arcs), key_s(arcs), val(arcs), arc_row(arcs);
        adj_arc_keys<<<sms * 16, 256, 0, s>>>(g->row_ptr.get(), g->col.get(), A->tinv.get(), n,
                                              key.get(), val.get(), arc_row.get());
        NKG_CUDA(cudaGetLastError());
        int bits = 1;
        while (bits < 32 && (1ull << bits) < n)
            ++bits;
        size_t tb = 0;
        NKG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.get(), key_s.get(), val.get(),
                                                 A->tarc.get(), static_cast<int64_t>(arcs), 0, bits,
                                                 s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, key.get(), key_s.get(), val.get(),
                                                 A->tarc.get(), static_cast<int64_t>(arcs), 0, bits,
                                                 s));
        adj_gather_u32<<<sms * 8, 256, 0, s>>>(A->tarc.get(), arc_row.get(), arcs, tcol.get());
        NKG_CUDA(cudaGetLastError());
        NKG_CUDA(cudaStreamSynchronize(s));
    }
    build_sell(A->tl, n, A->tptr.get(), tcol.get(), g->weighted ? g->w64src.get() : nullptr,
               A->tarc.get(), A->tdegc.get(), g->device, s);
    if (g->weighted) {
        A->w_sell32.alloc(A->tl.slots, 4);
        convert_to_float(A->tl.w_sell64.get(), A->w_sell32.get(), A->tl.slots, g->device, s);
        convert_to_float(A->tdegw64.get(), A->tdegw32.get(), n, g->device, s);
    }
    NKG_CUDA(cudaStreamSynchronize(s));
    g->adj.reset(A.release());
    return *g->adj;
}

OutLayoutView adjoint_out_layout(nkg_graph *g) {
    AdjointState &A = adjoint_ensure(g);
    return OutLayoutView{&A.tl, A.tinv.get()};
}

namespace {

// Slot -> caller arc maps of both layouts (first weight update only).
void ensure_weight_maps(nkg_graph *g, AdjointState &A) {
    if (A.fw_map)
        return;
    cudaStream_t s = g->stream;
    const uint32_t n = static_cast<uint32_t>(g->n);
    const unsigned sms = num_sms(g->device);
    DeviceArray<uint32_t> caller(std::max<uint64_t>(g->arcs, 1)), tcaller(std::max<uint64_t>(g->arcs, 1));
    if (g->arcs) {
        adj_caller_index<<<sms * 16, 256, 0, s>>>(g->row_ptr.get(), g->row_src.get(), n,
                                                  caller.get());
        adj_gather_u32<<<sms * 8, 256, 0, s>>>(A.tarc.get(), caller.get(), g->arcs, tcaller.get());
        NKG_CUDA(cudaGetLastError());
    }
    A.fw_map.alloc(std::max<uint64_t>(g->fw.slots, 1));
    A.t_map.alloc(std::max<uint64_t>(A.tl.slots, 1));
    build_slot_map(g->fw, n, g->row_ptr.get(), caller.get(), A.fw_map.get(), g->device, s);
    build_slot_map(A.tl, n, A.tptr.get(), tcaller.get(), A.t_map.get(), g->device, s);
    A.tchunk.alloc(static_cast<size_t>(A.tl.s_chunk) * 32 + 1);
    NKG_CUDA(cudaStreamSynchronize(s));
}

} // namespace

// Replace the arc weights (and weighted out-degrees) in place: every buffer
// keeps its address, so captured sweep graphs stay valid. w and wdeg are
// device arrays in the caller's order (wdeg may be null).
void set_weights_device(nkg_graph *g, const double *w, const double *wdeg) {
    AdjointState &A = adjoint_ensure(g);
    ensure_weight_maps(g, A);
    cudaStream_t s = g->stream;
    const uint32_t n = static_cast<uint32_t>(g->n);
    const unsigned sms = num_sms(g->device);
    if (g->fw.slots)
        adj_refresh_slots<<<sms * 8, 256, 0, s>>>(A.fw_map.get(), g->fw.slots, w,
                                                  g->fw.w_sell64.get(), g->p32.w_sell.get());
    if (A.tl.slots)
        adj_refresh_slots<<<sms * 8, 256, 0, s>>>(A.t_map.get(), A.tl.slots, w,
                                                  A.tl.w_sell64.get(), A.w_sell32.get());
    NKG_CUDA(cudaGetLastError());
    DegreeOut o{A.trow.get(), A.tdegw64.get(), A.tdegw32.get(), g->degw64src.get(),
                g->p32.degw.get()};
    if (wdeg) {
        adj_degree_given<<<ceil_div(n, 256), 256, 0, s>>>(wdeg, A.tperm.get(), n, o);
    } else {
        adj_degree_sums<<<sms * 8, 256, 0, s>>>(A.tl.slice_off.get(), A.tl.w_sell64.get(),
                                                A.tl.slices, A.tl.s_chunk, A.tl.n_long, n,
                                                A.tchunk.get(), o);
        if (A.tl.n_long)
            adj_degree_fix<<<ceil_div(A.tl.n_long, 256), 256, 0, s>>>(
                A.tl.chunk_begin.get(), A.tl.n_long, A.tchunk.get(), o);
    }
    NKG_CUDA(cudaGetLastError());
    // The relabelled CSR weights are not kept current: the sliced layouts
    // carry the weights from here on.
    g->w64src_stale = true;
    NKG_CUDA(cudaStreamSynchronize(s));
}

namespace {

// Grids and cost-balanced units of the two out-layout kernels (FP32 BiCGSTAB
// product, FP64 sweep) for the graph's launch shape.
template <bool WEIGHTED>
void adjoint_launch_setup(nkg_graph *g, AdjointState &A) {
    if (A.shape == g->sweep_shape)
        return;
    const unsigned sms = num_sms(g->device);
    cudaStream_t s = g->stream;
    int occ32 = 0, occ64 = 0, threads = 0;
    with_sweep_shape(g->sweep_shape, [&](auto S) {
        using Sh = decltype(S);
        auto k32 = bi_mv<WEIGHTED, 0, 1, Sh::threads, Sh::unroll, true>;
        auto k32b = bi_mv<WEIGHTED, 1, 1, Sh::threads, Sh::unroll, true>;
        auto k64 = adj_sweep<WEIGHTED, Sh::threads, Sh::unroll>;
        NKG_CUDA(cudaFuncSetAttribute(k32, cudaFuncAttributePreferredSharedMemoryCarveout, 0));
        NKG_CUDA(cudaFuncSetAttribute(k32b, cudaFuncAttributePreferredSharedMemoryCarveout, 0));
        NKG_CUDA(cudaFuncSetAttribute(k64, cudaFuncAttributePreferredSharedMemoryCarveout, 0));
        int o1 = 0, o2 = 0;
        NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o1, k32, Sh::threads, 0));
        NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o2, k32b, Sh::threads, 0));
        occ32 = std::min(o1, o2);
        NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ64, k64, Sh::threads, 0));
        threads = Sh::threads;
    });
    require(occ32 >= 1 && occ64 >= 1, "adjoint kernels do not fit on an SM");
    const uint64_t slices = A.tl.slices;
    auto ctas = [&](int occ) {
        return static_cast<unsigned>(std::max<uint64_t>(
            1, std::min<uint64_t>(static_cast<uint64_t>(occ) * sms,
                                  (slices * 32 + threads - 1) / threads)));
    };
    auto units = [&](unsigned c) {
        const uint64_t warps = static_cast<uint64_t>(c) * (threads / 32);
        return static_cast<uint32_t>(std::max<uint64_t>(
            1, std::min<uint64_t>(warps * kQueueUnitsPerWarp, std::max<uint64_t>(slices, 1))));
    };
    A.ctas32 = ctas(occ32);
    A.ctas64 = ctas(occ64);
    A.n_units32 = units(A.ctas32);
    A.n_units64 = units(A.ctas64);
    A.units32.alloc(static_cast<size_t>(A.n_units32) + 1);
    A.units64.alloc(static_cast<size_t>(A.n_units64) + 1);
    sell_units(A.tl, A.n_units32, A.units32.get(), s);
    sell_units(A.tl, A.n_units64, A.units64.get(), s);
    // dL/dw pass: a full grid of the arc-parallel kernel
    int occg = 0;
    NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occg, adj_grad_w, kGradThreads, 0));
    require(occg >= 1, "adjoint kernels do not fit on an SM");
    A.gw_ctas = static_cast<unsigned>(occg) * sms;
    NKG_CUDA(cudaStreamSynchronize(s));
    A.shape = g->sweep_shape;
    A.work.ready = false;  // partial-sum buffers depend on the grids
}

constexpr size_t kScalOffBi = 0, kScalOffAdj = 128, kScalOffSt = 256, kScalOffQueue = 320,
                 kScalBytes = 384;
static_assert(sizeof(AdjState) <= kScalOffQueue - kScalOffSt, "the queue counter follows the state");

void ensure_work(nkg_graph *g, AdjointState &A, unsigned vec_ctas, unsigned fix_ctas) {
    AdjWork &W = A.work;
    if (W.ready)
        return;
    const size_t n = g->n;
    const size_t part_n = std::max<size_t>(std::max(A.ctas32, A.ctas64), vec_ctas);
    const size_t chunks = static_cast<size_t>(A.tl.s_chunk) * 32 + 1;
    for (auto *a : {&W.p, &W.g, &W.t, &W.gbar, &W.c, &W.lam_f})
        a->alloc(n);
    W.lam[0].alloc(n + 1);
    W.lam[1].alloc(n + 1);
    W.part.alloc(std::max<size_t>(3 * part_n, 2 * static_cast<size_t>(
                                                   std::max(A.n_units32, A.n_units64))));
    W.fix_part.alloc(2 * static_cast<size_t>(fix_ctas));
    W.chunk64.alloc(chunks);
    W.chunk32.alloc(chunks);
    W.qc.alloc(n + 1);
    for (auto *a : {&W.t32, &W.x, &W.r, &W.rhat, &W.v, &W.tv})
        a->alloc(n);
    W.pv.alloc(n + 1);
    W.sv.alloc(n + 1);
    W.scal.alloc(kScalBytes);
    cudaStream_t s = g->stream;
    NKG_CUDA(cudaMemsetAsync(W.scal.get(), 0, kScalBytes, s));
    NKG_CUDA(cudaMemsetAsync(W.pv.get() + n, 0, sizeof(float), s));
    NKG_CUDA(cudaMemsetAsync(W.sv.get() + n, 0, sizeof(float), s));
    NKG_CUDA(cudaMemsetAsync(W.lam[1].get() + n, 0, sizeof(double), s));
    NKG_CUDA(cudaStreamSynchronize(s));
    W.ready = true;
}

struct AdjResult {
    uint64_t fp64_sweeps = 0, fp32_matvecs = 0, launches = 0;
    double residual = 0.0, ms = 0.0, ms_solve = 0.0;
};

template <bool WEIGHTED>
AdjResult run_adjoint(nkg_graph *g, const nkg_pr_params &p, const double *d_tele,
                      const double *d_scores, const double *d_grad, double *d_gw, double *d_gt) {
    AdjointState &A = adjoint_ensure(g);
    adjoint_launch_setup<WEIGHTED>(g, A);
    if (d_gw && !A.gw_src && g->arcs) {
        A.gw_src.alloc(g->arcs);
        A.gw_row.alloc(g->arcs);
        adj_caller_arcs<<<num_sms(g->device) * 16, 256, 0, g->stream>>>(
            g->row_ptr.get(), g->row_src.get(), g->col.get(), static_cast<uint32_t>(g->n),
            A.gw_src.get(), A.gw_row.get());
        NKG_CUDA(cudaGetLastError());
    }
    cudaStream_t s = g->stream;
    const uint32_t n = static_cast<uint32_t>(g->n);
    const unsigned sms = num_sms(g->device);
    const int personal = d_tele ? 1 : 0;
    const int distribute = p.distribute_sinks ? 1 : 0;
    const double inv_n = 1.0 / static_cast<double>(n);
    const unsigned vec_ctas = std::max<unsigned>(1, std::min<unsigned>(sms * 4, ceil_div(n, kBiThreads)));
    const unsigned fix_ctas = fix_ctas_with_units(
        split_fix_ctas<kBiThreads>(A.tl.n_long, A.tl.n_vlong), A.n_units32, kBiThreads);
    const unsigned adj_fix_ctas = fix_ctas_with_units(
        split_fix_ctas<kAdjThreads>(A.tl.n_long, A.tl.n_vlong), A.n_units64, kAdjThreads);
    ensure_work(g, A, vec_ctas, std::max(fix_ctas, adj_fix_ctas));
    AdjWork &W = A.work;
    AdjResult R;
    NKG_CUDA(cudaEventRecord(g->ev0, s));
    NKG_CUDA(cudaMemsetAsync(W.scal.get(), 0, kScalBytes, s));
    BiScalars *bsc = reinterpret_cast<BiScalars *>(W.scal.get() + kScalOffBi);
    AdjScalars *sc = reinterpret_cast<AdjScalars *>(W.scal.get() + kScalOffAdj);
    AdjState *st = reinterpret_cast<AdjState *>(W.scal.get() + kScalOffSt);
    static_assert(sizeof(BiScalars) <= 128 && sizeof(AdjScalars) <= 128 && sizeof(AdjState) <= 128,
                  "scalar blocks fit their slots");

    adj_inputs<<<vec_ctas, kAdjThreads, 0, s>>>(d_scores, d_grad, d_tele, A.tperm.get(),
                                                A.tdegc.get(), n, p.damp, distribute, W.p.get(),
                                                W.g.get(), W.t.get(), W.t32.get(), W.part.get(), sc);
    adj_rhs<<<vec_ctas, kAdjThreads, 0, s>>>(W.g.get(), W.t.get(), n, personal, inv_n,
                                             W.gbar.get(), W.r.get(), W.lam[0].get(), W.part.get(),
                                             sc, st);
    NKG_CUDA(cudaGetLastError());
    R.launches += 2;
    // Pinned read-back slots (16 doubles): BiScalars at 0 (80 bytes); the
    // adjoint's scalars and state at 12 (32 bytes).
    double *h2 = g->scalars_host.get() + 12;
    AdjState *hst = reinterpret_cast<AdjState *>(g->scalars_host.get() + 12);
    static_assert(sizeof(BiScalars) <= 12 * sizeof(double) && sizeof(AdjState) <= 4 * sizeof(double),
                  "read-back slots fit the pinned buffer");
    static_assert(offsetof(AdjScalars, sumx) == offsetof(AdjScalars, gnorm) + sizeof(double),
                  "gnorm and sumx are read back together");
    NKG_CUDA(cudaMemcpyAsync(h2, &sc->gnorm, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    const double gnorm = h2[0], sumx = h2[1];
    require(std::isfinite(gnorm) && std::isfinite(sumx) && sumx > 0.0,
            "scores / grad_scores are not finite or do not come from a converged forward run");
    const double tol_abs = p.tol * gnorm;

    AdjArgs aa{};
    aa.col_sell = A.tl.col_sell.get();
    aa.w_sell = A.tl.w_sell64.get();
    aa.slice_off = A.tl.slice_off.get();
    aa.unit_start = A.units64.get();
    aa.chunk_begin = A.tl.chunk_begin.get();
    aa.degc = A.tdegc.get();
    aa.degw = A.tdegw64.get();
    aa.tele = personal ? W.t.get() : nullptr;
    aa.gbar = W.gbar.get();
    aa.chunk_val = W.chunk64.get();
    aa.part = W.part.get();
    aa.fix_part = W.fix_part.get();
    aa.st = st;
    // The sweep's unit counter sits after the state in the zeroed scalars.
    aa.queue = reinterpret_cast<unsigned int *>(W.scal.get() + kScalOffQueue);
    aa.damp = p.damp;
    aa.inv_n = inv_n;
    aa.tol = tol_abs;
    aa.n = n;
    aa.n_long = A.tl.n_long;
    aa.n_vlong = A.tl.n_vlong;
    aa.s_chunk = A.tl.s_chunk;
    aa.units = A.n_units64;
    aa.sweep_ctas = A.ctas64;
    aa.distribute = distribute;
    aa.personal = personal;
    auto sweep64 = [&](const double *in, double *out, double *cout, unsigned long long max_it) {
        aa.lam_in = in;
        aa.lam_out = out;
        aa.c_out = cout;
        aa.max_iter = max_it;
        with_sweep_shape(g->sweep_shape, [&](auto S) {
            using Sh = decltype(S);
            adj_sweep<WEIGHTED, Sh::threads, Sh::unroll><<<A.ctas64, Sh::threads, 0, s>>>(aa);
        });
        adj_fix<WEIGHTED><<<adj_fix_ctas, kAdjThreads, 0, s>>>(aa);
        NKG_CUDA(cudaGetLastError());
        R.launches += 2;
        ++R.fp64_sweeps;
    };
    auto read_state = [&] {
        NKG_CUDA(cudaMemcpyAsync(hst, st, sizeof(AdjState), cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        check_cancel(g, "PageRank adjoint cancelled");
    };

    int fin = 0;  // W.lam[fin] holds the solution
    if (p.precision == NKG_PREC_FP64) {
        // Jacobi from lam0 = gbar until |lam' - lam|_1 <= tol |gbar|_1, in
        // batches of kSweepsPerGraph launches; the launches after the sweep
        // that meets the test return at once.
        uint64_t before = 0;
        for (;;) {
            const int fin0 = fin;
            for (int k = 0; k < kSweepsPerGraph; ++k)
                sweep64(W.lam[(fin0 + k) & 1].get(), W.lam[(fin0 + k + 1) & 1].get(), nullptr,
                        p.max_iterations);
            read_state();
            fin = fin0 ^ static_cast<int>((hst->iteration - before) & 1);
            before = hst->iteration;
            if (hst->done)
                break;
        }
        R.fp64_sweeps = before;
        R.residual = hst->residual;
    } else {
        BiArgs a{};
        a.col_sell = A.tl.col_sell.get();
        a.w_sell = A.w_sell32.get();
        a.slice_off = A.tl.slice_off.get();
        a.unit_start = A.units32.get();
        a.chunk_begin = A.tl.chunk_begin.get();
        a.degc = A.tdegc.get();
        a.degw = A.tdegw32.get();
        a.tele = personal ? W.t32.get() : nullptr;
        a.chunk_val = W.chunk32.get();
        a.x = W.x.get();
        a.r = W.r.get();
        a.rhat = W.rhat.get();
        a.p = W.pv.get();
        a.v = W.v.get();
        a.s = W.sv.get();
        a.t = W.tv.get();
        a.g = nullptr;
        a.part = W.part.get();
        a.fix_part = W.fix_part.get();
        a.sc = bsc;
        a.damp = p.damp;
        a.inv_n = inv_n;
        a.n = n;
        a.n_long = A.tl.n_long;
        a.n_vlong = A.tl.n_vlong;
        a.s_chunk = A.tl.s_chunk;
        a.units = A.n_units32;
        a.sweep_ctas = A.ctas32;
        // Queued products (the units of units32); their partials share W.part
        // with the vector kernels', which never run at the same time.
        a.unit_part = W.part.get();
        a.distribute = distribute;
        a.personal = personal;
        a.l2 = 0;
        BiLaunch bl;
        bl.stream = s;
        bl.sweep_shape = g->sweep_shape;
        bl.sweep_ctas = A.ctas32;
        bl.vec_ctas = vec_ctas;
        bl.fix_ctas = fix_ctas;
        bl.d_sc = bsc;
        bl.h_sc = reinterpret_cast<BiScalars *>(g->scalars_host.get());
        bl.cancel = &g->cancel;
        if (p.precision == NKG_PREC_FP32) {
            // FP32 alone: one solve to tol or the FP32 floor, whichever is larger.
            bi_solve<WEIGHTED, 1>(a, bl, std::max(p.tol, 3e-7), 0.0);
            adj_to_fp64<<<vec_ctas, kAdjThreads, 0, s>>>(W.x.get(), W.lam[0].get(), W.t.get(), n,
                                                         0, personal, inv_n, W.part.get(),
                                                         &sc->ticket, st);
            R.launches += 1;
            R.residual = bl.h_sc->res;
            // c = A^T lam for the solution.
            sweep64(W.lam[0].get(), nullptr, W.c.get(), ~0ull);
        } else {
            // FP32 solves, FP64 Jacobi residual sweeps: stop when the FP64
            // residual of lam is <= tol |gbar|_1 (lam is then the sweep's input,
            // and the sweep has written its c).
            bi_solve<WEIGHTED, 1>(a, bl, 1e-6, 0.25 * tol_abs);
            int add = 0;
            for (int round = 0;; ++round) {
                require(round < 40,
                        "FP32 refinement of the adjoint did not reach the tolerance in 40 rounds");
                adj_to_fp64<<<vec_ctas, kAdjThreads, 0, s>>>(W.x.get(), W.lam[0].get(), W.t.get(),
                                                             n, add, personal, inv_n, W.part.get(),
                                                             &sc->ticket, st);
                R.launches += 1;
                sweep64(W.lam[0].get(), W.lam[1].get(), W.c.get(), ~0ull);
                read_state();
                if (hst->residual <= tol_abs)
                    break;
                adj_residual_rhs<<<ceil_div(n, 256), 256, 0, s>>>(W.lam[1].get(), W.lam[0].get(),
                                                                  n, W.r.get());
                R.launches += 1;
                bi_solve<WEIGHTED, 1>(a, bl, 1e-5, 0.25 * tol_abs);
                add = 1;
            }
            R.residual = hst->residual;
        }
        R.fp32_matvecs = bl.matvecs;
        R.launches += bl.launches;
        fin = 0;
    }
    if (p.precision == NKG_PREC_FP64) {
        // c = A^T lam for the solution.
        NKG_CUDA(cudaMemsetAsync(st, 0, sizeof(AdjState), s));
        sweep64(W.lam[fin].get(), nullptr, W.c.get(), ~0ull);
    }
    NKG_CUDA(cudaEventRecord(g->ev1, s));
    const double *lam_t = W.lam[fin].get();
    if (d_gw && g->arcs) {
        adj_to_forward<WEIGHTED><<<ceil_div(static_cast<uint64_t>(n) + 1, 256), 256, 0, s>>>(
            A.tinv.get(), lam_t, W.c.get(), W.p.get(), A.tdegc.get(), A.tdegw64.get(), n, p.damp,
            W.lam_f.get(), W.qc.get());
        adj_grad_w<<<A.gw_ctas, kGradThreads, 0, s>>>(A.gw_src.get(), A.gw_row.get(),
                                                       W.lam_f.get(), W.qc.get(), g->arcs, d_gw);
        R.launches += 2;
    }
    if (d_gt) {
        adj_grad_t<<<ceil_div(g->z, 256), 256, 0, s>>>(g->inv.get(), A.tinv.get(), g->z, lam_t, sc,
                                                       d_gt);
        R.launches += 1;
    }
    NKG_CUDA(cudaGetLastError());
    NKG_CUDA(cudaEventRecord(g->ev2, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    NKG_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev2));
    R.ms = ms;
    NKG_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    R.ms_solve = ms;
    return R;
}

// Device copy of a caller array (host arrays are uploaded; device arrays are
// used in place).
const double *device_input(const double *p, size_t count, bool on_device, DeviceArray<double> &tmp,
                           cudaStream_t s) {
    if (!p || on_device)
        return p;
    tmp.alloc(std::max<size_t>(count, 1));
    if (count)
        NKG_CUDA(cudaMemcpyAsync(tmp.get(), p, count * sizeof(double), cudaMemcpyHostToDevice, s));
    return tmp.get();
}

} // namespace
} // namespace nkg

using namespace nkg;

extern "C" {

int nkg_graph_set_weights(nkg_graph *g, const double *in_w, const double *out_wdeg, int flags) {
    return guarded([&] {
        require(g != nullptr && in_w != nullptr, "NULL argument");
        require((flags & ~NKG_DEVICE_PTRS) == 0, "unknown flags");
        require(g->weighted, "the graph was created unweighted (in_w NULL)");
        require(!g->arc_sorted, "new weights need the in-rows in the caller's order (arc_order 0)");
        DeviceGuard guard(g->device);
        const bool dev = (flags & NKG_DEVICE_PTRS) != 0;
        DeviceArray<double> w_tmp, d_tmp;
        const double *d_w = device_input(in_w, g->arcs, dev, w_tmp, g->stream);
        const double *d_wdeg = device_input(out_wdeg, g->z, dev, d_tmp, g->stream);
        set_weights_device(g, d_w, d_wdeg);
    });
}

int nkg_pagerank_adjoint(nkg_graph *g, const nkg_pr_params *p, const double *teleport,
                         const double *scores, const double *grad_scores, double *grad_w_out,
                         double *grad_t_out, int flags, uint64_t *iterations_out,
                         nkg_stats *stats) {
    return guarded([&] {
        require(g != nullptr && p != nullptr, "NULL argument");
        require(scores != nullptr && grad_scores != nullptr, "scores / grad_scores is NULL");
        require((flags & ~NKG_DEVICE_PTRS) == 0, "unknown flags");
        require(p->norm == NKG_NORM_L1 || p->norm == NKG_NORM_L2, "norm must be L1 (0) or L2 (1)");
        require(p->precision >= NKG_PREC_FP64 && p->precision <= NKG_PREC_FP32,
                "unknown precision");
        require(!p->normalized, "the adjoint covers normalized = false (scores summing to 1)");
        require(std::isfinite(p->damp) && p->damp >= 0.0 && p->damp < 1.0,
                "damp must be in [0, 1)");
        require(p->tol >= 0.0, "tol must be >= 0");
        DeviceGuard guard(g->device);
        RunScope scope(g);
        const bool dev = (flags & NKG_DEVICE_PTRS) != 0;
        cudaStream_t s = g->stream;
        DeviceArray<double> t_tmp, s_tmp, g_tmp, gw_tmp, gt_tmp;
        const double *d_tele = device_input(teleport, g->z, dev, t_tmp, s);
        const double *d_scores = device_input(scores, g->z, dev, s_tmp, s);
        const double *d_grad = device_input(grad_scores, g->z, dev, g_tmp, s);
        double *d_gw = grad_w_out;
        double *d_gt = grad_t_out;
        if (!dev) {
            if (grad_w_out) {
                gw_tmp.alloc(std::max<uint64_t>(g->arcs, 1));
                d_gw = gw_tmp.get();
            }
            if (grad_t_out) {
                gt_tmp.alloc(g->z);
                d_gt = gt_tmp.get();
            }
        }
        const AdjResult R = g->weighted
                                ? run_adjoint<true>(g, *p, d_tele, d_scores, d_grad, d_gw, d_gt)
                                : run_adjoint<false>(g, *p, d_tele, d_scores, d_grad, d_gw, d_gt);
        if (!dev) {
            if (grad_w_out && g->arcs)
                NKG_CUDA(cudaMemcpyAsync(grad_w_out, d_gw, g->arcs * sizeof(double),
                                         cudaMemcpyDeviceToHost, s));
            if (grad_t_out)
                NKG_CUDA(cudaMemcpyAsync(grad_t_out, d_gt, g->z * sizeof(double),
                                         cudaMemcpyDeviceToHost, s));
            NKG_CUDA(cudaStreamSynchronize(s));
        }
        if (iterations_out)
            *iterations_out = R.fp64_sweeps + R.fp32_matvecs;
        if (stats) {
            clear_stats(stats);
            stats->iterations = R.fp64_sweeps + R.fp32_matvecs;
            stats->residual = R.residual;
            stats->ms_total = R.ms;
            stats->ms_iterations = R.ms_solve;
            stats->kernel_launches = R.launches;
            stats->fp64_sweeps = R.fp64_sweeps;
            stats->fp32_sweeps = R.fp32_matvecs;
        }
    });
}

} // extern "C"
