// Differentiable PageRank: the adjoint (backward) solve and the gradients
// with respect to the arc weights and the teleport vector. No reference
// counterpart; the forward it differentiates is PageRank.cpp:20-104 with a
// weighted graph (optionally distributeSinks and a personalised teleport).
//
// Forward fixed point, in the relabelled order, with t the teleport
// distribution (1/n without one), m the sink mask and A[u,v] = w(v->u)/wdeg[v]:
//     x = d (A x + [distributeSinks] (m.x) t) + (1-d) t,    p = x / sum(x).
// For a loss L with g = dL/dp, with gbar = g - (g.p) 1, the adjoint lam solves
//     (I - d M^T) lam = gbar,   M^T q = A^T q + [distributeSinks] m (t.q),
// and, with c = A^T lam (c[v] = sum_{v->u} w lam[u] / wdeg[v]),
//     dL/dw(v->u) = d (p[v] / wdeg[v]) (lam[u] - c[v])
//     dL/dt[u]    = (d [distributeSinks] m.p + (1-d) / sum(x)) lam[u]
// where sum(x) follows from p alone at the fixed point (summing the forward
// equation over all nodes, tau = sum(t)):
//     sum(x) = (1-d) tau / (1 - d + d (m.p) (1 - [distributeSinks] tau)).
// (The lam here is sum(x) times the lam of the un-normalised system, which is
// why neither gradient needs sum(x) beyond that one factor.)
//
// A^T is a pull over the out-adjacency, so the graph gets a second sliced
// layout: the out-CSR of the relabelled graph, its rows (nodes) sorted by
// out-degree, descending, each row listing its out-arcs in the order they
// appear in the in-CSR. The FP32 solve is the BiCGSTAB of refine.cuh with
// OP = 1; the FP64 Jacobi sweep of the adjoint system below gives the
// residual of the refinement, the FP64 solve and the final c.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "graph.hpp"
#include "host.hpp"
#include "refine.cuh"

namespace nkg {

struct AdjointState {
    SellLayout tl;                  // out-adjacency, rows in out-degree order
    DeviceArray<uint32_t> trow;     // n: node of out-row rt
    DeviceArray<uint32_t> tptr;     // n+1: out-CSR offsets (out-row order)
    DeviceArray<uint32_t> tarc;     // arcs: in-CSR index of every out-CSR entry
    DeviceArray<float> w_sell32;    // slots (weighted graphs)
    DeviceArray<float> degw32;      // n (weighted graphs)
    DeviceArray<uint32_t> units32, units64;
    uint32_t n_units32 = 0, n_units64 = 0;
    unsigned ctas32 = 0, ctas64 = 0;
    int shape = -1;
};

void destroy_adjoint(AdjointState *a) { delete a; }

namespace {

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

__global__ void adj_row_lengths(const uint32_t *__restrict__ trow, const uint32_t *__restrict__ degc,
                                uint32_t n, uint32_t *__restrict__ tlen,
                                uint32_t *__restrict__ tinv) {
    const uint32_t rt = blockIdx.x * blockDim.x + threadIdx.x;
    if (rt < n) {
        const uint32_t v = trow[rt];
        tlen[rt] = degc[v];
        tinv[v] = rt;
    }
}

// Per in-arc e (row u, source v): sort key = out-row of v, value = e; and the
// row of every arc. One warp per in-row.
__global__ void adj_arc_keys(const uint32_t *__restrict__ row_ptr, const uint32_t *__restrict__ col,
                             const uint32_t *__restrict__ tinv, uint32_t n,
                             uint32_t *__restrict__ key, uint32_t *__restrict__ val,
                             uint32_t *__restrict__ arc_row) {
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint64_t u = warp; u < n; u += nwarps) {
        const uint32_t b = row_ptr[u], e = row_ptr[u + 1];
        for (uint32_t k = b + lane; k < e; k += 32) {
            key[k] = tinv[col[k]];
            val[k] = k;
            arc_row[k] = static_cast<uint32_t>(u);
        }
    }
}

__global__ void adj_gather_cols(const uint32_t *__restrict__ tarc,
                                const uint32_t *__restrict__ arc_row, uint64_t arcs,
                                uint32_t *__restrict__ tcol) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < arcs;
         k += stride)
        tcol[k] = arc_row[tarc[k]];
}

// Weighted out-degree: one warp per out-row, lane-strided partial sums
// combined by a fixed shuffle tree (deterministic).
__global__ void adj_out_wdeg(const uint32_t *__restrict__ tptr, const uint32_t *__restrict__ tarc,
                             const uint32_t *__restrict__ trow, const double *__restrict__ w,
                             uint32_t n, double *__restrict__ degw) {
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint64_t rt = warp; rt < n; rt += nwarps) {
        double s = 0.0;
        for (uint32_t k = tptr[rt] + lane; k < tptr[rt + 1]; k += 32)
            s += w[tarc[k]];
        s = warp_sum(s);
        if (lane == 0)
            degw[trow[rt]] = s;
    }
}

// ---------------------------------------------------------------------------
// FP64 Jacobi sweep of the adjoint system

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
    const uint32_t *__restrict__ row_label;
    const uint32_t *__restrict__ degc;
    const double *__restrict__ degw;
    const double *__restrict__ tele;      // relabelled teleport or null
    const double *__restrict__ gbar;
    const double *__restrict__ lam_in;    // n+1, lam_in[n] = 0
    double *__restrict__ lam_out;         // n+1 or null (c only)
    double *__restrict__ c_out;           // n or null
    double *__restrict__ chunk_val;
    double *__restrict__ part;            // 2 per sweep CTA
    double *__restrict__ fix_part;        // 2 per fix-up CTA
    AdjState *st;
    double damp, inv_n, tol;
    unsigned long long max_iter;
    uint32_t n, n_long, s_chunk, units, sweep_ctas;
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
__global__ void __launch_bounds__(THREADS) adj_sweep(AdjArgs a) {
    __shared__ double s_red[32];
    if (*(volatile int *)&a.st->done)
        return;
    const double tdot = a.st->tdot;
    const int lane = threadIdx.x & 31;
    const uint32_t wpc = THREADS / 32;
    const uint32_t gw = blockIdx.x * wpc + (threadIdx.x >> 5);
    const uint32_t nw = gridDim.x * wpc;
    double res = 0.0, td = 0.0;
    for (uint32_t u = gw; u < a.units; u += nw) {
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
                    v[k] = __ldg(a.lam_in + c[k]);
                if (WEIGHTED) {
#pragma unroll
                    for (int k = 0; k < UNROLL; ++k)
                        v[k] *= ld_stream(a.w_sell + base + static_cast<size_t>(j + k) * 32);
                }
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    acc += v[k];
            }
            for (; j < len; ++j) {
                double v = __ldg(a.lam_in + ld_stream(cp + static_cast<size_t>(j) * 32));
                if (WEIGHTED)
                    v *= ld_stream(a.w_sell + base + static_cast<size_t>(j) * 32);
                acc += v;
            }
            if (s < a.s_chunk) {
                a.chunk_val[static_cast<size_t>(s) * 32 + lane] = acc;
            } else {
                const uint32_t r = a.n_long + (s - a.s_chunk) * 32 + lane;
                if (r < a.n)
                    adj_row<WEIGHTED>(a, a.row_label[r], acc, tdot, res, td);
            }
        }
    }
    res = block_sum<THREADS>(res, s_red);
    td = block_sum<THREADS>(td, s_red);
    if (threadIdx.x == 0) {
        a.part[2 * blockIdx.x] = res;
        a.part[2 * blockIdx.x + 1] = td;
    }
}

constexpr int kAdjThreads = 256;

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
    const uint32_t r = blockIdx.x * kAdjThreads + threadIdx.x;
    if (r < a.n_long) {
        double acc = 0.0;
        for (uint32_t k = a.chunk_begin[r]; k < a.chunk_begin[r + 1]; ++k)
            acc += a.chunk_val[k];
        adj_row<WEIGHTED>(a, a.row_label[r], acc, tdot, res, td);
    }
    res = block_sum<kAdjThreads>(res, s_red);
    td = block_sum<kAdjThreads>(td, s_red);
    if (threadIdx.x == 0) {
        a.fix_part[2 * blockIdx.x] = res;
        a.fix_part[2 * blockIdx.x + 1] = td;
    }
    if (!bi_last_block(&a.st->ticket, &s_last))
        return;
    double t1 = 0.0, t2 = 0.0;
    for (uint32_t i = threadIdx.x; i < a.sweep_ctas; i += kAdjThreads) {
        t1 += ((volatile double *)a.part)[2 * i];
        t2 += ((volatile double *)a.part)[2 * i + 1];
    }
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

// p and g into the relabelled order; g.p, m.p and sum(t).
__global__ void __launch_bounds__(kAdjThreads)
    adj_inputs(const double *__restrict__ scores, const double *__restrict__ grad,
               const double *__restrict__ tele_orig, const uint32_t *__restrict__ perm,
               const uint32_t *__restrict__ degc, uint32_t n, double damp, int distribute,
               double *__restrict__ p_lab, double *__restrict__ g_lab, double *__restrict__ t_lab,
               float *__restrict__ t32, double *__restrict__ part, AdjScalars *sc) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    double gp = 0.0, sp = 0.0, tau = 0.0;
    for (uint32_t r = blockIdx.x * kAdjThreads + threadIdx.x; r < n; r += gridDim.x * kAdjThreads) {
        const uint32_t o = perm[r];
        const double pv = scores[o], gv = grad[o];
        p_lab[r] = pv;
        g_lab[r] = gv;
        gp += gv * pv;
        if (degc[r] == 0)
            sp += pv;
        if (tele_orig) {
            const double t = tele_orig[o];
            t_lab[r] = t;
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

// gbar = g - (g.p) 1 (FP64 and FP32 copies), lam0 = gbar, |gbar|_1 and
// tel.gbar (the state of a Jacobi sweep from lam0).
__global__ void __launch_bounds__(kAdjThreads)
    adj_rhs(const double *__restrict__ g_lab, const double *__restrict__ t_lab, uint32_t n,
            int personal, double inv_n, double *__restrict__ gbar, float *__restrict__ r32,
            double *__restrict__ lam0, double *__restrict__ part, AdjScalars *sc, AdjState *st) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    const double gp = sc->gp;
    double nrm = 0.0, td = 0.0;
    for (uint32_t r = blockIdx.x * kAdjThreads + threadIdx.x; r < n; r += gridDim.x * kAdjThreads) {
        const double b = g_lab[r] - gp;
        gbar[r] = b;
        r32[r] = static_cast<float>(b);
        lam0[r] = b;
        nrm += fabs(b);
        td += personal ? t_lab[r] * b : b;
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
        sc->ticket = 0;
    }
}

// lam64 = x32 (add = 0) or lam64 += x32 (add = 1), lam64[n] = 0, and the
// sweep state for lam64 (tel.lam64; not done).
__global__ void __launch_bounds__(kAdjThreads)
    adj_to_fp64(const float *__restrict__ x32, double *__restrict__ lam, const double *t_lab,
                uint32_t n, int add, int personal, double inv_n, double *__restrict__ part,
                unsigned int *ticket, AdjState *st) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    double td = 0.0;
    for (uint32_t r = blockIdx.x * kAdjThreads + threadIdx.x; r < n; r += gridDim.x * kAdjThreads) {
        const double v = add ? lam[r] + static_cast<double>(x32[r]) : static_cast<double>(x32[r]);
        lam[r] = v;
        td += personal ? t_lab[r] * v : v;
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

// dL/dw for every in-arc, written at the arc's index in the caller's in-CSR.
// One warp per in-row u.
template <bool WEIGHTED>
__global__ void adj_grad_w(const uint32_t *__restrict__ row_ptr, const uint32_t *__restrict__ col,
                           const uint64_t *__restrict__ row_src, const double *__restrict__ p_lab,
                           const uint32_t *__restrict__ degc, const double *__restrict__ degw,
                           const double *__restrict__ lam, const double *__restrict__ c,
                           uint32_t n, double damp, double *__restrict__ grad_w) {
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint64_t u = warp; u < n; u += nwarps) {
        const uint32_t b = row_ptr[u], e = row_ptr[u + 1];
        const uint64_t dst = row_src[u];
        const double lu = lam[u];
        for (uint32_t k = b + lane; k < e; k += 32) {
            const uint32_t v = col[k];
            const double deg = WEIGHTED ? degw[v] : static_cast<double>(degc[v]);
            grad_w[dst + (k - b)] = damp * (p_lab[v] / deg) * (lu - c[v]);
        }
    }
}

// dL/dt in the caller's ids (0 for ids of deleted nodes).
__global__ void adj_grad_t(const uint32_t *__restrict__ inv, uint64_t z,
                           const double *__restrict__ lam, const AdjScalars *sc,
                           double *__restrict__ grad_t) {
    const uint64_t o = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (o >= z)
        return;
    const uint32_t r = inv[o];
    grad_t[o] = r == kNone ? 0.0 : sc->tfac * lam[r];
}

} // namespace

// ---------------------------------------------------------------------------
// Host side

AdjointState &adjoint_ensure(nkg_graph *g) {
    if (g->adj)
        return *g->adj;
    require(!g->arc_sorted,
            "the adjoint needs the in-rows in the caller's arc order (arc_order 0)");
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
    DeviceArray<uint32_t> tlen(n), tinv(n);
    adj_row_lengths<<<ceil_div(n, 256), 256, 0, s>>>(A->trow.get(), g->degc.get(), n, tlen.get(),
                                                     tinv.get());
    NKG_CUDA(cudaGetLastError());
    A->tptr.alloc(static_cast<size_t>(n) + 1);
    NKG_CUDA(cudaMemsetAsync(A->tptr.get(), 0, sizeof(uint32_t), s));
    {
        size_t tb = 0;
        NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, tlen.get(), A->tptr.get() + 1,
                                               static_cast<int64_t>(n), s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb, tlen.get(), A->tptr.get() + 1,
                                               static_cast<int64_t>(n), s));
    }

    // Group the in-arcs by out-row (stable: in-CSR order inside a row).
    A->tarc.alloc(std::max<uint64_t>(arcs, 1));
    DeviceArray<uint32_t> tcol(std::max<uint64_t>(arcs, 1));
    if (arcs) {
        DeviceArray<uint32_t> key(arcs), key_s(arcs), val(arcs), arc_row(arcs);
        adj_arc_keys<<<sms * 16, 256, 0, s>>>(g->row_ptr.get(), g->col.get(), tinv.get(), n,
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
        adj_gather_cols<<<sms * 8, 256, 0, s>>>(A->tarc.get(), arc_row.get(), arcs, tcol.get());
        NKG_CUDA(cudaGetLastError());
        NKG_CUDA(cudaStreamSynchronize(s));
    }
    build_sell(A->tl, n, A->tptr.get(), tcol.get(), g->weighted ? g->w64src.get() : nullptr,
               A->tarc.get(), tlen.get(), g->device, s);
    if (g->weighted) {
        A->w_sell32.alloc(A->tl.slots, 4);
        A->degw32.alloc(n);
        convert_to_float(A->tl.w_sell64.get(), A->w_sell32.get(), A->tl.slots, g->device, s);
        convert_to_float(g->degw64src.get(), A->degw32.get(), n, g->device, s);
    }
    NKG_CUDA(cudaStreamSynchronize(s));
    g->adj.reset(A.release());
    return *g->adj;
}

void adjoint_refresh_weights(nkg_graph *g) {
    if (!g->adj || !g->weighted)
        return;
    AdjointState &A = *g->adj;
    const uint32_t n = static_cast<uint32_t>(g->n);
    refill_sell_weights(A.tl, n, A.tptr.get(), g->w64src.get(), A.tarc.get(), g->device, g->stream);
    convert_to_float(A.tl.w_sell64.get(), A.w_sell32.get(), A.tl.slots, g->device, g->stream);
    convert_to_float(g->degw64src.get(), A.degw32.get(), n, g->device, g->stream);
    NKG_CUDA(cudaStreamSynchronize(g->stream));
}

void adjoint_out_wdeg(nkg_graph *g, double *degw) {
    AdjointState &A = adjoint_ensure(g);
    const uint32_t n = static_cast<uint32_t>(g->n);
    adj_out_wdeg<<<num_sms(g->device) * 16, 256, 0, g->stream>>>(A.tptr.get(), A.tarc.get(),
                                                                A.trow.get(), g->w64src.get(), n,
                                                                degw);
    NKG_CUDA(cudaGetLastError());
}

namespace {

// Grids and cost-balanced units of the two out-adjacency kernels (FP32
// BiCGSTAB product, FP64 sweep) for the graph's launch shape.
template <bool WEIGHTED>
void adjoint_launch_setup(nkg_graph *g, AdjointState &A) {
    if (A.shape == g->sweep_shape)
        return;
    const unsigned sms = num_sms(g->device);
    cudaStream_t s = g->stream;
    int occ32 = 0, occ64 = 0, threads = 0;
    with_sweep_shape(g->sweep_shape, [&](auto S) {
        using Sh = decltype(S);
        auto k32 = bi_mv<WEIGHTED, 0, 1, Sh::threads, Sh::unroll>;
        auto k32b = bi_mv<WEIGHTED, 1, 1, Sh::threads, Sh::unroll>;
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
        return static_cast<uint32_t>(
            std::max<uint64_t>(1, std::min<uint64_t>(warps * kUnitsPerWarp, std::max<uint64_t>(slices, 1))));
    };
    A.ctas32 = ctas(occ32);
    A.ctas64 = ctas(occ64);
    A.n_units32 = units(A.ctas32);
    A.n_units64 = units(A.ctas64);
    A.units32.alloc(static_cast<size_t>(A.n_units32) + 1);
    A.units64.alloc(static_cast<size_t>(A.n_units64) + 1);
    sell_units(A.tl, A.n_units32, A.units32.get(), s);
    sell_units(A.tl, A.n_units64, A.units64.get(), s);
    NKG_CUDA(cudaStreamSynchronize(s));
    A.shape = g->sweep_shape;
}

struct AdjResult {
    uint64_t fp64_sweeps = 0, fp32_matvecs = 0, launches = 0;
    double residual = 0.0, ms = 0.0;
};

template <bool WEIGHTED>
AdjResult run_adjoint(nkg_graph *g, const nkg_pr_params &p, const double *d_tele,
                      const double *d_scores, const double *d_grad, double *d_gw, double *d_gt) {
    AdjointState &A = adjoint_ensure(g);
    adjoint_launch_setup<WEIGHTED>(g, A);
    cudaStream_t s = g->stream;
    const uint32_t n = static_cast<uint32_t>(g->n);
    const unsigned sms = num_sms(g->device);
    const int personal = d_tele ? 1 : 0;
    const int distribute = p.distribute_sinks ? 1 : 0;
    const double inv_n = 1.0 / static_cast<double>(n);
    AdjResult R;
    NKG_CUDA(cudaEventRecord(g->ev0, s));

    const unsigned vec_ctas = std::max<unsigned>(1, std::min<unsigned>(sms * 4, ceil_div(n, kBiThreads)));
    const unsigned fix_ctas = std::max<unsigned>(1, ceil_div(A.tl.n_long, kBiThreads));
    const unsigned part_n = std::max<unsigned>(std::max(A.ctas32, A.ctas64), vec_ctas);
    DeviceArray<double> p_lab(n), g_lab(n), t_lab(personal ? n : 0), gbar(n), c(n), part(3ull * part_n),
        fix_part(2ull * fix_ctas), chunk64(static_cast<size_t>(A.tl.s_chunk) * 32 + 1);
    DeviceArray<double> lam[2] = {DeviceArray<double>(n + 1), DeviceArray<double>(n + 1)};
    DeviceArray<float> t32(personal ? n : 0), chunk32(static_cast<size_t>(A.tl.s_chunk) * 32 + 1);
    DeviceArray<float> bx(n), br(n), brhat(n), bp(n + 1), bv(n), bs(n + 1), bt(n);
    DeviceArray<AdjScalars> sc(1);
    DeviceArray<BiScalars> bsc(1);
    DeviceArray<AdjState> st(1);
    NKG_CUDA(cudaMemsetAsync(sc.get(), 0, sizeof(AdjScalars), s));
    NKG_CUDA(cudaMemsetAsync(bsc.get(), 0, sizeof(BiScalars), s));
    NKG_CUDA(cudaMemsetAsync(st.get(), 0, sizeof(AdjState), s));
    NKG_CUDA(cudaMemsetAsync(bp.get() + n, 0, sizeof(float), s));
    NKG_CUDA(cudaMemsetAsync(bs.get() + n, 0, sizeof(float), s));
    NKG_CUDA(cudaMemsetAsync(lam[1].get() + n, 0, sizeof(double), s));

    const double *degw64 = g->degw64src.get();
    adj_inputs<<<vec_ctas, kAdjThreads, 0, s>>>(d_scores, d_grad, d_tele, g->perm.get(),
                                                g->degc.get(), n, p.damp, distribute, p_lab.get(),
                                                g_lab.get(), t_lab.get(), t32.get(), part.get(),
                                                sc.get());
    adj_rhs<<<vec_ctas, kAdjThreads, 0, s>>>(g_lab.get(), t_lab.get(), n, personal, inv_n,
                                             gbar.get(), br.get(), lam[0].get(), part.get(),
                                             sc.get(), st.get());
    NKG_CUDA(cudaGetLastError());
    R.launches += 2;
    AdjScalars *hsc = reinterpret_cast<AdjScalars *>(g->scalars_host.get());
    static_assert(sizeof(AdjScalars) <= 16 * sizeof(double), "AdjScalars fits the pinned buffer");
    NKG_CUDA(cudaMemcpyAsync(hsc, sc.get(), sizeof(AdjScalars), cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    const double gnorm = hsc->gnorm;
    require(std::isfinite(gnorm) && std::isfinite(hsc->sumx) && hsc->sumx > 0.0,
            "scores / grad_scores are not finite or do not come from a converged forward run");
    const double tol_abs = p.tol * gnorm;

    // FP64 sweep arguments (lam_in / lam_out / c_out set per launch).
    AdjArgs aa{};
    aa.col_sell = A.tl.col_sell.get();
    aa.w_sell = A.tl.w_sell64.get();
    aa.slice_off = A.tl.slice_off.get();
    aa.unit_start = A.units64.get();
    aa.chunk_begin = A.tl.chunk_begin.get();
    aa.row_label = A.trow.get();
    aa.degc = g->degc.get();
    aa.degw = degw64;
    aa.tele = t_lab.get();
    aa.gbar = gbar.get();
    aa.chunk_val = chunk64.get();
    aa.part = part.get();
    aa.fix_part = fix_part.get();
    aa.st = st.get();
    aa.damp = p.damp;
    aa.inv_n = inv_n;
    aa.tol = tol_abs;
    aa.n = n;
    aa.n_long = A.tl.n_long;
    aa.s_chunk = A.tl.s_chunk;
    aa.units = A.n_units64;
    aa.sweep_ctas = A.ctas64;
    aa.distribute = distribute;
    aa.personal = personal;
    const unsigned adj_fix_ctas = std::max<unsigned>(1, ceil_div(A.tl.n_long, kAdjThreads));
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
    // Pinned read-back slots: BiScalars at 0 (80 bytes), AdjState at 96.
    AdjState *hst = reinterpret_cast<AdjState *>(g->scalars_host.get() + 12);
    static_assert(sizeof(BiScalars) <= 12 * sizeof(double) && sizeof(AdjState) <= 4 * sizeof(double),
                  "read-back slots fit the pinned buffer");
    auto read_state = [&] {
        NKG_CUDA(cudaMemcpyAsync(hst, st.get(), sizeof(AdjState), cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        if (g->cancel.load()) {
            g->cancel.store(0);
            throw Error(NKG_ERR_CANCELLED, "PageRank adjoint cancelled");
        }
    };

    int fin = 0;  // lam[fin] is the solution
    if (p.precision == NKG_PREC_FP64) {
        // Jacobi from lam0 = gbar until |lam' - lam|_1 <= tol |gbar|_1, in
        // batches of kSweepsPerGraph launches; the launches after the sweep
        // that meets the test return at once.
        uint64_t before = 0;
        R.fp64_sweeps = 0;
        for (;;) {
            const int fin0 = fin;
            for (int k = 0; k < kSweepsPerGraph; ++k)
                sweep64(lam[(fin0 + k) & 1].get(), lam[(fin0 + k + 1) & 1].get(), nullptr,
                        p.max_iterations);
            read_state();
            const uint64_t eff = hst->iteration - before;
            fin = fin0 ^ static_cast<int>(eff & 1);
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
        a.degc = g->degc.get();
        a.degw = A.degw32.get();
        a.tele = t32.get();
        a.row_label = A.trow.get();
        a.chunk_val = chunk32.get();
        a.x = bx.get();
        a.r = br.get();
        a.rhat = brhat.get();
        a.p = bp.get();
        a.v = bv.get();
        a.s = bs.get();
        a.t = bt.get();
        a.g = nullptr;
        a.part = part.get();
        a.fix_part = fix_part.get();
        a.sc = bsc.get();
        a.damp = p.damp;
        a.inv_n = inv_n;
        a.n = n;
        a.n_long = A.tl.n_long;
        a.n_vlong = A.tl.n_vlong;
        a.s_chunk = A.tl.s_chunk;
        a.units = A.n_units32;
        a.sweep_ctas = A.ctas32;
        a.distribute = distribute;
        a.personal = personal;
        a.l2 = 0;
        BiLaunch bl;
        bl.stream = s;
        bl.sweep_shape = g->sweep_shape;
        bl.sweep_ctas = A.ctas32;
        bl.vec_ctas = vec_ctas;
        bl.fix_ctas = fix_ctas;
        bl.d_sc = bsc.get();
        bl.h_sc = reinterpret_cast<BiScalars *>(g->scalars_host.get());
        bl.cancel = &g->cancel;
        if (p.precision == NKG_PREC_FP32) {
            // FP32 alone: one solve to the FP32 floor or tol, whichever is larger.
            bi_solve<WEIGHTED, 1>(a, bl, std::max(p.tol, 3e-7), 0.0);
            adj_to_fp64<<<vec_ctas, kAdjThreads, 0, s>>>(bx.get(), lam[0].get(), t_lab.get(), n,
                                                         0, personal, inv_n, part.get(),
                                                         &sc.get()->ticket, st.get());
            R.launches += 1;
            NKG_CUDA(cudaMemcpyAsync(bl.h_sc, bsc.get(), sizeof(BiScalars), cudaMemcpyDeviceToHost, s));
            NKG_CUDA(cudaStreamSynchronize(s));
            R.residual = bl.h_sc->res;
        } else {
            // FP32 solves, FP64 Jacobi residual sweeps: stop when the FP64
            // residual of lam is <= tol |gbar|_1 (lam is then the sweep's input).
            bi_solve<WEIGHTED, 1>(a, bl, 1e-6, 0.25 * tol_abs);
            int add = 0;
            for (int round = 0;; ++round) {
                require(round < 40, "FP32 refinement of the adjoint did not reach the tolerance in 40 rounds");
                adj_to_fp64<<<vec_ctas, kAdjThreads, 0, s>>>(bx.get(), lam[0].get(), t_lab.get(),
                                                             n, add, personal, inv_n, part.get(),
                                                             &sc.get()->ticket, st.get());
                R.launches += 1;
                sweep64(lam[0].get(), lam[1].get(), c.get(), ~0ull);
                read_state();
                if (hst->residual <= tol_abs)
                    break;
                adj_residual_rhs<<<ceil_div(n, 256), 256, 0, s>>>(lam[1].get(), lam[0].get(), n,
                                                                  br.get());
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
    // c = A^T lam for the solution (the refinement's last sweep already has it).
    if (!(p.precision == NKG_PREC_FP32_REFINE)) {
        NKG_CUDA(cudaMemsetAsync(st.get(), 0, sizeof(AdjState), s));
        sweep64(lam[fin].get(), nullptr, c.get(), ~0ull);
    }
    NKG_CUDA(cudaEventRecord(g->ev1, s));
    if (d_gw && g->arcs) {
        if (WEIGHTED)
            adj_grad_w<true><<<sms * 16, 256, 0, s>>>(g->row_ptr.get(), g->col.get(),
                                                      g->row_src.get(), p_lab.get(), g->degc.get(),
                                                      degw64, lam[fin].get(), c.get(), n, p.damp,
                                                      d_gw);
        else
            adj_grad_w<false><<<sms * 16, 256, 0, s>>>(g->row_ptr.get(), g->col.get(),
                                                       g->row_src.get(), p_lab.get(), g->degc.get(),
                                                       nullptr, lam[fin].get(), c.get(), n, p.damp,
                                                       d_gw);
        R.launches += 1;
    }
    if (d_gt) {
        adj_grad_t<<<ceil_div(g->z, 256), 256, 0, s>>>(g->inv.get(), g->z, lam[fin].get(), sc.get(),
                                                       d_gt);
        R.launches += 1;
    }
    NKG_CUDA(cudaGetLastError());
    NKG_CUDA(cudaEventRecord(g->ev2, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    NKG_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev2));
    R.ms = ms;
    return R;
}

// Device copy of a caller array (host arrays are uploaded; device arrays
// are used in place).
const double *device_input(const double *p, size_t count, bool on_device, DeviceArray<double> &tmp,
                           cudaStream_t s) {
    if (!p || on_device)
        return p;
    tmp.alloc(count);
    if (count)
        NKG_CUDA(cudaMemcpyAsync(tmp.get(), p, count * sizeof(double), cudaMemcpyHostToDevice, s));
    return tmp.get();
}

} // namespace
} // namespace nkg

using namespace nkg;

extern "C" {

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
        g->cancel.store(0);
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
            std::memset(stats, 0, sizeof(*stats));
            stats->iterations = R.fp64_sweeps + R.fp32_matvecs;
            stats->residual = R.residual;
            stats->ms_total = R.ms;
            float ms = 0.f;
            NKG_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
            stats->ms_iterations = ms;
            stats->kernel_launches = R.launches;
            stats->fp64_sweeps = R.fp64_sweeps;
            stats->fp32_sweeps = R.fp32_matvecs;
        }
    });
}

} // extern "C"
