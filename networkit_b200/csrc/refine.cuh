// FP32 bulk solve with FP64 refinement (the FP32_REFINE precision). The
// PageRank fixed point is the linear system (I - d M) x = b with
// M = A + [distributeSinks] t m^T, A[u,v] = w(v->u)/wdeg[v], m the sink mask
// and b = (1-d) t. The bulk work is an FP32 BiCGSTAB solve of that system
// (van der Vorst, SIAM J. Sci. Stat. Comput. 13(2), 1992; applied to
// PageRank by Gleich, Zhukov and Berkhin, 2005) whose matrix-vector product is
// the sliced-ELLPACK SpMV of sweep.cuh in FP32 with FP32 accumulation. Dot
// products, norms and sink masses are FP64 with fixed-order reductions; the
// scalars stay on the device. The FP64 part is the reference's own Jacobi
// step (the FP64 sweep), which gives the residual x' - x; while its norm is
// above tol the residual is solved for a correction in FP32 again.
//
// The same kernels solve the adjoint system (I - d M^T) lam = gbar of the
// differentiable form (OP = 1): the product then runs over the sliced
// out-adjacency, M^T q = A^T q + [distributeSinks] m (t.q) with
// (A^T q)[v] = sum_{v->u} w q[u] / wdeg[v]: the vector is gathered as it is
// (no degree scaling) and every row is scaled after its sum. All vectors of an
// OP 1 solve are indexed in the out-adjacency's row order (degc, degw and tele
// too), so rows are written in place.
#pragma once

#include <atomic>

#include "sweep.cuh"

namespace nkg {

// Device-side scalars of one BiCGSTAB solve (FP64).
struct BiScalars {
    double rho, rho_prev, alpha, omega;
    double vdot;      // (rhat, v)
    double ts, tt;    // (t, s), (t, t)
    double res;       // norm of the current residual r
    double sink_vec;  // m.q (OP 0) or tel.q (OP 1), q the next product's input
    int breakdown;
    unsigned int ticket;
    unsigned int queue;  // next work unit of a queued product (reset by bi_mv_fix)
};

struct BiArgs {
    // SELL structure of the graph (FP32 plane).
    const uint32_t *__restrict__ col_sell;
    const float *__restrict__ w_sell;
    const uint32_t *__restrict__ slice_off;
    const uint32_t *__restrict__ unit_start;
    const uint32_t *__restrict__ chunk_begin;
    const uint32_t *__restrict__ degc;
    const float *__restrict__ degw;
    const float *__restrict__ tele;   // personalised teleport (n) or null
    float *__restrict__ chunk_val;
    // vectors (x-form, n entries; g is the gather form, n+1 with g[n] = 0;
    // for OP 1, p and s have n+1 entries with p[n] = s[n] = 0 and g is unused)
    float *x, *r, *rhat, *p, *v, *s, *t, *g;
    double *__restrict__ part;        // per-CTA partial sums (3 per CTA)
    double *__restrict__ fix_part;
    BiScalars *sc;
    double damp, inv_n;
    uint32_t n, n_long, n_vlong, s_chunk, units, sweep_ctas;
    int distribute, personal, l2;
    // Queued product (unit_part non-null): warps take units from sc->queue
    // and store each unit's two partial sums at unit_part[2u], [2u+1], which
    // bi_mv_fix adds in a fixed order; `units` / `unit_start` are then the
    // queued cut. Null: round-robin units with per-CTA partials in `part`.
    double *__restrict__ unit_part;
};

__device__ __forceinline__ float bi_tel(const BiArgs &a, uint32_t r) {
    return a.personal ? a.tele[r] : static_cast<float>(a.inv_n);
}

template <bool WEIGHTED>
__device__ __forceinline__ float bi_deg(const BiArgs &a, uint32_t r, uint32_t &dc) {
    dc = a.degc[r];
    return WEIGHTED ? a.degw[r] : static_cast<float>(dc);
}

// Last-CTA detection; every thread of the winning CTA returns true.
__device__ __forceinline__ bool bi_last_block(unsigned int *ticket, bool *s_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        *s_flag = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (*s_flag)
        __threadfence();
    return *s_flag;
}

constexpr int kBiThreads = 256;

// OP 0: out = in - d (A in + (m.in) tel), the product with (I - d M); `in`
// is given in gather form g (in/deg, sinks in) and x-form px.
// OP 1: out = in - d (A^T in + m (tel.in)), the product with (I - d M^T);
// acc is the weighted sum of `in` over the out-arcs of node r.
// MODE 0 accumulates (rhat, out); MODE 1 accumulates (out, s) and (out, out).
template <bool WEIGHTED, int MODE, int OP>
__device__ __forceinline__ void bi_mv_row(const BiArgs &a, uint32_t r, float acc, const float *px,
                                          float *out, double &d1, double &d2) {
    const float sv = static_cast<float>(a.sc->sink_vec);
    float q = acc;
    if (OP == 0) {
        if (a.distribute)
            q = __fadd_rn(q, __fmul_rn(sv, bi_tel(a, r)));
    } else {
        uint32_t dc;
        const float deg = bi_deg<WEIGHTED>(a, r, dc);
        q = dc ? __fdiv_rn(acc, deg) : (a.distribute ? sv : 0.f);
    }
    q = __fsub_rn(px[r], __fmul_rn(static_cast<float>(a.damp), q));
    out[r] = q;
    if (MODE == 0) {
        d1 += static_cast<double>(a.rhat[r]) * static_cast<double>(q);
    } else {
        d1 += static_cast<double>(q) * static_cast<double>(a.s[r]);
        d2 += static_cast<double>(q) * static_cast<double>(q);
    }
}

// The SpMV of one work unit per warp (the loop of sweep_unit in FP32):
// slices [s_begin, s_end), each lane one virtual row.
template <bool WEIGHTED, int MODE, int OP, int UNROLL>
__device__ __forceinline__ void bi_mv_unit(const BiArgs &a, const float *px, float *out,
                                           const float *gsrc, uint32_t s_begin, uint32_t s_end,
                                           int lane, double &d1, double &d2) {
    for (uint32_t s = s_begin; s < s_end; ++s) {
        const uint32_t off = a.slice_off[s];
        const uint32_t len = a.slice_off[s + 1] - off;
        const size_t base = static_cast<size_t>(off) * 32 + lane;
        const uint32_t *cp = a.col_sell + base;
        float acc = 0.f;
        uint32_t j = 0;
        for (; j + UNROLL <= len; j += UNROLL) {
            uint32_t c[UNROLL];
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                c[k] = ld_stream(cp + static_cast<size_t>(j + k) * 32);
            float vv[UNROLL];
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                vv[k] = c[k] != a.n ? __ldg(gsrc + c[k]) : 0.f;
            if (WEIGHTED) {
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    vv[k] = __fmul_rn(vv[k], ld_stream(a.w_sell + base + static_cast<size_t>(j + k) * 32));
            }
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                acc += vv[k];
        }
        if (j < len) {
            // the last len - j < UNROLL steps as one predicated batch (same order)
            uint32_t c[UNROLL];
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                c[k] = j + k < len ? ld_stream(cp + static_cast<size_t>(j + k) * 32) : 0u;
            float vv[UNROLL];
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                vv[k] = j + k < len && c[k] != a.n ? __ldg(gsrc + c[k]) : 0.f;
            if (WEIGHTED) {
#pragma unroll
                for (int k = 0; k < UNROLL; ++k)
                    if (j + k < len)
                        vv[k] = __fmul_rn(vv[k], ld_stream(a.w_sell + base + static_cast<size_t>(j + k) * 32));
            }
#pragma unroll
            for (int k = 0; k < UNROLL; ++k)
                if (j + k < len)
                    acc += vv[k];
        }
        if (s < a.s_chunk) {
            a.chunk_val[static_cast<size_t>(s) * 32 + lane] = acc;
        } else {
            const uint32_t r = a.n_long + (s - a.s_chunk) * 32 + lane;
            if (r < a.n)
                bi_mv_row<WEIGHTED, MODE, OP>(a, r, acc, px, out, d1, d2);
        }
    }
}

// The product. QUEUED: warps take units from sc->queue in order (as the
// queued PageRank sweep) and every unit's partials go to unit_part; else
// round-robin units with per-CTA partials.
template <bool WEIGHTED, int MODE, int OP, int THREADS, int UNROLL, bool QUEUED = false>
__global__ void __launch_bounds__(THREADS, UNROLL > 8 ? 1024 / THREADS : 1536 / THREADS) bi_mv(BiArgs a) {
    __shared__ double s_red[32];
    if (a.sc->breakdown)
        return;
    const float *px = MODE == 0 ? a.p : a.s;
    float *out = MODE == 0 ? a.v : a.t;
    const float *gsrc = OP == 0 ? a.g : px;
    const int lane = threadIdx.x & 31;
    if (QUEUED) {
        const uint32_t nw = gridDim.x * (THREADS / 32);
        for (uint32_t u = blockIdx.x * (THREADS / 32) + (threadIdx.x >> 5); u < a.units;
             u = next_unit(&a.sc->queue, a.units, nw, lane)) {
            double d1 = 0.0, d2 = 0.0;
            bi_mv_unit<WEIGHTED, MODE, OP, UNROLL>(a, px, out, gsrc, a.unit_start[u],
                                                   a.unit_start[u + 1], lane, d1, d2);
            d1 = warp_sum(d1);
            d2 = warp_sum(d2);
            if (lane == 0) {
                a.unit_part[2 * static_cast<size_t>(u)] = d1;
                a.unit_part[2 * static_cast<size_t>(u) + 1] = d2;
            }
        }
        return;
    }
    const uint32_t wpc = THREADS / 32;
    const uint32_t gw = blockIdx.x * wpc + (threadIdx.x >> 5);
    const uint32_t nw = gridDim.x * wpc;
    double d1 = 0.0, d2 = 0.0;
    for (uint32_t u = gw; u < a.units; u += nw)
        bi_mv_unit<WEIGHTED, MODE, OP, UNROLL>(a, px, out, gsrc, a.unit_start[u], a.unit_start[u + 1],
                                               lane, d1, d2);
    d1 = block_sum<THREADS>(d1, s_red);
    d2 = block_sum<THREADS>(d2, s_red);
    if (threadIdx.x == 0) {
        a.part[2 * blockIdx.x] = d1;
        a.part[2 * blockIdx.x + 1] = d2;
    }
}

// Split rows of the product, then (last CTA) the scalar that follows it:
// MODE 0: alpha = rho / (rhat, v); MODE 1: omega = (t, s) / (t, t).
template <bool WEIGHTED, int MODE, int OP>
__global__ void __launch_bounds__(kBiThreads) bi_mv_fix(BiArgs a) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    if (a.sc->breakdown)
        return;
    const float *px = MODE == 0 ? a.p : a.s;
    float *out = MODE == 0 ? a.v : a.t;
    double d1 = 0.0, d2 = 0.0;
    if (a.unit_part) {
        // Partials of a queued product: a fixed share of the units per thread.
        for (uint32_t i = blockIdx.x * kBiThreads + threadIdx.x; i < a.units;
             i += gridDim.x * kBiThreads) {
            d1 += a.unit_part[2 * static_cast<size_t>(i)];
            d2 += a.unit_part[2 * static_cast<size_t>(i) + 1];
        }
    }
    uint32_t r;
    float acc;
    if (split_row_sum<kBiThreads>(a.chunk_begin, a.chunk_val, a.n_long, a.n_vlong, r, acc))
        bi_mv_row<WEIGHTED, MODE, OP>(a, r, acc, px, out, d1, d2);
    d1 = block_sum<kBiThreads>(d1, s_red);
    d2 = block_sum<kBiThreads>(d2, s_red);
    if (threadIdx.x == 0) {
        a.fix_part[2 * blockIdx.x] = d1;
        a.fix_part[2 * blockIdx.x + 1] = d2;
    }
    if (!bi_last_block(&a.sc->ticket, &s_last))
        return;
    double t1 = 0.0, t2 = 0.0;
    const uint32_t sweep_parts = a.unit_part ? 0u : a.sweep_ctas;
    for (uint32_t i = threadIdx.x; i < sweep_parts; i += kBiThreads) {
        t1 += ((volatile double *)a.part)[2 * i];
        t2 += ((volatile double *)a.part)[2 * i + 1];
    }
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kBiThreads) {
        t1 += ((volatile double *)a.fix_part)[2 * i];
        t2 += ((volatile double *)a.fix_part)[2 * i + 1];
    }
    t1 = block_sum<kBiThreads>(t1, s_red);
    t2 = block_sum<kBiThreads>(t2, s_red);
    if (threadIdx.x == 0) {
        BiScalars *sc = a.sc;
        if (MODE == 0) {
            sc->vdot = t1;
            if (!(fabs(t1) > 1e-300) || !isfinite(t1))
                sc->breakdown = 1;
            else
                sc->alpha = sc->rho / t1;
        } else {
            sc->ts = t1;
            sc->tt = t2;
            sc->omega = t2 > 0.0 ? t1 / t2 : 0.0;
            if (!(t2 > 0.0))
                sc->breakdown = 1;
        }
        sc->ticket = 0;
        sc->queue = 0;
    }
}

// Contribution of entry i with value vv to sink_vec: m.vec (OP 0, which also
// writes the gather form g) or tel.vec (OP 1; a uniform 1/n is applied once
// to the total).
template <bool WEIGHTED, int OP>
__device__ __forceinline__ void bi_vec_entry(const BiArgs &a, uint32_t i, float vv, double &sk) {
    if (OP == 0) {
        uint32_t dc;
        const float d = bi_deg<WEIGHTED>(a, i, dc);
        a.g[i] = dc ? vv / d : vv;
        if (!dc)
            sk += vv;
    } else {
        sk += a.personal ? static_cast<double>(a.tele[i]) * static_cast<double>(vv)
                         : static_cast<double>(vv);
    }
}

// Four consecutive vector entries, moved as one 16-byte access. Every vector of
// a solve is its own allocation (256-byte aligned), so quad q of any of them
// starts on a 16-byte boundary; the vector kernels walk the n/4 full quads and
// leave the n % 4 tail to the first threads of CTA 0.
struct Quad {
    float v[4];
};

__device__ __forceinline__ Quad ld_quad(const float *p, uint32_t q) {
    const float4 t = reinterpret_cast<const float4 *>(p)[q];
    return Quad{{t.x, t.y, t.z, t.w}};
}

__device__ __forceinline__ void st_quad(float *p, uint32_t q, const Quad &f) {
    reinterpret_cast<float4 *>(p)[q] = make_float4(f.v[0], f.v[1], f.v[2], f.v[3]);
}

// bi_vec_entry over quad q (entries 4q .. 4q+3, in that order).
template <bool WEIGHTED, int OP>
__device__ __forceinline__ void bi_vec_quad(const BiArgs &a, uint32_t q, const Quad &vv, double &sk) {
    if (OP == 0) {
        const uint4 dc = reinterpret_cast<const uint4 *>(a.degc)[q];
        const uint32_t c[4] = {dc.x, dc.y, dc.z, dc.w};
        Quad d;
        if (WEIGHTED) {
            d = ld_quad(a.degw, q);
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                d.v[k] = static_cast<float>(c[k]);
        }
        Quad gq;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            gq.v[k] = c[k] ? vv.v[k] / d.v[k] : vv.v[k];
            if (!c[k])
                sk += vv.v[k];
        }
        st_quad(a.g, q, gq);
    } else if (a.personal) {
        const Quad t = ld_quad(a.tele, q);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            sk += static_cast<double>(t.v[k]) * static_cast<double>(vv.v[k]);
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            sk += static_cast<double>(vv.v[k]);
    }
}

template <int OP>
__device__ __forceinline__ double bi_sink_total(const BiArgs &a, double t) {
    return OP == 1 && !a.personal ? t * a.inv_n : t;
}

// Vector step 1: p = r + beta (p - omega v), beta = (rho/rho_prev)(alpha/omega);
// g = p in gather form; sink_vec = m.p (OP 0) or tel.p (OP 1).
template <bool WEIGHTED, int OP>
__global__ void __launch_bounds__(kBiThreads) bi_vec_p(BiArgs a) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    BiScalars *sc = a.sc;
    if (sc->breakdown)
        return;
    const double beta = (sc->rho / sc->rho_prev) * (sc->alpha / sc->omega);
    const float b = static_cast<float>(beta), om = static_cast<float>(sc->omega);
    auto step = [b, om](float r, float p, float v) {
        return __fadd_rn(r, __fmul_rn(b, __fsub_rn(p, __fmul_rn(om, v))));
    };
    double sk = 0.0;
    const uint32_t n4 = a.n >> 2, stride = gridDim.x * kBiThreads, tid = blockIdx.x * kBiThreads + threadIdx.x;
    for (uint32_t q = tid; q < n4; q += stride) {
        const Quad r = ld_quad(a.r, q), pp = ld_quad(a.p, q), v = ld_quad(a.v, q);
        Quad pv;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            pv.v[k] = step(r.v[k], pp.v[k], v.v[k]);
        st_quad(a.p, q, pv);
        bi_vec_quad<WEIGHTED, OP>(a, q, pv, sk);
    }
    for (uint32_t i = 4 * n4 + tid; i < a.n; i += stride) {
        const float pv = step(a.r[i], a.p[i], a.v[i]);
        a.p[i] = pv;
        bi_vec_entry<WEIGHTED, OP>(a, i, pv, sk);
    }
    sk = block_sum<kBiThreads>(sk, s_red);
    if (threadIdx.x == 0)
        a.part[blockIdx.x] = sk;
    if (!bi_last_block(&sc->ticket, &s_last))
        return;
    double t = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kBiThreads)
        t += ((volatile double *)a.part)[i];
    t = block_sum<kBiThreads>(t, s_red);
    if (threadIdx.x == 0) {
        sc->sink_vec = bi_sink_total<OP>(a, t);
        sc->rho_prev = sc->rho;
        sc->ticket = 0;
    }
}

// Vector step 2: s = r - alpha v; g = s in gather form; sink_vec = m.s (OP 0)
// or tel.s (OP 1).
template <bool WEIGHTED, int OP>
__global__ void __launch_bounds__(kBiThreads) bi_vec_s(BiArgs a) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    BiScalars *sc = a.sc;
    if (sc->breakdown)
        return;
    const float al = static_cast<float>(sc->alpha);
    double sk = 0.0;
    const uint32_t n4 = a.n >> 2, stride = gridDim.x * kBiThreads, tid = blockIdx.x * kBiThreads + threadIdx.x;
    for (uint32_t q = tid; q < n4; q += stride) {
        const Quad r = ld_quad(a.r, q), v = ld_quad(a.v, q);
        Quad sv;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            sv.v[k] = __fsub_rn(r.v[k], __fmul_rn(al, v.v[k]));
        st_quad(a.s, q, sv);
        bi_vec_quad<WEIGHTED, OP>(a, q, sv, sk);
    }
    for (uint32_t i = 4 * n4 + tid; i < a.n; i += stride) {
        const float sv = __fsub_rn(a.r[i], __fmul_rn(al, a.v[i]));
        a.s[i] = sv;
        bi_vec_entry<WEIGHTED, OP>(a, i, sv, sk);
    }
    sk = block_sum<kBiThreads>(sk, s_red);
    if (threadIdx.x == 0)
        a.part[blockIdx.x] = sk;
    if (!bi_last_block(&sc->ticket, &s_last))
        return;
    double t = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kBiThreads)
        t += ((volatile double *)a.part)[i];
    t = block_sum<kBiThreads>(t, s_red);
    if (threadIdx.x == 0) {
        sc->sink_vec = bi_sink_total<OP>(a, t);
        sc->ticket = 0;
    }
}

// Vector step 3: x += alpha p + omega s; r = s - omega t; res = |r|; rho = (rhat, r).
static __global__ void __launch_bounds__(kBiThreads) bi_vec_x(BiArgs a) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    BiScalars *sc = a.sc;
    if (sc->breakdown)
        return;
    const float al = static_cast<float>(sc->alpha), om = static_cast<float>(sc->omega);
    double nr = 0.0, rr = 0.0;
    auto acc = [&](float rv, float rh) {
        const double d = rv;
        nr += a.l2 ? d * d : fabs(d);
        rr += static_cast<double>(rh) * d;
    };
    const uint32_t n4 = a.n >> 2, stride = gridDim.x * kBiThreads, tid = blockIdx.x * kBiThreads + threadIdx.x;
    for (uint32_t q = tid; q < n4; q += stride) {
        const Quad x = ld_quad(a.x, q), p = ld_quad(a.p, q), sv = ld_quad(a.s, q), t = ld_quad(a.t, q),
                   rh = ld_quad(a.rhat, q);
        Quad xn, rn;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            xn.v[k] = __fadd_rn(x.v[k], __fadd_rn(__fmul_rn(al, p.v[k]), __fmul_rn(om, sv.v[k])));
            rn.v[k] = __fsub_rn(sv.v[k], __fmul_rn(om, t.v[k]));
        }
        st_quad(a.x, q, xn);
        st_quad(a.r, q, rn);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            acc(rn.v[k], rh.v[k]);
    }
    for (uint32_t i = 4 * n4 + tid; i < a.n; i += stride) {
        a.x[i] = __fadd_rn(a.x[i], __fadd_rn(__fmul_rn(al, a.p[i]), __fmul_rn(om, a.s[i])));
        const float rv = __fsub_rn(a.s[i], __fmul_rn(om, a.t[i]));
        a.r[i] = rv;
        acc(rv, a.rhat[i]);
    }
    nr = block_sum<kBiThreads>(nr, s_red);
    rr = block_sum<kBiThreads>(rr, s_red);
    if (threadIdx.x == 0) {
        a.part[2 * blockIdx.x] = nr;
        a.part[2 * blockIdx.x + 1] = rr;
    }
    if (!bi_last_block(&sc->ticket, &s_last))
        return;
    double t1 = 0.0, t2 = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kBiThreads) {
        t1 += ((volatile double *)a.part)[2 * i];
        t2 += ((volatile double *)a.part)[2 * i + 1];
    }
    t1 = block_sum<kBiThreads>(t1, s_red);
    t2 = block_sum<kBiThreads>(t2, s_red);
    if (threadIdx.x == 0) {
        sc->res = a.l2 ? sqrt(t1) : t1;
        sc->rho = t2;
        if (!(fabs(t2) > 1e-300) || !isfinite(t2))
            sc->breakdown = 1;
        sc->ticket = 0;
    }
}

// Start of a solve from x = 0: r = rhat = b (x-form, given in r), p = v = 0;
// rho = (b, b), res = |b|; rho_prev = alpha = omega = 1.
static __global__ void __launch_bounds__(kBiThreads) bi_start(BiArgs a) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    BiScalars *sc = a.sc;
    double nr = 0.0, rr = 0.0;
    auto acc = [&](float b) {
        const double d = b;
        nr += a.l2 ? d * d : fabs(d);
        rr += d * d;
    };
    const Quad zero{{0.f, 0.f, 0.f, 0.f}};
    const uint32_t n4 = a.n >> 2, stride = gridDim.x * kBiThreads, tid = blockIdx.x * kBiThreads + threadIdx.x;
    for (uint32_t q = tid; q < n4; q += stride) {
        const Quad b = ld_quad(a.r, q);
        st_quad(a.rhat, q, b);
        st_quad(a.x, q, zero);
        st_quad(a.p, q, zero);
        st_quad(a.v, q, zero);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            acc(b.v[k]);
    }
    for (uint32_t i = 4 * n4 + tid; i < a.n; i += stride) {
        const float b = a.r[i];
        a.rhat[i] = b;
        a.x[i] = 0.f;
        a.p[i] = 0.f;
        a.v[i] = 0.f;
        acc(b);
    }
    if (a.g && blockIdx.x == 0 && threadIdx.x == 0)
        a.g[a.n] = 0.f;
    nr = block_sum<kBiThreads>(nr, s_red);
    rr = block_sum<kBiThreads>(rr, s_red);
    if (threadIdx.x == 0) {
        a.part[2 * blockIdx.x] = nr;
        a.part[2 * blockIdx.x + 1] = rr;
    }
    if (!bi_last_block(&sc->ticket, &s_last))
        return;
    double t1 = 0.0, t2 = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kBiThreads) {
        t1 += ((volatile double *)a.part)[2 * i];
        t2 += ((volatile double *)a.part)[2 * i + 1];
    }
    t1 = block_sum<kBiThreads>(t1, s_red);
    t2 = block_sum<kBiThreads>(t2, s_red);
    if (threadIdx.x == 0) {
        sc->res = a.l2 ? sqrt(t1) : t1;
        sc->rho = t2;
        sc->rho_prev = 1.0;
        sc->alpha = 1.0;
        sc->omega = 1.0;
        sc->breakdown = t2 > 0.0 ? 0 : 1;
        sc->ticket = 0;
    }
}

// Right-hand side of the first solve: b = (1-d) t.
static __global__ void bi_rhs_teleport(BiArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.n)
        a.r[i] = static_cast<float>(1.0 - a.damp) * bi_tel(a, i);
}

// FP64 iterate from the FP32 solution (x64 = x32), or add a correction
// (x64 += x32); write its gather form y64 and the sink term of the FP64 sweep.
template <bool WEIGHTED>
__global__ void __launch_bounds__(kBiThreads)
    bi_to_fp64(const float *__restrict__ x32, double *__restrict__ x64, double *__restrict__ y64,
               const uint32_t *__restrict__ degc, const double *__restrict__ degw, uint32_t n,
               int add, double *part, IterState *st, unsigned int *ticket, int distribute,
               int personal) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    double sk = 0.0;
    auto entry = [&](double x32v, double x64v, uint32_t dc, double dw, double &xo, double &yo) {
        const double x = add ? x64v + x32v : x32v;
        xo = x;
        const double d = WEIGHTED ? dw : static_cast<double>(dc);
        yo = dc ? x / d : x;
        if (!dc)
            sk += x;
    };
    // Quads of entries: 16-byte loads of x32 and degc, 2 x 16 bytes of each
    // FP64 vector (all separate allocations, so 16-byte aligned).
    const uint32_t n4 = n >> 2, stride = gridDim.x * kBiThreads, tid = blockIdx.x * kBiThreads + threadIdx.x;
    for (uint32_t q = tid; q < n4; q += stride) {
        const Quad xs = ld_quad(x32, q);
        const uint4 dc = reinterpret_cast<const uint4 *>(degc)[q];
        const uint32_t c[4] = {dc.x, dc.y, dc.z, dc.w};
        double xo[4], yo[4], xi[4] = {0.0, 0.0, 0.0, 0.0}, dw[4] = {0.0, 0.0, 0.0, 0.0};
        if (add) {
            const double2 a0 = reinterpret_cast<const double2 *>(x64)[2 * q];
            const double2 a1 = reinterpret_cast<const double2 *>(x64)[2 * q + 1];
            xi[0] = a0.x, xi[1] = a0.y, xi[2] = a1.x, xi[3] = a1.y;
        }
        if (WEIGHTED) {
            const double2 w0 = reinterpret_cast<const double2 *>(degw)[2 * q];
            const double2 w1 = reinterpret_cast<const double2 *>(degw)[2 * q + 1];
            dw[0] = w0.x, dw[1] = w0.y, dw[2] = w1.x, dw[3] = w1.y;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
            entry(static_cast<double>(xs.v[k]), xi[k], c[k], dw[k], xo[k], yo[k]);
        reinterpret_cast<double2 *>(x64)[2 * q] = make_double2(xo[0], xo[1]);
        reinterpret_cast<double2 *>(x64)[2 * q + 1] = make_double2(xo[2], xo[3]);
        reinterpret_cast<double2 *>(y64)[2 * q] = make_double2(yo[0], yo[1]);
        reinterpret_cast<double2 *>(y64)[2 * q + 1] = make_double2(yo[2], yo[3]);
    }
    for (uint32_t i = 4 * n4 + tid; i < n; i += stride)
        entry(static_cast<double>(x32[i]), add ? x64[i] : 0.0, degc[i], WEIGHTED ? degw[i] : 0.0,
              x64[i], y64[i]);
    sk = block_sum<kBiThreads>(sk, s_red);
    if (threadIdx.x == 0)
        part[blockIdx.x] = sk;
    if (!bi_last_block(ticket, &s_last))
        return;
    double t = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kBiThreads)
        t += ((volatile double *)part)[i];
    t = block_sum<kBiThreads>(t, s_red);
    if (threadIdx.x == 0) {
        st->sink_mass = t;
        st->sink_coef = distribute ? (personal ? t : t / static_cast<double>(n)) : 0.0;
        *ticket = 0;
    }
}

// Right-hand side of a correction solve: r32 = x' - x from the FP64 sweep.
template <bool WEIGHTED>
__global__ void bi_residual_rhs(const double *__restrict__ y64_new, const double *__restrict__ x64,
                                const uint32_t *__restrict__ degc, const double *__restrict__ degw,
                                uint32_t n, float *__restrict__ r32) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t dc = degc[i];
    const double d = WEIGHTED ? degw[i] : static_cast<double>(dc);
    const double xn = dc ? __dmul_rn(y64_new[i], d) : y64_new[i];
    r32[i] = static_cast<float>(xn - x64[i]);
}

// ---------------------------------------------------------------------------
// Host driver of one BiCGSTAB solve

struct BiLaunch {
    cudaStream_t stream = nullptr;
    int sweep_shape = 0;
    unsigned sweep_ctas = 0, vec_ctas = 0, fix_ctas = 0;
    BiScalars *d_sc = nullptr;    // device scalars
    BiScalars *h_sc = nullptr;    // pinned host copy
    std::atomic<int> *cancel = nullptr;
    uint64_t launches = 0, matvecs = 0;
};

// Solve (I - d M) x = r (OP 0) or (I - d M^T) x = r (OP 1) from x = 0, with
// the right-hand side in a.r, until |r| <= max(rel * |r0|, floor). Four
// BiCGSTAB steps (28 launches) go out between status read-backs.
template <bool WEIGHTED, int OP>
void bi_solve(const BiArgs &a, BiLaunch &L, double rel, double floor) {
    cudaStream_t s = L.stream;
    for (const void *v : {static_cast<const void *>(a.x), static_cast<const void *>(a.r),
                          static_cast<const void *>(a.rhat), static_cast<const void *>(a.p),
                          static_cast<const void *>(a.v), static_cast<const void *>(a.s),
                          static_cast<const void *>(a.t), static_cast<const void *>(a.g),
                          static_cast<const void *>(a.degc), static_cast<const void *>(a.degw),
                          static_cast<const void *>(a.tele)})
        if (reinterpret_cast<uintptr_t>(v) % 16)
            throw Error(NKG_ERR_INVALID_ARG, "BiCGSTAB vectors must be 16-byte aligned");
    bi_start<<<L.vec_ctas, kBiThreads, 0, s>>>(a);
    NKG_CUDA(cudaMemcpyAsync(L.h_sc, L.d_sc, sizeof(BiScalars), cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    const double inner_tol = L.h_sc->res * rel > floor ? L.h_sc->res * rel : floor;
    L.launches += 1;
    for (int it = 0; it < 400 && !L.h_sc->breakdown && L.h_sc->res > inner_tol; it += 4) {
        for (int k = 0; k < 4; ++k) {
            bi_vec_p<WEIGHTED, OP><<<L.vec_ctas, kBiThreads, 0, s>>>(a);
            with_sweep_shape(L.sweep_shape, [&](auto S) {
                using Sh = decltype(S);
                if (a.unit_part)
                    bi_mv<WEIGHTED, 0, OP, Sh::threads, Sh::unroll, true>
                        <<<L.sweep_ctas, Sh::threads, 0, s>>>(a);
                else
                    bi_mv<WEIGHTED, 0, OP, Sh::threads, Sh::unroll><<<L.sweep_ctas, Sh::threads, 0, s>>>(a);
            });
            bi_mv_fix<WEIGHTED, 0, OP><<<L.fix_ctas, kBiThreads, 0, s>>>(a);
            bi_vec_s<WEIGHTED, OP><<<L.vec_ctas, kBiThreads, 0, s>>>(a);
            with_sweep_shape(L.sweep_shape, [&](auto S) {
                using Sh = decltype(S);
                if (a.unit_part)
                    bi_mv<WEIGHTED, 1, OP, Sh::threads, Sh::unroll, true>
                        <<<L.sweep_ctas, Sh::threads, 0, s>>>(a);
                else
                    bi_mv<WEIGHTED, 1, OP, Sh::threads, Sh::unroll><<<L.sweep_ctas, Sh::threads, 0, s>>>(a);
            });
            bi_mv_fix<WEIGHTED, 1, OP><<<L.fix_ctas, kBiThreads, 0, s>>>(a);
            bi_vec_x<<<L.vec_ctas, kBiThreads, 0, s>>>(a);
        }
        NKG_CUDA(cudaGetLastError());
        L.launches += 28;
        L.matvecs += 8;
        NKG_CUDA(cudaMemcpyAsync(L.h_sc, L.d_sc, sizeof(BiScalars), cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        if (L.cancel && L.cancel->load())
            throw Error(NKG_ERR_CANCELLED, "PageRank run cancelled");
    }
}

} // namespace nkg
