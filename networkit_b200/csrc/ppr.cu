// Batched personalised PageRank: k teleport vectors t_j = e_{seed_j} solved
// together as one FP32 SpMM over the shared in-CSR (no reference counterpart;
// each column is PageRank.cpp:56-70 with the uniform teleport replaced by
// t_j). Per column: FP64 residual, FP64 sink mass, and the column stops
// (freezes) once its residual is at most tol.
//
// Layout: the iterate is node-major, Y[r * kp + j] (kp = 32 * CPL columns,
// CPL per lane), in gather form (x/deg, sinks x). A warp owns one virtual
// row (a whole row, or a kChunk-arc chunk of a long row); per arc it broadcasts
// the source id and every lane loads its CPL columns of that source's row:
// kp * 4 contiguous bytes per arc, float4-coalesced. Warps walk contiguous,
// cost-balanced ranges of virtual rows, so every sum has a fixed order.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "graph.hpp"
#include "host.hpp"

namespace nkg {
namespace {

constexpr int kPprThreads = 256;
constexpr int kPprWarps = kPprThreads / 32;

struct PprState {
    unsigned long long iteration;
    int all_done;
    unsigned int ticket;
};

struct PprArgs {
    const uint32_t *__restrict__ row_ptr;    // n+1 (relabelled in-CSR)
    const uint32_t *__restrict__ col;
    const uint32_t *__restrict__ degc;
    const uint32_t *__restrict__ chunk_begin;  // n_long+1
    const uint32_t *__restrict__ chunk_row;    // per chunk: its row
    const uint32_t *__restrict__ unit_start;   // units+1 virtual-row indices
    const uint32_t *__restrict__ seed;         // kp: relabelled seed id (kNone: padding column)
    const float *__restrict__ y_in;            // n * kp
    float *__restrict__ y_out;
    float *__restrict__ chunk_val;             // n_chunks * kp
    int *__restrict__ active;                  // kp
    float *__restrict__ sink_coef;             // kp: sink term of the next sweep
    double *__restrict__ cta_res;              // per CTA * kp
    double *__restrict__ cta_sink;
    double *__restrict__ col_res;              // kp: last residual
    unsigned long long *__restrict__ col_iter; // kp: sweeps until converged
    PprState *st;
    double damp, tol;
    unsigned long long max_iterations;
    uint32_t n, n_long, n_chunks, units, kp, sweep_ctas;
    int l2, distribute;
};

// Virtual rows: [0, n_chunks) chunks of the long rows, then rows n_long..n-1.
__device__ __forceinline__ void vrow_range(const PprArgs &a, uint32_t v, uint32_t &r, uint32_t &b,
                                           uint32_t &e) {
    if (v < a.n_chunks) {
        r = a.chunk_row[v];
        const uint32_t c = v - a.chunk_begin[r];
        b = a.row_ptr[r] + c * kChunk;
        e = min(a.row_ptr[r + 1], b + kChunk);
    } else {
        r = a.n_long + (v - a.n_chunks);
        b = a.row_ptr[r];
        e = a.row_ptr[r + 1];
    }
}

template <int CPL>
__device__ __forceinline__ void accumulate(const PprArgs &a, uint32_t b, uint32_t e, int lane,
                                           float (&acc)[CPL]) {
#pragma unroll
    for (int q = 0; q < CPL; ++q)
        acc[q] = 0.f;
    for (uint32_t base = b; base < e; base += 32) {
        const uint32_t cnt = min(32u, e - base);
        const uint32_t cl = lane < static_cast<int>(cnt) ? ld_stream(a.col + base + lane) : 0u;
        uint32_t i = 0;
        for (; i + 4 <= cnt; i += 4) {
            float4 v[4][CPL / 4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t src = __shfl_sync(0xffffffffu, cl, i + u);
                const float4 *p =
                    reinterpret_cast<const float4 *>(a.y_in + static_cast<size_t>(src) * a.kp) +
                    lane * (CPL / 4);
#pragma unroll
                for (int q = 0; q < CPL / 4; ++q)
                    v[u][q] = __ldg(p + q);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int q = 0; q < CPL / 4; ++q) {
                    acc[4 * q + 0] += v[u][q].x;
                    acc[4 * q + 1] += v[u][q].y;
                    acc[4 * q + 2] += v[u][q].z;
                    acc[4 * q + 3] += v[u][q].w;
                }
        }
        for (; i < cnt; ++i) {
            const uint32_t src = __shfl_sync(0xffffffffu, cl, i);
            const float4 *p =
                reinterpret_cast<const float4 *>(a.y_in + static_cast<size_t>(src) * a.kp) +
                lane * (CPL / 4);
#pragma unroll
            for (int q = 0; q < CPL / 4; ++q) {
                const float4 v = __ldg(p + q);
                acc[4 * q + 0] += v.x;
                acc[4 * q + 1] += v.y;
                acc[4 * q + 2] += v.z;
                acc[4 * q + 3] += v.w;
            }
        }
    }
}

// Finish row r for this lane's CPL columns.
template <int CPL>
__device__ __forceinline__ void finish(const PprArgs &a, uint32_t r, int lane, const float (&acc)[CPL],
                                       const int (&act)[CPL], const float (&sc)[CPL],
                                       const uint32_t (&seed)[CPL], double (&res)[CPL],
                                       double (&sink)[CPL]) {
    const uint32_t dc = ld_stream(a.degc + r);
    const float deg = static_cast<float>(dc);
    const float4 *pin = reinterpret_cast<const float4 *>(a.y_in + static_cast<size_t>(r) * a.kp) +
                        lane * (CPL / 4);
    float4 *pout = reinterpret_cast<float4 *>(a.y_out + static_cast<size_t>(r) * a.kp) +
                   lane * (CPL / 4);
    const float dampf = static_cast<float>(a.damp), omd = static_cast<float>(1.0 - a.damp);
#pragma unroll
    for (int q = 0; q < CPL / 4; ++q) {
        const float4 yo4 = __ldg(pin + q);
        float yo[4] = {yo4.x, yo4.y, yo4.z, yo4.w};
        float yn[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int c = 4 * q + t;
            if (!act[c]) {
                yn[t] = yo[t];
                continue;
            }
            const float tel = (r == seed[c]) ? 1.f : 0.f;
            float s = acc[c];
            if (a.distribute)
                s = __fadd_rn(s, __fmul_rn(sc[c], tel));
            float x = __fmul_rn(s, dampf);
            x = __fadd_rn(x, __fmul_rn(omd, tel));
            const float xo = dc ? __fmul_rn(yo[t], deg) : yo[t];
            const double d = static_cast<double>(xo) - static_cast<double>(x);
            res[c] += a.l2 ? d * d : fabs(d);
            if (dc) {
                yn[t] = x / deg;
            } else {
                yn[t] = x;
                sink[c] += static_cast<double>(x);
            }
        }
        pout[q] = make_float4(yn[0], yn[1], yn[2], yn[3]);
    }
}

// Per-column block reduction of res/sink into cta_res/cta_sink[blockIdx.x*kp ..].
template <int CPL>
__device__ __forceinline__ void column_partials(const PprArgs &a, int lane, const double (&res)[CPL],
                                                const double (&sink)[CPL], double *s_buf,
                                                double *out_res, double *out_sink) {
    const int wid = threadIdx.x >> 5;
    const uint32_t kp = a.kp;
    for (int pass = 0; pass < 2; ++pass) {
        __syncthreads();
#pragma unroll
        for (int c = 0; c < CPL; ++c)
            s_buf[wid * kp + lane * CPL + c] = pass == 0 ? res[c] : sink[c];
        __syncthreads();
        for (uint32_t col = threadIdx.x; col < kp; col += kPprThreads) {
            double s = 0.0;
            for (int w = 0; w < kPprWarps; ++w)
                s += s_buf[w * kp + col];
            (pass == 0 ? out_res : out_sink)[static_cast<size_t>(blockIdx.x) * kp + col] = s;
        }
    }
    __threadfence();  // partials visible device-wide before any ticket
}

template <int CPL>
__device__ __forceinline__ void load_columns(const PprArgs &a, int lane, int (&act)[CPL],
                                             float (&sc)[CPL], uint32_t (&seed)[CPL]) {
#pragma unroll
    for (int c = 0; c < CPL; ++c) {
        const uint32_t col = lane * CPL + c;
        act[c] = a.active[col];
        sc[c] = a.sink_coef[col];
        seed[c] = a.seed[col];
    }
}

template <int CPL>
__global__ void __launch_bounds__(kPprThreads) ppr_sweep(PprArgs a) {
    extern __shared__ double s_buf[];
    if (*(volatile int *)&a.st->all_done)
        return;
    const int lane = threadIdx.x & 31;
    int act[CPL];
    float sc[CPL];
    uint32_t seed[CPL];
    load_columns<CPL>(a, lane, act, sc, seed);
    double res[CPL], sink[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c)
        res[c] = sink[c] = 0.0;
    const uint32_t gw = blockIdx.x * kPprWarps + (threadIdx.x >> 5);
    const uint32_t nw = gridDim.x * kPprWarps;
    for (uint32_t u = gw; u < a.units; u += nw) {
        const uint32_t v_end = a.unit_start[u + 1];
        for (uint32_t v = a.unit_start[u]; v < v_end; ++v) {
            uint32_t r, b, e;
            vrow_range(a, v, r, b, e);
            float acc[CPL];
            accumulate<CPL>(a, b, e, lane, acc);
            if (v < a.n_chunks) {
                float4 *p = reinterpret_cast<float4 *>(a.chunk_val + static_cast<size_t>(v) * a.kp) +
                            lane * (CPL / 4);
#pragma unroll
                for (int q = 0; q < CPL / 4; ++q)
                    p[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
            } else {
                finish<CPL>(a, r, lane, acc, act, sc, seed, res, sink);
            }
        }
    }
    column_partials<CPL>(a, lane, res, sink, s_buf, a.cta_res, a.cta_sink);
}

// Long rows: sum their chunk partials in order (one warp per row), finish
// them, then the last CTA closes the iteration per column.
template <int CPL>
__global__ void __launch_bounds__(kPprThreads) ppr_fixup(PprArgs a, double *fix_res,
                                                         double *fix_sink) {
    extern __shared__ double s_buf[];
    __shared__ bool s_last;
    if (*(volatile int *)&a.st->all_done)
        return;
    const int lane = threadIdx.x & 31;
    int act[CPL];
    float sc[CPL];
    uint32_t seed[CPL];
    load_columns<CPL>(a, lane, act, sc, seed);
    double res[CPL], sink[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c)
        res[c] = sink[c] = 0.0;
    const uint32_t gw = blockIdx.x * kPprWarps + (threadIdx.x >> 5);
    const uint32_t nw = gridDim.x * kPprWarps;
    for (uint32_t r = gw; r < a.n_long; r += nw) {
        float acc[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c)
            acc[c] = 0.f;
        for (uint32_t k = a.chunk_begin[r]; k < a.chunk_begin[r + 1]; ++k) {
            const float4 *p = reinterpret_cast<const float4 *>(a.chunk_val + static_cast<size_t>(k) * a.kp) +
                              lane * (CPL / 4);
#pragma unroll
            for (int q = 0; q < CPL / 4; ++q) {
                const float4 v = p[q];
                acc[4 * q] += v.x;
                acc[4 * q + 1] += v.y;
                acc[4 * q + 2] += v.z;
                acc[4 * q + 3] += v.w;
            }
        }
        finish<CPL>(a, r, lane, acc, act, sc, seed, res, sink);
    }
    column_partials<CPL>(a, lane, res, sink, s_buf, fix_res, fix_sink);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&a.st->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    const unsigned long long it = a.st->iteration + 1;
    int any_active = 0;
    for (uint32_t col = threadIdx.x; col < a.kp; col += kPprThreads) {
        double r = 0.0, s = 0.0;
        for (uint32_t i = 0; i < a.sweep_ctas; ++i) {
            r += ((volatile double *)a.cta_res)[static_cast<size_t>(i) * a.kp + col];
            s += ((volatile double *)a.cta_sink)[static_cast<size_t>(i) * a.kp + col];
        }
        for (uint32_t i = 0; i < gridDim.x; ++i) {
            r += ((volatile double *)fix_res)[static_cast<size_t>(i) * a.kp + col];
            s += ((volatile double *)fix_sink)[static_cast<size_t>(i) * a.kp + col];
        }
        if (a.active[col]) {
            const double norm = a.l2 ? sqrt(r) : r;
            a.col_res[col] = norm;
            a.col_iter[col] = it;
            a.sink_coef[col] = static_cast<float>(s);
            if (norm <= a.tol || it >= a.max_iterations)
                a.active[col] = 0;
            else
                any_active = 1;
        }
    }
    any_active = __syncthreads_or(any_active);
    if (threadIdx.x == 0) {
        a.st->iteration = it;
        a.st->ticket = 0;
        __threadfence();
        a.st->all_done = any_active ? 0 : 1;
    }
}

// x = 1/n in gather form for every column.
__global__ void ppr_init(float *__restrict__ y, const uint32_t *__restrict__ degc, uint32_t n,
                         uint32_t kp, float x0) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= static_cast<uint64_t>(n) * kp)
        return;
    const uint32_t dc = degc[i / kp];
    y[i] = dc ? x0 / static_cast<float>(dc) : x0;
}

// Column sums of x (and of x over sinks), FP64, fixed order: one warp per row.
template <int CPL>
__global__ void __launch_bounds__(kPprThreads) ppr_colsum(const float *__restrict__ y,
                                                          const uint32_t *__restrict__ degc,
                                                          uint32_t n, uint32_t kp, double *part_sum,
                                                          double *part_sink) {
    extern __shared__ double s_buf[];
    const int lane = threadIdx.x & 31;
    double sum[CPL], sink[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c)
        sum[c] = sink[c] = 0.0;
    for (uint32_t r = blockIdx.x * kPprWarps + (threadIdx.x >> 5); r < n; r += gridDim.x * kPprWarps) {
        const uint32_t dc = degc[r];
        const float4 *p = reinterpret_cast<const float4 *>(y + static_cast<size_t>(r) * kp) +
                          lane * (CPL / 4);
#pragma unroll
        for (int q = 0; q < CPL / 4; ++q) {
            const float4 v = p[q];
            const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const float x = dc ? __fmul_rn(vv[t], static_cast<float>(dc)) : vv[t];
                sum[4 * q + t] += x;
                if (!dc)
                    sink[4 * q + t] += x;
            }
        }
    }
    PprArgs dummy{};
    dummy.kp = kp;
    column_partials<CPL>(dummy, lane, sum, sink, s_buf, part_sum, part_sink);
}

// Column j of the output (caller's ids): out[j*z + o] = x_j(inv[o]) / factor_j.
// A block transposes 32 nodes x kp columns through shared memory.
__global__ void ppr_output(const float *__restrict__ y, const uint32_t *__restrict__ degc,
                           const uint32_t *__restrict__ inv, uint64_t z, uint32_t n, uint32_t k,
                           uint32_t kp, const double *__restrict__ factor, float *__restrict__ out) {
    extern __shared__ float s_tile[];  // 32 x (kp + 1)
    const uint64_t o0 = static_cast<uint64_t>(blockIdx.x) * 32;
    for (uint32_t i = threadIdx.x; i < 32 * kp; i += blockDim.x) {
        const uint32_t node = i / kp, col = i % kp;
        const uint64_t o = o0 + node;
        float v = 0.f;
        if (o < z) {
            const uint32_t r = inv[o];
            if (r == kNone) {
                v = 1.f / static_cast<float>(n);
            } else {
                const uint32_t dc = degc[r];
                const float yv = y[static_cast<size_t>(r) * kp + col];
                const double x = dc ? static_cast<double>(__fmul_rn(yv, static_cast<float>(dc)))
                                    : static_cast<double>(yv);
                v = static_cast<float>(x / factor[col]);
            }
        }
        s_tile[node * (kp + 1) + col] = v;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < 32 * k; i += blockDim.x) {
        const uint32_t col = i / 32, node = i % 32;
        const uint64_t o = o0 + node;
        if (o < z)
            out[static_cast<size_t>(col) * z + o] = s_tile[node * (kp + 1) + col];
    }
}

__global__ void ppr_vrow_cost(const uint32_t *__restrict__ row_ptr,
                              const uint32_t *__restrict__ chunk_begin,
                              const uint32_t *__restrict__ chunk_row, uint32_t n_chunks,
                              uint32_t n_long, uint32_t n, uint64_t *__restrict__ cost) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nv = n_chunks + (n - n_long);
    if (v >= nv)
        return;
    uint32_t len;
    if (v < n_chunks) {
        const uint32_t r = chunk_row[v];
        const uint32_t c = v - chunk_begin[r];
        const uint32_t b = row_ptr[r] + c * kChunk;
        len = min(row_ptr[r + 1], b + kChunk) - b;
    } else {
        const uint32_t r = n_long + (v - n_chunks);
        len = row_ptr[r + 1] - row_ptr[r];
    }
    cost[v] = static_cast<uint64_t>(len) + 4;  // arcs + the row's epilogue
}

__global__ void ppr_unit_bounds(const uint64_t *__restrict__ cost_incl, uint32_t nv, uint32_t units,
                                uint32_t *__restrict__ unit_start) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u > units)
        return;
    if (u == 0) {
        unit_start[0] = 0;
        return;
    }
    if (u == units) {
        unit_start[u] = nv;
        return;
    }
    const uint64_t target = cost_incl[nv - 1] * u / units;
    uint32_t lo = 0, hi = nv;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (cost_incl[mid] < target)
            lo = mid + 1;
        else
            hi = mid;
    }
    unit_start[u] = lo + 1 < nv ? lo + 1 : nv;
}

__global__ void ppr_chunk_rows(const uint32_t *__restrict__ chunk_begin, uint32_t n_long,
                               uint32_t *__restrict__ chunk_row) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint32_t r = warp; r < n_long; r += nwarps)
        for (uint32_t k = chunk_begin[r] + lane; k < chunk_begin[r + 1]; k += 32)
            chunk_row[k] = r;
}

__global__ void ppr_seeds(const uint32_t *__restrict__ seeds_orig, const uint32_t *__restrict__ inv,
                          uint32_t k, uint32_t kp, uint32_t *__restrict__ seed, int *__restrict__ active,
                          float *__restrict__ sink_coef, float s0, int *__restrict__ bad) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= kp)
        return;
    if (j < k) {
        const uint32_t r = inv[seeds_orig[j]];
        if (r == kNone)
            atomicExch(bad, 1);
        seed[j] = r;
        active[j] = 1;
        sink_coef[j] = s0;
    } else {
        seed[j] = kNone;
        active[j] = 0;
        sink_coef[j] = 0.f;
    }
}

template <int CPL>
void run_ppr(nkg_graph *g, const nkg_pr_params &p, uint32_t k, const uint32_t *seeds_host,
             float *out, bool out_on_device, uint64_t *iters_out, nkg_stats *stats) {
    cudaStream_t s = g->stream;
    const uint32_t n = static_cast<uint32_t>(g->n);
    const uint32_t kp = 32u * CPL;
    const unsigned sms = num_sms(g->device);
    NKG_CUDA(cudaEventRecord(g->ev0, s));

    // Virtual rows and their cost-balanced units.
    const uint32_t nv = g->fw.n_chunks + (n - g->fw.n_long);
    DeviceArray<uint32_t> chunk_row(std::max<uint32_t>(g->fw.n_chunks, 1));
    if (g->fw.n_long)
        ppr_chunk_rows<<<sms * 4, 256, 0, s>>>(g->fw.chunk_begin.get(), g->fw.n_long, chunk_row.get());
    int occ = 0;
    const size_t smem_sweep = static_cast<size_t>(kPprWarps) * kp * sizeof(double);
    NKG_CUDA(cudaFuncSetAttribute(ppr_sweep<CPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem_sweep)));
    NKG_CUDA(cudaFuncSetAttribute(ppr_fixup<CPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem_sweep)));
    NKG_CUDA(cudaFuncSetAttribute(ppr_colsum<CPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem_sweep)));
    NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ppr_sweep<CPL>, kPprThreads,
                                                           smem_sweep));
    occ = std::max(occ, 1);
    const uint32_t sweep_ctas = static_cast<uint32_t>(
        std::max<uint64_t>(1, std::min<uint64_t>(static_cast<uint64_t>(occ) * sms,
                                                 (nv + kPprWarps - 1) / kPprWarps)));
    const uint32_t units = std::max<uint32_t>(
        1, std::min<uint32_t>(sweep_ctas * kPprWarps * 4, std::max<uint32_t>(nv, 1)));
    DeviceArray<uint64_t> cost(std::max<uint32_t>(nv, 1)), cost_incl(std::max<uint32_t>(nv, 1));
    DeviceArray<uint32_t> unit_start(units + 1);
    if (nv) {
        ppr_vrow_cost<<<ceil_div(nv, 256), 256, 0, s>>>(g->row_ptr.get(), g->fw.chunk_begin.get(),
                                                        chunk_row.get(), g->fw.n_chunks, g->fw.n_long,
                                                        n, cost.get());
        size_t tb = 0;
        NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, cost.get(), cost_incl.get(),
                                               static_cast<int64_t>(nv), s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb, cost.get(), cost_incl.get(),
                                               static_cast<int64_t>(nv), s));
    }
    ppr_unit_bounds<<<ceil_div(units + 1, 256), 256, 0, s>>>(cost_incl.get(), nv, units,
                                                             unit_start.get());
    const uint32_t fix_ctas = std::max<uint32_t>(
        1, std::min<uint32_t>(sms * 2, (g->fw.n_long + kPprWarps - 1) / kPprWarps));

    // Per-call buffers.
    DeviceArray<float> y0(static_cast<size_t>(n) * kp), y1(static_cast<size_t>(n) * kp);
    DeviceArray<float> chunk_val(static_cast<size_t>(std::max<uint32_t>(g->fw.n_chunks, 1)) * kp);
    DeviceArray<uint32_t> d_seeds_orig(k), seed(kp);
    DeviceArray<int> active(kp), bad(1);
    DeviceArray<float> sink_coef(kp);
    DeviceArray<double> cta_res(static_cast<size_t>(sweep_ctas) * kp),
        cta_sink(static_cast<size_t>(sweep_ctas) * kp), fix_res(static_cast<size_t>(fix_ctas) * kp),
        fix_sink(static_cast<size_t>(fix_ctas) * kp), col_res(kp);
    DeviceArray<unsigned long long> col_iter(kp);
    DeviceArray<PprState> st(1);
    NKG_CUDA(cudaMemcpyAsync(d_seeds_orig.get(), seeds_host, k * sizeof(uint32_t),
                             cudaMemcpyHostToDevice, s));
    NKG_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(int), s));
    NKG_CUDA(cudaMemsetAsync(st.get(), 0, sizeof(PprState), s));
    NKG_CUDA(cudaMemsetAsync(col_iter.get(), 0, kp * sizeof(unsigned long long), s));
    NKG_CUDA(cudaMemsetAsync(col_res.get(), 0, kp * sizeof(double), s));
    const float x0 = 1.f / static_cast<float>(n);
    // distributeSinks: the first sweep spreads the start vector's sink mass.
    const float s0 = p.distribute_sinks ? static_cast<float>(static_cast<double>(g->sinks) / n) : 0.f;
    ppr_seeds<<<ceil_div(kp, 256), 256, 0, s>>>(d_seeds_orig.get(), g->inv.get(), k, kp,
                                                seed.get(), active.get(), sink_coef.get(), s0,
                                                bad.get());
    require(read_scalar(bad.get(), s) == 0, "a seed is not an existing node");
    ppr_init<<<ceil_div(static_cast<uint64_t>(n) * kp, 256), 256, 0, s>>>(y0.get(), g->degc.get(),
                                                                          n, kp, x0);
    NKG_CUDA(cudaGetLastError());

    PprArgs a{};
    a.row_ptr = g->row_ptr.get();
    a.col = g->col.get();
    a.degc = g->degc.get();
    a.chunk_begin = g->fw.chunk_begin.get();
    a.chunk_row = chunk_row.get();
    a.unit_start = unit_start.get();
    a.seed = seed.get();
    a.chunk_val = chunk_val.get();
    a.active = active.get();
    a.sink_coef = sink_coef.get();
    a.cta_res = cta_res.get();
    a.cta_sink = cta_sink.get();
    a.col_res = col_res.get();
    a.col_iter = col_iter.get();
    a.st = st.get();
    a.damp = p.damp;
    a.tol = p.tol;
    a.max_iterations = p.max_iterations;
    a.n = n;
    a.n_long = g->fw.n_long;
    a.n_chunks = g->fw.n_chunks;
    a.units = units;
    a.kp = kp;
    a.sweep_ctas = sweep_ctas;
    a.l2 = p.norm == NKG_NORM_L2;
    a.distribute = p.distribute_sinks ? 1 : 0;

    uint64_t launches = 4;
    PprState h{};
    for (uint64_t it = 0;; it += 8) {
        for (int i = 0; i < 8; ++i) {
            a.y_in = ((it + i) & 1) ? y1.get() : y0.get();
            a.y_out = ((it + i) & 1) ? y0.get() : y1.get();
            ppr_sweep<CPL><<<sweep_ctas, kPprThreads, smem_sweep, s>>>(a);
            ppr_fixup<CPL><<<fix_ctas, kPprThreads, smem_sweep, s>>>(a, fix_res.get(), fix_sink.get());
        }
        launches += 16;
        NKG_CUDA(cudaGetLastError());
        h = read_scalar(st.get(), s);
        if (h.all_done)
            break;
        check_cancel(g, "personalised PageRank run cancelled");
    }
    NKG_CUDA(cudaEventRecord(g->ev1, s));
    const float *yfin = (h.iteration & 1) ? y1.get() : y0.get();

    // Normalisation per column (PageRank.cpp:75-92), output in the caller's ids.
    const uint32_t cs_ctas = std::min<uint32_t>(sms * 2, std::max<uint32_t>((n + kPprWarps - 1) / kPprWarps, 1));
    DeviceArray<double> part_sum(static_cast<size_t>(cs_ctas) * kp), part_sink(static_cast<size_t>(cs_ctas) * kp);
    ppr_colsum<CPL><<<cs_ctas, kPprThreads, smem_sweep, s>>>(yfin, g->degc.get(), n, kp,
                                                             part_sum.get(), part_sink.get());
    std::vector<double> hs(static_cast<size_t>(cs_ctas) * kp), hk(static_cast<size_t>(cs_ctas) * kp);
    NKG_CUDA(cudaMemcpyAsync(hs.data(), part_sum.get(), hs.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaMemcpyAsync(hk.data(), part_sink.get(), hk.size() * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    std::vector<double> factor(kp, 1.0);
    for (uint32_t c = 0; c < kp; ++c) {
        double sum = 0.0, sk = 0.0;
        for (uint32_t i = 0; i < cs_ctas; ++i) {
            sum += hs[static_cast<size_t>(i) * kp + c];
            sk += hk[static_cast<size_t>(i) * kp + c];
        }
        factor[c] = p.normalized ? (1.0 / static_cast<double>(n)) * ((1 - p.damp) + (p.damp * sk))
                                 : sum;
        if (!(factor[c] != 0.0))
            factor[c] = 1.0;
    }
    DeviceArray<double> d_factor(kp);
    NKG_CUDA(cudaMemcpyAsync(d_factor.get(), factor.data(), kp * sizeof(double),
                             cudaMemcpyHostToDevice, s));
    DeviceArray<float> dev_out;
    float *d_out = out;
    if (!out_on_device) {
        dev_out.alloc(static_cast<size_t>(k) * g->z);
        d_out = dev_out.get();
    }
    const size_t smem_out = 32 * (kp + 1) * sizeof(float);
    ppr_output<<<ceil_div(g->z, 32), 256, smem_out, s>>>(yfin, g->degc.get(), g->inv.get(), g->z,
                                                          n, k, kp, d_factor.get(), d_out);
    NKG_CUDA(cudaGetLastError());
    launches += 2;
    NKG_CUDA(cudaEventRecord(g->ev2, s));
    if (!out_on_device)
        NKG_CUDA(cudaMemcpyAsync(out, d_out, static_cast<size_t>(k) * g->z * sizeof(float),
                                 cudaMemcpyDeviceToHost, s));
    std::vector<unsigned long long> hit(kp);
    std::vector<double> hres(kp);
    NKG_CUDA(cudaMemcpyAsync(hit.data(), col_iter.get(), kp * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaMemcpyAsync(hres.data(), col_res.get(), kp * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    if (iters_out)
        for (uint32_t j = 0; j < k; ++j)
            iters_out[j] = hit[j];
    if (stats) {
        clear_stats(stats);
        float ms = 0.f;
        NKG_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev2));
        stats->ms_total = ms;
        NKG_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
        stats->ms_iterations = ms;
        stats->iterations = h.iteration;
        double worst = 0.0;
        for (uint32_t j = 0; j < k; ++j)
            worst = std::max(worst, hres[j]);
        stats->residual = worst;
        stats->kernel_launches = launches;
        stats->fp32_sweeps = h.iteration;
        // SpMM sweep, k columns: column ids, row offsets, degrees, and per
        // column the gathered, previous and new iterate.
        stats->bytes_per_sweep_fp32 = 4 * g->arcs + 4 * (g->n + 1) + 4 * g->n + 12ull * g->n * k;
        stats->bytes_per_sweep_fp64 = 0;
    }
}

} // namespace
} // namespace nkg

extern "C" int nkg_ppr_run(nkg_graph *g, const nkg_pr_params *p, uint32_t k, const uint32_t *seeds,
                           float *scores_out, int out_on_device, uint64_t *iterations_out,
                           nkg_stats *stats) {
    using namespace nkg;
    return guarded([&] {
        require(g != nullptr && p != nullptr && seeds != nullptr && scores_out != nullptr,
                "NULL argument");
        require(k >= 1 && k <= 256, "k must be in [1, 256]");
        require(!g->weighted, "batched personalised PageRank takes unweighted graphs");
        require(p->norm == NKG_NORM_L1 || p->norm == NKG_NORM_L2, "norm must be L1 or L2");
        require(std::isfinite(p->damp) && !std::isnan(p->tol), "damp/tol must be numbers");
        for (uint32_t j = 0; j < k; ++j)
            require(seeds[j] < g->z, "seed id out of range");
        DeviceGuard guard(g->device);
        RunScope scope(g);
        // CPL columns per lane (float4 loads): 128 or 256 columns per sweep.
        if (k <= 128)
            run_ppr<4>(g, *p, k, seeds, scores_out, out_on_device != 0, iterations_out, stats);
        else
            run_ppr<8>(g, *p, k, seeds, scores_out, out_on_device != 0, iterations_out, stats);
    });
}
