// Allocation-free PageRank entry point (nkg_pagerank_csr_noalloc).
//
// Some callers cannot allocate device memory when they call in: frameworks
// whose caching allocator already owns the device memory (a cudaMalloc behind
// its back can fail or fragment it), services whose memory budget is fixed at
// start-up, and latency-critical loops where cudaMalloc/cudaFree would
// synchronise the device. For them this file runs the FP64 power iteration
// on buffers the caller passes in, with all working storage in one
// file-scope __device__ array of kNoAllocScratchBytes. That array is part of
// the library's device image: every GPU that loads the library holds it until
// the process exits.
//
// The kernels are a plain warp-per-row variant of the sweep (no relabelling,
// no sliced layout), so graphs are limited to kNoAllocMaxNodes nodes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "common.cuh"

namespace nkg {
namespace {

// Working storage: two iterates (n+1 doubles each), the out-degree counts
// (n uint32) and a fixed block of reduction partials and state, each region
// rounded up to 256 bytes.
constexpr uint64_t kNoAllocMaxNodes = 1u << 19;   // 524,288
constexpr uint64_t kPartials = 4096;               // per-CTA partial sums

struct NaState {
    unsigned long long iteration;
    double residual;
    double sink_coef;
    double sum, sink_sum, maxv;
    int done;
    unsigned int ticket;
};

struct NaLayout {
    double *y0, *y1;
    uint32_t *deg;
    double *part_res, *part_sink, *part_max;
    NaState *st;
};

__host__ __device__ constexpr uint64_t round256(uint64_t b) { return (b + 255) / 256 * 256; }

// Bytes na_layout() uses for an n-node graph.
constexpr uint64_t na_bytes(uint64_t n) {
    return 2 * round256((n + 1) * sizeof(double)) + round256(n * sizeof(uint32_t)) +
           3 * round256(kPartials * sizeof(double)) + round256(sizeof(NaState));
}

// 12.1 MB: the maximum graph's working storage.
constexpr uint64_t kNoAllocScratchBytes = na_bytes(kNoAllocMaxNodes);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

__host__ __device__ inline NaLayout na_layout(unsigned char *base, uint64_t n) {
    NaLayout L;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char *p = base + off;
        off += round256(bytes);
        return p;
    };
    L.y0 = reinterpret_cast<double *>(take((n + 1) * sizeof(double)));
    L.y1 = reinterpret_cast<double *>(take((n + 1) * sizeof(double)));
    L.deg = reinterpret_cast<uint32_t *>(take(n * sizeof(uint32_t)));
    L.part_res = reinterpret_cast<double *>(take(kPartials * sizeof(double)));
    L.part_sink = reinterpret_cast<double *>(take(kPartials * sizeof(double)));
    L.part_max = reinterpret_cast<double *>(take(kPartials * sizeof(double)));
    L.st = reinterpret_cast<NaState *>(take(sizeof(NaState)));
    return L;
}

constexpr int kNaThreads = 256;

struct NaParams {
    double damp, tele, tol;
    unsigned long long max_iterations;
    int l2, distribute;
    uint32_t n;
};

// Zero the counters that every call must start from, count out-degrees.
__global__ void na_init(NaLayout L, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        L.deg[i] = 0;
    if (i == 0) {
        NaState s{};
        *L.st = s;
    }
}

__global__ void na_count(NaLayout L, const uint32_t *__restrict__ col, uint64_t arcs,
                         uint32_t n, int *err) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < arcs;
         e += stride) {
        const uint32_t v = col[e];
        if (v >= n) {
            atomicExch(err, 1);
            continue;
        }
        atomicAdd(L.deg + v, 1u);
    }
}

// The caller's in-CSR offsets, checked before any sweep walks them (the
// checks of the regular path's graph upload): row_ptr[0] = 0, non-decreasing,
// row_ptr[n] = arcs. A bad offset sets *err to 2, so no sweep is launched.
__global__ void na_check_rows(const uint64_t *__restrict__ row_ptr, uint64_t arcs, uint32_t n,
                              int *err) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        const uint64_t a = row_ptr[i], b = row_ptr[i + 1];
        if (b < a || b > arcs || (i == 0 && a != 0) || (i + 1 == n && b != arcs))
            atomicExch(err, 2);
    }
}

__global__ void na_start(NaLayout L, uint32_t n, double x0, double sink_coef0) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) {
        const uint32_t d = L.deg[r];
        L.y0[r] = d ? x0 / static_cast<double>(d) : x0;
    }
    if (r == 0) {
        L.y0[n] = 0.0;
        L.y1[n] = 0.0;
        L.st->sink_coef = sink_coef0;
    }
}

// One Jacobi sweep (PageRank.cpp:56-66): a warp per row, lanes striding over
// the row's arcs, a fixed warp tree for the row sum; the last CTA closes the
// iteration (PageRank.cpp:41-51,68-70).
__global__ void __launch_bounds__(kNaThreads)
    na_sweep(NaLayout L, NaParams p, const uint64_t *__restrict__ row_ptr,
             const uint32_t *__restrict__ col, int in_buf) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    if (*(volatile int *)&L.st->done)
        return;
    const double *yi = in_buf ? L.y1 : L.y0;
    double *yo = in_buf ? L.y0 : L.y1;
    const double sink_coef = L.st->sink_coef;
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * kNaThreads + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * kNaThreads) >> 5;
    double res = 0.0, sink = 0.0;
    for (uint32_t r = warp; r < p.n; r += nwarps) {
        double acc = 0.0;
        for (uint64_t e = row_ptr[r] + lane; e < row_ptr[r + 1]; e += 32)
            acc += yi[col[e]];
        acc = warp_sum(acc);
        if (lane == 0) {
            if (p.distribute)
                acc = __dadd_rn(acc, sink_coef);
            double x = __dmul_rn(acc, p.damp);
            x = __dadd_rn(x, p.tele);
            const uint32_t d = L.deg[r];
            const double xo = d ? __dmul_rn(yi[r], static_cast<double>(d)) : yi[r];
            const double diff = xo - x;
            res += p.l2 ? __dmul_rn(diff, diff) : fabs(diff);
            if (d) {
                yo[r] = x / static_cast<double>(d);
            } else {
                yo[r] = x;
                sink += x;
            }
        }
    }
    res = block_sum<kNaThreads>(res, s_red);
    sink = block_sum<kNaThreads>(sink, s_red);
    if (threadIdx.x == 0) {
        L.part_res[blockIdx.x] = res;
        L.part_sink[blockIdx.x] = sink;
        __threadfence();
        s_last = atomicAdd(&L.st->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    double r = 0.0, s = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kNaThreads) {
        r += ((volatile double *)L.part_res)[i];
        s += ((volatile double *)L.part_sink)[i];
    }
    r = block_sum<kNaThreads>(r, s_red);
    s = block_sum<kNaThreads>(s, s_red);
    if (threadIdx.x == 0) {
        NaState *st = L.st;
        const unsigned long long it = st->iteration + 1;
        const double norm = p.l2 ? sqrt(r) : r;
        st->iteration = it;
        st->residual = norm;
        st->sink_coef = p.distribute ? s / static_cast<double>(p.n) : 0.0;
        st->ticket = 0;
        __threadfence();
        st->done = (it >= p.max_iterations || norm <= p.tol) ? 1 : 0;
    }
}

// Final sums (PageRank.cpp:75-92,95-102) and the scaled scores.
__global__ void __launch_bounds__(kNaThreads) na_final(NaLayout L, uint32_t n, int fin_buf) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    const double *y = fin_buf ? L.y1 : L.y0;
    double sum = 0.0, ss = 0.0, mx = -1.0 / 0.0;
    for (uint32_t r = blockIdx.x * kNaThreads + threadIdx.x; r < n; r += gridDim.x * kNaThreads) {
        const uint32_t d = L.deg[r];
        const double x = d ? __dmul_rn(y[r], static_cast<double>(d)) : y[r];
        sum += x;
        if (!d)
            ss += x;
        mx = fmax(mx, x);
    }
    sum = block_sum<kNaThreads>(sum, s_red);
    ss = block_sum<kNaThreads>(ss, s_red);
    mx = block_max<kNaThreads>(mx, s_red);
    if (threadIdx.x == 0) {
        L.part_res[blockIdx.x] = sum;
        L.part_sink[blockIdx.x] = ss;
        L.part_max[blockIdx.x] = mx;
        __threadfence();
        s_last = atomicAdd(&L.st->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    sum = 0.0;
    ss = 0.0;
    mx = -1.0 / 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kNaThreads) {
        sum += ((volatile double *)L.part_res)[i];
        ss += ((volatile double *)L.part_sink)[i];
        mx = fmax(mx, ((volatile double *)L.part_max)[i]);
    }
    sum = block_sum<kNaThreads>(sum, s_red);
    ss = block_sum<kNaThreads>(ss, s_red);
    mx = block_max<kNaThreads>(mx, s_red);
    if (threadIdx.x == 0) {
        L.st->sum = sum;
        L.st->sink_sum = ss;
        L.st->maxv = mx;
        L.st->ticket = 0;
    }
}

__global__ void na_scale(NaLayout L, uint32_t n, int fin_buf, int normalized, double damp,
                         double *__restrict__ out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n)
        return;
    const double *y = fin_buf ? L.y1 : L.y0;
    const double factor = normalized
                              ? (1.0 / static_cast<double>(n)) * ((1 - damp) + (damp * L.st->sink_sum))
                              : L.st->sum;
    const uint32_t d = L.deg[r];
    const double x = d ? __dmul_rn(y[r], static_cast<double>(d)) : y[r];
    out[r] = x / factor;
}

// Scratch address per device, looked up once with that device current (the
// first call on the device). A cudaDeviceReset of the device gives the
// module a new context, so the cached address is not valid after one.
std::mutex g_na_mutex;
unsigned char *g_na_addr[64] = {};

unsigned char *scratch_address(int dev) {
    require(dev >= 0 && dev < 64, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_addr[dev]) {
        void *ptr = nullptr;
        NKG_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        g_na_addr[dev] = static_cast<unsigned char *>(ptr);
    }
    return g_na_addr[dev];
}

} // namespace
} // namespace nkg

extern "C" int nkg_pagerank_csr_noalloc(uint64_t n, uint64_t arcs, const uint64_t *d_in_row_ptr,
                                        const uint32_t *d_in_col, const nkg_pr_params *p,
                                        double *d_scores_out, uint64_t *iterations_out,
                                        void *stream) {
    using namespace nkg;
    try {
        require(p != nullptr && d_in_row_ptr != nullptr && d_scores_out != nullptr,
                "NULL argument");
        require(arcs == 0 || d_in_col != nullptr, "d_in_col is NULL");
        require(n >= 1, "graph must have at least one node");
        require(n <= kNoAllocMaxNodes,
                "nkg_pagerank_csr_noalloc handles at most 524288 nodes (its scratch is fixed)");
        require(p->precision == NKG_PREC_FP64, "nkg_pagerank_csr_noalloc computes in FP64 only");
        require(p->norm == NKG_NORM_L1 || p->norm == NKG_NORM_L2, "norm must be L1 or L2");
        require(std::isfinite(p->damp) && !std::isnan(p->tol), "damp/tol must be numbers");
        int dev = 0;
        NKG_CUDA(cudaGetDevice(&dev));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const NaLayout L = na_layout(scratch_address(dev), n);
        const uint32_t nn = static_cast<uint32_t>(n);
        const unsigned blocks_n = ceil_div(n, kNaThreads);
        na_init<<<blocks_n, kNaThreads, 0, s>>>(L, nn);
        // The error word lives in the partials block (zeroed here).
        int *err = reinterpret_cast<int *>(L.part_max);
        NKG_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
        na_check_rows<<<std::min<unsigned>(blocks_n, 1024), kNaThreads, 0, s>>>(d_in_row_ptr,
                                                                                 arcs, nn, err);
        if (arcs)
            na_count<<<256, kNaThreads, 0, s>>>(L, d_in_col, arcs, nn, err);
        NKG_CUDA(cudaGetLastError());
        int h_err = 0;
        NKG_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        require(h_err != 2, "d_in_row_ptr is not a valid CSR offset array (row_ptr[0] must be 0, "
                            "the offsets non-decreasing and row_ptr[n] = arcs)");
        require(h_err == 0, "d_in_col holds a node id >= n");
        const double x0 = 1.0 / static_cast<double>(n);
        NaParams np{};
        np.damp = p->damp;
        np.tele = (1.0 - p->damp) / static_cast<double>(n);
        np.tol = p->tol;
        np.max_iterations = p->max_iterations;
        np.l2 = p->norm == NKG_NORM_L2;
        np.distribute = p->distribute_sinks != 0;
        np.n = nn;
        // Initial sink mass: sinks * (1/n), spread over n (distributeSinks).
        // The count is read back once, so the start needs no extra kernel.
        na_start<<<blocks_n, kNaThreads, 0, s>>>(L, nn, x0, 0.0);
        NKG_CUDA(cudaGetLastError());
        if (np.distribute) {
            // sum of x0 over sinks = x0 * #sinks; #sinks from the degrees
            na_final<<<std::min<unsigned>(blocks_n, kPartials), kNaThreads, 0, s>>>(L, nn, 0);
            NaState h{};
            NKG_CUDA(cudaMemcpyAsync(&h, L.st, sizeof(NaState), cudaMemcpyDeviceToHost, s));
            NKG_CUDA(cudaStreamSynchronize(s));
            const double c0 = h.sink_sum / static_cast<double>(n);
            NKG_CUDA(cudaMemcpyAsync(&L.st->sink_coef, &c0, sizeof(double), cudaMemcpyHostToDevice,
                                     s));
        }
        const unsigned sweep_blocks =
            static_cast<unsigned>(std::min<uint64_t>(kPartials, (n * 32 + kNaThreads - 1) / kNaThreads));
        NaState h{};
        for (int chunk = 0;; ++chunk) {
            for (int i = 0; i < 8; ++i)
                na_sweep<<<sweep_blocks, kNaThreads, 0, s>>>(L, np, d_in_row_ptr, d_in_col,
                                                             static_cast<int>((chunk * 8 + i) & 1));
            NKG_CUDA(cudaGetLastError());
            NKG_CUDA(cudaMemcpyAsync(&h, L.st, sizeof(NaState), cudaMemcpyDeviceToHost, s));
            NKG_CUDA(cudaStreamSynchronize(s));
            if (h.done)
                break;
        }
        const int fin = static_cast<int>(h.iteration & 1ull);
        na_final<<<std::min<unsigned>(blocks_n, kPartials), kNaThreads, 0, s>>>(L, nn, fin);
        na_scale<<<blocks_n, kNaThreads, 0, s>>>(L, nn, fin, p->normalized ? 1 : 0, p->damp,
                                                 d_scores_out);
        NKG_CUDA(cudaGetLastError());
        NKG_CUDA(cudaStreamSynchronize(s));
        if (iterations_out)
            *iterations_out = h.iteration;
        return NKG_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return NKG_ERR_CUDA;
    }
}
