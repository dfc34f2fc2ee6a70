// Row partition of the PageRank sweep over several GPUs (nkg_part_*).
//
// The 1-D partition of the destination rows of the in-CSR: every GPU holds a
// contiguous range of rows (a "slice", cut so that the slices carry about the
// same number of arcs) and computes that range of the next iterate from the
// whole previous one. Between sweeps the slices are all-gathered into the
// shared iterate and the residual and sink-mass partial sums are all-reduced
// (the caller's collectives, e.g. NCCL through torch.distributed); the
// stopping test and the sink term are then the same on every GPU.
//
// The shared iterate is in gather form (x / deg, x for sinks), laid out by
// slices: slice q occupies [q * stride, q * stride + rows_q) for a common
// stride, so that an all-gather of equal-sized blocks assembles it, and one
// extra zero entry at its end is the target of padding slots. The caller
// numbers the columns of its slice in that layout. A slice keeps its own
// sliced (SELL-32) layout with its rows relabelled by in-degree; the sweep and
// fix-up are the single-GPU kernels of sweep.cuh with the PART flag, which
// maps each relabelled row back to its slice position for the degree, the
// previous value and the output. Every row sum runs in the arc order of the
// slice's CSR, the reference's order (PageRank.cpp:56-66).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "graph.hpp"
#include "host.hpp"

struct nkg_part {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t vec_len = 0;  // entries of the shared iterate (the last one the zero)
    uint32_t row_base = 0, rows = 0, pad = 0;
    uint64_t arcs = 0;
    bool weighted = false;
    nkg::DeviceArray<uint32_t> row_map;  // relabelled row -> slice row
    nkg::DeviceArray<uint32_t> degc;     // out-degree counts, slice order
    nkg::DeviceArray<double> degw;       // weighted out-degrees, slice order (weighted)
    nkg::SellLayout fw;
    nkg::DeviceArray<uint32_t> unit_start;
    uint32_t units = 0;
    unsigned sweep_ctas = 0, fix_ctas = 0;
    // unit_part: the residual and sink partials of each work unit (2 x units)
    nkg::DeviceArray<double> chunk_val, unit_part, fix_res, fix_sink, part;
    nkg::DeviceArray<nkg::RunParams> rp;
    nkg::DeviceArray<nkg::IterState> st;
    nkg::PinnedHost<nkg::IterState> st_host;
    nkg::PinnedHost<double> scal;
    unsigned long long iteration = 0;
    bool begun = false;
};

namespace nkg {
namespace {

constexpr int kPartThreads = 512;
constexpr int kPartUnroll = 8;
constexpr int kRedBlocks = 256;

__global__ void part_rowlen(const uint64_t *__restrict__ ptr, uint32_t rows,
                            uint32_t *__restrict__ len_key, uint32_t *__restrict__ ids) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows)
        return;
    // Descending length as an ascending key; the stable sort keeps ids in order.
    len_key[r] = ~static_cast<uint32_t>(ptr[r + 1] - ptr[r]);
    ids[r] = r;
}

__global__ void part_sorted_len(const uint32_t *__restrict__ key, uint32_t rows,
                                uint32_t *__restrict__ len) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < rows)
        len[r] = ~key[r];
}

// Copy every slice row to its relabelled place, one warp per row.
__global__ void part_copy_rows(const uint64_t *__restrict__ ptr, const uint32_t *__restrict__ col,
                               const double *__restrict__ w, const uint32_t *__restrict__ row_map,
                               const uint32_t *__restrict__ new_ptr, uint32_t rows,
                               uint32_t *__restrict__ new_col, double *__restrict__ new_w) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint32_t r = warp; r < rows; r += nwarps) {
        const uint32_t o = row_map[r];
        const uint64_t b = ptr[o], e = ptr[o + 1];
        const uint32_t nb = new_ptr[r];
        for (uint64_t k = b + lane; k < e; k += 32) {
            new_col[nb + (k - b)] = col[k];
            if (w)
                new_w[nb + (k - b)] = w[k];
        }
    }
}

// x = 1/n in gather form for the slice rows (PageRank.cpp:26).
__global__ void part_init(const uint32_t *__restrict__ degc, const double *__restrict__ degw,
                          uint32_t rows, double x0, double *__restrict__ y) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows)
        return;
    const uint32_t dc = degc[r];
    y[r] = dc == 0 ? x0 : x0 / (degw ? degw[r] : static_cast<double>(dc));
}

// Per-block partial sums of x, x over sinks, and the max of x over the slice
// (fixed tree per block), for PageRank.cpp:75-102.
__global__ void __launch_bounds__(256) part_sums(const double *__restrict__ y,
                                                 const uint32_t *__restrict__ degc,
                                                 const double *__restrict__ degw, uint32_t rows,
                                                 double *__restrict__ part) {
    __shared__ double s_red[32];
    double sum = 0.0, ss = 0.0, mx = -1.0 / 0.0;
    for (uint32_t r = blockIdx.x * 256 + threadIdx.x; r < rows; r += gridDim.x * 256) {
        const uint32_t dc = degc[r];
        const double x = dc ? __dmul_rn(y[r], degw ? degw[r] : static_cast<double>(dc)) : y[r];
        sum += x;
        if (!dc)
            ss += x;
        mx = fmax(mx, x);
    }
    sum = block_sum<256>(sum, s_red);
    ss = block_sum<256>(ss, s_red);
    mx = block_max<256>(mx, s_red);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = sum;
        part[gridDim.x + blockIdx.x] = ss;
        part[2 * gridDim.x + blockIdx.x] = mx;
    }
}

// The block partials in block order (one block).
__global__ void __launch_bounds__(256) part_sums_close(const double *__restrict__ part,
                                                       uint32_t blocks, double *__restrict__ out) {
    __shared__ double s_red[32];
    double sum = 0.0, ss = 0.0, mx = -1.0 / 0.0;
    for (uint32_t i = threadIdx.x; i < blocks; i += 256) {
        sum += part[i];
        ss += part[blocks + i];
        mx = fmax(mx, part[2 * blocks + i]);
    }
    sum = block_sum<256>(sum, s_red);
    ss = block_sum<256>(ss, s_red);
    mx = block_max<256>(mx, s_red);
    if (threadIdx.x == 0) {
        out[0] = sum;
        out[1] = ss;
        out[2] = mx;
    }
}

__global__ void part_scale(const double *__restrict__ y, const uint32_t *__restrict__ degc,
                           const double *__restrict__ degw, uint32_t rows, double factor,
                           double *__restrict__ out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows)
        return;
    const uint32_t dc = degc[r];
    const double x = dc ? __dmul_rn(y[r], degw ? degw[r] : static_cast<double>(dc)) : y[r];
    out[r] = x / factor;
}

cudaStream_t stream_of(const nkg_part *p, void *stream) {
    return stream ? static_cast<cudaStream_t>(stream) : p->stream;
}

nkg_part *create_part(uint64_t vec_len, uint64_t row_base, uint64_t rows, uint64_t arcs,
                      const uint64_t *row_ptr, const uint32_t *col, const double *w,
                      const uint32_t *out_deg, const double *out_wdeg, int device) {
    require(vec_len >= 2 && vec_len <= 0xffffffffull,
            "vec_len must be in [2, 2^32) (the shared iterate and its zero entry)");
    require(rows >= 1 && row_base + rows <= vec_len - 1, "rows must lie inside the shared iterate");
    require(row_ptr != nullptr && out_deg != nullptr, "row_ptr / out_deg is NULL");
    require(arcs == 0 || col != nullptr, "col is NULL");
    require(arcs < 0xffffffffull, "a slice holds fewer than 2^32 arcs");
    require(row_ptr[0] == 0 && row_ptr[rows] == arcs,
            "row_ptr[0] must be 0 and row_ptr[rows] = arcs");
    const uint32_t pad = static_cast<uint32_t>(vec_len - 1);
    for (uint64_t r = 0; r < rows; ++r)
        require(row_ptr[r + 1] >= row_ptr[r], "row_ptr must be non-decreasing");
    for (uint64_t e = 0; e < arcs; ++e)
        require(col[e] < pad, "a column lies outside the shared iterate");
    if (w) {
        require(out_wdeg != nullptr, "a weighted slice needs out_wdeg");
        for (uint64_t r = 0; r < rows; ++r)
            require(out_deg[r] == 0 || out_wdeg[r] > 0.0,
                    "weighted degree must be positive where the out-degree is");
    }
    int dev = device;
    if (dev < 0)
        NKG_CUDA(cudaGetDevice(&dev));
    DeviceGuard guard(dev);
    auto p = std::make_unique<nkg_part>();
    p->device = dev;
    p->vec_len = vec_len;
    p->row_base = static_cast<uint32_t>(row_base);
    p->rows = static_cast<uint32_t>(rows);
    p->pad = pad;
    p->arcs = arcs;
    p->weighted = w != nullptr;
    p->stream = stream_acquire(dev);
    cudaStream_t s = p->stream;
    const unsigned sms = num_sms(dev);
    const uint32_t n = p->rows;

    DeviceArray<uint64_t> d_ptr(rows + 1);
    DeviceArray<uint32_t> d_col(std::max<uint64_t>(arcs, 1));
    DeviceArray<double> d_w;
    NKG_CUDA(cudaMemcpyAsync(d_ptr.get(), row_ptr, (rows + 1) * sizeof(uint64_t),
                             cudaMemcpyHostToDevice, s));
    if (arcs)
        NKG_CUDA(cudaMemcpyAsync(d_col.get(), col, arcs * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                 s));
    if (w) {
        d_w.alloc(std::max<uint64_t>(arcs, 1));
        if (arcs)
            NKG_CUDA(cudaMemcpyAsync(d_w.get(), w, arcs * sizeof(double), cudaMemcpyHostToDevice,
                                     s));
        p->degw.alloc(n);
        NKG_CUDA(cudaMemcpyAsync(p->degw.get(), out_wdeg, n * sizeof(double),
                                 cudaMemcpyHostToDevice, s));
    }
    p->degc.alloc(n);
    NKG_CUDA(cudaMemcpyAsync(p->degc.get(), out_deg, n * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             s));

    // Relabel the slice rows by in-degree, descending (stable by slice row).
    DeviceArray<uint32_t> key(n), key_s(n), ids(n), len(n), new_ptr(n + 1, 4);
    p->row_map.alloc(n);
    part_rowlen<<<ceil_div(n, 256), 256, 0, s>>>(d_ptr.get(), n, key.get(), ids.get());
    size_t tb = 0;
    NKG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.get(), key_s.get(), ids.get(),
                                             p->row_map.get(), static_cast<int64_t>(n), 0, 32, s));
    DeviceArray<unsigned char> tmp(std::max<size_t>(tb, 1));
    NKG_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, key.get(), key_s.get(), ids.get(),
                                             p->row_map.get(), static_cast<int64_t>(n), 0, 32, s));
    part_sorted_len<<<ceil_div(n, 256), 256, 0, s>>>(key_s.get(), n, len.get());
    NKG_CUDA(cudaMemsetAsync(new_ptr.get(), 0, sizeof(uint32_t), s));
    tb = 0;
    NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, len.get(), new_ptr.get() + 1,
                                           static_cast<int64_t>(n), s));
    tmp.alloc(std::max<size_t>(tb, 1));
    NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb, len.get(), new_ptr.get() + 1,
                                           static_cast<int64_t>(n), s));
    DeviceArray<uint32_t> new_col(std::max<uint64_t>(arcs, 1), 4);
    DeviceArray<double> new_w;
    if (w)
        new_w.alloc(std::max<uint64_t>(arcs, 1), 4);
    part_copy_rows<<<sms * 16, 256, 0, s>>>(d_ptr.get(), d_col.get(), w ? d_w.get() : nullptr,
                                            p->row_map.get(), new_ptr.get(), n, new_col.get(),
                                            w ? new_w.get() : nullptr);
    NKG_CUDA(cudaGetLastError());
    build_sell(p->fw, n, new_ptr.get(), new_col.get(), w ? new_w.get() : nullptr, nullptr,
               len.get(), dev, s, pad);

    // Launch shape of the regular sweep (512 threads, 8 gathers in flight),
    // warps taking units from the state's counter as in the single-GPU run.
    auto kfn = sweep_kernel<double, false, kPartThreads, kPartUnroll, false, true, true>;
    NKG_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, 0));
    auto kfw = sweep_kernel<double, true, kPartThreads, kPartUnroll, false, true, true>;
    NKG_CUDA(cudaFuncSetAttribute(kfw, cudaFuncAttributePreferredSharedMemoryCarveout, 0));
    int occ = 0;
    NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, w ? kfw : kfn, kPartThreads, 0));
    require(occ >= 1, "sweep kernel does not fit on an SM");
    p->sweep_ctas = static_cast<unsigned>(std::max<uint64_t>(
        1, std::min<uint64_t>(static_cast<uint64_t>(occ) * sms,
                              (static_cast<uint64_t>(p->fw.slices) * 32 + kPartThreads - 1) /
                                  kPartThreads)));
    const uint64_t warps = static_cast<uint64_t>(p->sweep_ctas) * (kPartThreads / 32);
    p->units = static_cast<uint32_t>(
        std::max<uint64_t>(1, std::min<uint64_t>(warps * kQueueUnitsPerWarp,
                                                 std::max<uint32_t>(p->fw.slices, 1))));
    p->unit_start.alloc(static_cast<size_t>(p->units) + 1);
    sell_units(p->fw, p->units, p->unit_start.get(), s);
    p->fix_ctas = fix_ctas_with_units(
        fix_vlong_ctas(p->fw.n_vlong) +
            ceil_div(std::max<uint32_t>(p->fw.n_long - p->fw.n_vlong, 1), kFixThreads),
        p->units, kFixThreads);
    p->chunk_val.alloc(static_cast<size_t>(p->fw.s_chunk) * 32 + 1);
    p->unit_part.alloc(2 * static_cast<size_t>(p->units));
    p->fix_res.alloc(p->fix_ctas);
    p->fix_sink.alloc(p->fix_ctas);
    p->part.alloc(3 * kRedBlocks + 3);
    p->rp.alloc(1);
    p->st.alloc(1);
    p->st_host.alloc(1);
    p->scal.alloc(4);
    NKG_CUDA(cudaStreamSynchronize(s));
    return p.release();
}

SweepArgs<double> part_args(const nkg_part *p, const double *y_in, double *y_out) {
    SweepArgs<double> a{};
    a.col_sell = p->fw.col_sell.get();
    a.w_sell = p->fw.w_sell64.get();
    a.slice_off = p->fw.slice_off.get();
    a.unit_start = p->unit_start.get();
    a.chunk_begin = p->fw.chunk_begin.get();
    a.degc = p->degc.get();
    a.degw = p->degw.get();
    a.tele = nullptr;
    a.y_in = y_in;
    a.y_out = y_out;
    a.chunk_val = p->chunk_val.get();
    a.unit_res = p->unit_part.get();
    a.unit_sink = p->unit_part.get() + p->units;
    a.fix_res = p->fix_res.get();
    a.fix_sink = p->fix_sink.get();
    a.rp = p->rp.get();
    a.st = p->st.get();
    a.n = p->rows;
    a.n_long = p->fw.n_long;
    a.n_vlong = p->fw.n_vlong;
    a.s_chunk = p->fw.s_chunk;
    a.units = p->units;
    a.sweep_ctas = p->sweep_ctas;
    a.row_map = p->row_map.get();
    a.row_base = p->row_base;
    a.pad = p->pad;
    return a;
}

} // namespace
} // namespace nkg

extern "C" {

int nkg_part_create(nkg_part **out, uint64_t vec_len, uint64_t row_base, uint64_t rows,
                    uint64_t arcs, const uint64_t *row_ptr, const uint32_t *col, const double *w,
                    const uint32_t *out_deg, const double *out_wdeg, int device) {
    using namespace nkg;
    return guarded([&] {
        require(out != nullptr, "out is NULL");
        *out = nullptr;
        *out = create_part(vec_len, row_base, rows, arcs, row_ptr, col, w, out_deg, out_wdeg,
                           device);
    });
}

void nkg_part_destroy(nkg_part *p) {
    if (!p)
        return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    cudaStreamSynchronize(p->stream);
    cudaStream_t s = p->stream;
    const int dev = p->device;
    delete p;
    nkg::stream_release(dev, s);
    if (prev >= 0)
        cudaSetDevice(prev);
}

int nkg_part_begin(nkg_part *p, const nkg_pr_params *prm, uint64_t n_global, double *d_y_out,
                   void *stream) {
    using namespace nkg;
    return guarded([&] {
        require(p != nullptr && prm != nullptr && d_y_out != nullptr, "NULL argument");
        require(n_global >= 1, "n_global must be at least 1");
        require(prm->precision == NKG_PREC_FP64, "the partitioned sweep computes in FP64");
        require(prm->norm == NKG_NORM_L1 || prm->norm == NKG_NORM_L2, "norm must be L1 or L2");
        require(std::isfinite(prm->damp), "damp must be finite");
        DeviceGuard guard(p->device);
        cudaStream_t s = stream_of(p, stream);
        RunParams h{};
        h.damp = prm->damp;
        h.tele_uniform = (1.0 - prm->damp) / static_cast<double>(n_global);
        h.one_minus_damp = 1.0 - prm->damp;
        h.inv_n = 1.0 / static_cast<double>(n_global);
        h.distribute = prm->distribute_sinks ? 1 : 0;
        h.personal = 0;
        h.l2 = prm->norm == NKG_NORM_L2 ? 1 : 0;
        h.tol = -1.0;  // the caller applies the stopping test to the reduced sums
        h.max_iterations = ~0ull;
        NKG_CUDA(cudaMemcpyAsync(p->rp.get(), &h, sizeof(RunParams), cudaMemcpyHostToDevice, s));
        part_init<<<ceil_div(p->rows, 256), 256, 0, s>>>(
            p->degc.get(), p->weighted ? p->degw.get() : nullptr, p->rows,
            1.0 / static_cast<double>(n_global), d_y_out);
        NKG_CUDA(cudaGetLastError());
        NKG_CUDA(cudaStreamSynchronize(s));
        p->iteration = 0;
        p->begun = true;
    });
}

int nkg_part_sweep(nkg_part *p, const double *d_y_in, double sink_coef, double *d_y_out,
                   double *residual_sum_out, double *sink_sum_out, void *stream) {
    using namespace nkg;
    return guarded([&] {
        require(p != nullptr && d_y_in != nullptr && d_y_out != nullptr, "NULL argument");
        require(p->begun, "nkg_part_begin must come first");
        DeviceGuard guard(p->device);
        cudaStream_t s = stream_of(p, stream);
        IterState *h = p->st_host.get();
        std::memset(h, 0, sizeof(IterState));
        h->iteration = p->iteration;
        h->sink_coef = sink_coef;
        NKG_CUDA(cudaMemcpyAsync(p->st.get(), h, sizeof(IterState), cudaMemcpyHostToDevice, s));
        const SweepArgs<double> a = part_args(p, d_y_in, d_y_out);
        if (p->weighted) {
            sweep_kernel<double, true, kPartThreads, kPartUnroll, false, true, true>
                <<<p->sweep_ctas, kPartThreads, 0, s>>>(a);
            fixup_kernel<double, true, true><<<p->fix_ctas, kFixThreads, 0, s>>>(a);
        } else {
            sweep_kernel<double, false, kPartThreads, kPartUnroll, false, true, true>
                <<<p->sweep_ctas, kPartThreads, 0, s>>>(a);
            fixup_kernel<double, false, true><<<p->fix_ctas, kFixThreads, 0, s>>>(a);
        }
        NKG_CUDA(cudaGetLastError());
        NKG_CUDA(cudaMemcpyAsync(h, p->st.get(), sizeof(IterState), cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        p->iteration = h->iteration;
        if (residual_sum_out)
            *residual_sum_out = h->residual_sum;
        if (sink_sum_out)
            *sink_sum_out = h->sink_mass;
    });
}

int nkg_part_sums(nkg_part *p, const double *d_y, double *sum_out, double *sink_sum_out,
                  double *max_out, void *stream) {
    using namespace nkg;
    return guarded([&] {
        require(p != nullptr && d_y != nullptr, "NULL argument");
        DeviceGuard guard(p->device);
        cudaStream_t s = stream_of(p, stream);
        const unsigned blocks = std::min<unsigned>(kRedBlocks, ceil_div(p->rows, 256));
        const double *degw = p->weighted ? p->degw.get() : nullptr;
        part_sums<<<blocks, 256, 0, s>>>(d_y, p->degc.get(), degw, p->rows, p->part.get());
        part_sums_close<<<1, 256, 0, s>>>(p->part.get(), blocks, p->part.get() + 3 * kRedBlocks);
        NKG_CUDA(cudaGetLastError());
        double *h = p->scal.get();
        NKG_CUDA(cudaMemcpyAsync(h, p->part.get() + 3 * kRedBlocks, 3 * sizeof(double),
                                 cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        if (sum_out)
            *sum_out = h[0];
        if (sink_sum_out)
            *sink_sum_out = h[1];
        if (max_out)
            *max_out = h[2];
    });
}

int nkg_part_scores(nkg_part *p, const double *d_y, double factor, double *d_out, void *stream) {
    using namespace nkg;
    return guarded([&] {
        require(p != nullptr && d_y != nullptr && d_out != nullptr, "NULL argument");
        require(std::isfinite(factor) && factor != 0.0, "factor must be finite and non-zero");
        DeviceGuard guard(p->device);
        cudaStream_t s = stream_of(p, stream);
        part_scale<<<ceil_div(p->rows, 256), 256, 0, s>>>(
            d_y, p->degc.get(), p->weighted ? p->degw.get() : nullptr, p->rows, factor, d_out);
        NKG_CUDA(cudaGetLastError());
        NKG_CUDA(cudaStreamSynchronize(s));
    });
}

} // extern "C"
