// Device-resident graph handle (the opaque nkg_graph of nkgpu.h).
#pragma once

#include <atomic>
#include <memory>

#include "common.cuh"
#include "sweep.cuh"

namespace nkg {

// Sweeps per captured CUDA graph (even, so every graph starts on buffer 0).
constexpr int kSweepsPerGraph = 8;
// Work units per resident warp of the sweep kernel.
constexpr uint32_t kUnitsPerWarp = 8;
// Work units per resident warp of the queued PageRank sweep. Measured on
// R-MAT scale 24 (FP64 sweep, B200): 4 / 8 / 12 / 16 / 24 / 32 / 64 units per
// warp ran 0.941 / 0.880 / 0.876 / 0.875 / 0.889 / 0.900 / 0.975 ms, against
// 0.956 ms for 8 static units per warp. Fewer units leave a longer tail;
// more units pay the ticket round trip and a cold start more often.
constexpr uint32_t kQueueUnitsPerWarp = 16;
// Cost of a slice in units of one slot step, besides its length (the
// epilogue of its 32 rows).
constexpr uint32_t kSliceOverhead = 3;

// Work buffers of the FP32 refinement solve, kept between runs.
struct RefineWork {
    DeviceArray<float> x, r, rhat, p, v, s, t, g;  // g: n+1 (gather form, g[n] = 0)
    DeviceArray<double> x64, part, fix_part;
    DeviceArray<double> unit_part;                  // queued product: 2 per unit
    DeviceArray<unsigned char> sc;                  // BiScalars
};

// Sliced layout (SELL-32 with chunked long rows, see sweep.cuh) of one
// adjacency: the in-adjacency for the forward sweeps, the out-adjacency for
// the adjoint.
struct SellLayout {
    uint32_t n_long = 0, n_vlong = 0, n_chunks = 0, s_chunk = 0, slices = 0;
    uint64_t slots = 0;
    DeviceArray<uint32_t> chunk_begin;  // n_long+1
    DeviceArray<uint32_t> slice_off;    // slices+1
    DeviceArray<uint64_t> slice_cost;   // slices, inclusive prefix of slice costs
    DeviceArray<uint32_t> col_sell;     // slots
    DeviceArray<double> w_sell64;       // slots (weighted)
};

// Build the sliced layout of a CSR whose n rows are sorted by length,
// descending; the weight of entry k is w[w_index[k]] (w[k] without an index,
// no weights when w is null). Padding slots hold pad_col (kNone: n, the zero
// entry of an iterate of n + 1).
void build_sell(SellLayout &L, uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                const double *w, const uint32_t *w_index, const uint32_t *rowlen, int device,
                cudaStream_t s, uint32_t pad_col = kNone);
// map[slot] = index[k] for the CSR entry k each slot of L holds (kNone for
// padding slots).
void build_slot_map(const SellLayout &L, uint32_t n, const uint32_t *row_ptr, const uint32_t *index,
                    uint32_t *map, int device, cudaStream_t s);
// Cost-balanced unit boundaries over the slices of L (units+1 entries).
void sell_units(const SellLayout &L, uint32_t units, uint32_t *unit_start, cudaStream_t s);
void convert_to_float(const double *in, float *out, uint64_t m, int device, cudaStream_t s);

struct AdjointState;
void destroy_adjoint(AdjointState *a);
struct AdjointDeleter {
    void operator()(AdjointState *a) const { destroy_adjoint(a); }
};

// Per-precision work buffers and the captured sweep graph.
template <typename T>
struct Plane {
    DeviceArray<T> y[2];         // ping-pong iterate in gather form (n+1, y[n] = 0)
    DeviceArray<T> chunk_val;    // per chunk slot
    DeviceArray<T> w_sell;       // slot weights in this precision (weighted)
    DeviceArray<T> degw;         // weighted degree in this precision (weighted)
    DeviceArray<T> tele;         // personalised teleport, relabelled
    DeviceArray<uint32_t> unit_start;
    uint32_t units = 0;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // [personal]
    unsigned sweep_ctas = 0;
    unsigned fix_ctas = 0;
    uint32_t hot = 0;            // ids in the shared-memory tier (0: none)
    // The tier kernel's own grid and work units; the fields above stay those
    // of the regular shape, which the FP32 product of the refinement solve
    // also uses.
    DeviceArray<uint32_t> hot_unit_start;
    uint32_t hot_units = 0;
    unsigned hot_ctas = 0;
    int hot_threads = 0;         // kHotThreads or kHotThreadsPair
    // Queued sweep (warps take units from a device counter): its units and
    // their residual / sink partials (2 x q_units). q_units 0: the static
    // assignment of unit_start (the shared-memory tier).
    DeviceArray<uint32_t> q_unit_start;
    DeviceArray<double> q_part;
    uint32_t q_units = 0;
    // The sweep's last CTA closes each iteration (no fix-up launch): graphs
    // with no split rows and at most kCloseInSweepUnits units.
    bool close_in_sweep = false;
};

} // namespace nkg

struct nkg_graph {
    nkg_graph() = default;
    nkg_graph(const nkg_graph &) = delete;
    nkg_graph &operator=(const nkg_graph &) = delete;
    ~nkg_graph();
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t z = 0, n = 0, arcs = 0, sinks = 0;
    bool weighted = false, directed = false;
    double ms_create = 0.0;
    int row_order = 0;  // relabelling used: 0 in-degree, 1 in-degree buckets

    nkg::DeviceArray<uint32_t> perm;     // new id -> original id (n)
    nkg::DeviceArray<uint32_t> inv;      // original id -> new id (z), kNone if absent
    nkg::DeviceArray<uint32_t> row_ptr;  // n+1, in-CSR in new ids
    nkg::DeviceArray<uint32_t> col;      // arcs
    nkg::DeviceArray<uint32_t> degc;     // out-degree count (n)
    nkg::DeviceArray<double> w64src;     // CSR arc weights (FP64, relabelled order)
    nkg::DeviceArray<double> degw64src;  // weighted degree (FP64)

    nkg::DeviceArray<uint64_t> row_src; // n: offset of new row r in the caller's in-CSR

    // Sliced layout of the sweep (the in-adjacency).
    nkg::SellLayout fw;
    int sweep_shape = 0;
    bool arc_sorted = false;
    bool w64src_stale = false;  // w64src predates nkg_graph_set_weights

    // Out-adjacency layout and buffers of the adjoint (built on first use).
    std::unique_ptr<nkg::AdjointState, nkg::AdjointDeleter> adj;

    nkg::Plane<double> p64;
    nkg::Plane<float> p32;
    nkg::RefineWork refine_work;

    nkg::DeviceArray<double> cta_res, cta_sink, fix_res, fix_sink;
    nkg::DeviceArray<double> out_buf;    // scores staging for host output (z)
    nkg::DeviceArray<double> red;        // scratch for finalisation reductions
    nkg::DeviceArray<unsigned int> red_ticket;
    nkg::DeviceArray<nkg::RunParams> rp;
    nkg::DeviceArray<nkg::IterState> st;
    nkg::PinnedHost<nkg::IterState> st_host;
    nkg::PinnedHost<double> scalars_host;

    nkg::DeviceArray<double> trace;      // residual of sweep i at [i] (kTraceCapacity)
    int hot_tier_kb = -1;                // nkg_graph_options.hot_tier_kb

    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    std::atomic<int> cancel{0};
    bool has_run = false;
};

namespace nkg {
// Cancellation (nkg_cancel): a request stays set until a run on the handle
// ends, so one issued just before a run starts stops that run. Every run
// holds a RunScope, which clears the request when the run ends (normally or
// by an error); the checks between chunks of sweeps only read it.
struct RunScope {
    nkg_graph *g;
    explicit RunScope(nkg_graph *h) : g(h) {}
    RunScope(const RunScope &) = delete;
    RunScope &operator=(const RunScope &) = delete;
    ~RunScope() { g->cancel.store(0); }
};
inline void check_cancel(const nkg_graph *g, const char *what) {
    if (g->cancel.load())
        throw Error(NKG_ERR_CANCELLED, what);
}

// A graph from an in-CSR already in device memory (nkgpu.cu): the shell on the
// options' device (its stream is the one to build on), then the regular upload
// steps from the device arrays (host copy of the existence mask, nullable).
std::unique_ptr<nkg_graph> device_graph_shell(const nkg_graph_options *opt, uint64_t z,
                                              bool weighted, int directed);
nkg_graph *device_graph_build(std::unique_ptr<nkg_graph> g, uint64_t arcs,
                              DeviceArray<uint64_t> &d_ptr, DeviceArray<uint32_t> &d_col,
                              DeviceArray<double> &d_w, DeviceArray<double> &d_wdeg,
                              DeviceArray<uint8_t> &d_ex, const uint8_t *exists_host,
                              const nkg_graph_options *opt);

// Most sweeps whose residual a run records for nkg_stats.residual_trace.
constexpr uint32_t kTraceCapacity = 65536;

// The out-adjacency layout of the adjoint (adjoint.cu), built on first use.
AdjointState &adjoint_ensure(nkg_graph *g);
// Read-only view of that layout for other kernels: rows are the nodes in
// out-degree order (tinv: relabelled id -> row), columns row numbers.
struct OutLayoutView {
    const SellLayout *tl;
    const uint32_t *tinv;
};
OutLayoutView adjoint_out_layout(nkg_graph *g);
// Replace the arc weights in place (device arrays in the caller's order;
// wdeg null: summed on the device over every node's out-arcs).
void set_weights_device(nkg_graph *g, const double *w, const double *wdeg);
} // namespace nkg
