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
// Cost of a slice in units of one slot step, besides its length (the
// epilogue of its 32 rows).
constexpr uint32_t kSliceOverhead = 3;

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
};

} // namespace nkg

struct nkg_graph {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t z = 0, n = 0, arcs = 0, sinks = 0;
    bool weighted = false, directed = false;
    double ms_create = 0.0;

    nkg::DeviceArray<uint32_t> perm;     // new id -> original id (n)
    nkg::DeviceArray<uint32_t> inv;      // original id -> new id (z), kNone if absent
    nkg::DeviceArray<uint32_t> row_ptr;  // n+1, in-CSR in new ids
    nkg::DeviceArray<uint32_t> col;      // arcs
    nkg::DeviceArray<uint32_t> degc;     // out-degree count (n)
    nkg::DeviceArray<double> w64src;     // CSR arc weights (FP64, relabelled order)
    nkg::DeviceArray<double> degw64src;  // weighted degree (FP64)

    // Sliced layout of the sweep.
    uint32_t n_long = 0, n_vlong = 0, n_chunks = 0, s_chunk = 0, slices = 0;
    int sweep_shape = 0;
    bool arc_sorted = false;
    uint64_t slots = 0;
    nkg::DeviceArray<uint32_t> chunk_begin;  // n_long+1
    nkg::DeviceArray<uint32_t> slice_off;    // slices+1
    nkg::DeviceArray<uint64_t> slice_cost;   // slices, inclusive prefix of slice costs
    nkg::DeviceArray<uint32_t> col_sell;     // slots
    nkg::DeviceArray<double> w_sell64;       // slots (weighted)

    nkg::Plane<double> p64;
    nkg::Plane<float> p32;

    nkg::DeviceArray<double> cta_res, cta_sink, fix_res, fix_sink;
    nkg::DeviceArray<double> out_buf;    // scores staging for host output (z)
    nkg::DeviceArray<double> red;        // scratch for finalisation reductions
    nkg::DeviceArray<unsigned int> red_ticket;
    nkg::DeviceArray<nkg::RunParams> rp;
    nkg::DeviceArray<nkg::IterState> st;
    nkg::PinnedHost<nkg::IterState> st_host;
    nkg::PinnedHost<double> scalars_host;

    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    std::atomic<int> cancel{0};
    bool has_run = false;
};
