// Device-resident graph handle (the opaque nkg_graph of nkgpu.h).
#pragma once

#include <atomic>
#include <memory>

#include "common.cuh"
#include "sweep.cuh"

namespace nkg {

// Launch shape of the merge-path sweep (items per tile = THREADS * IPT).
constexpr int kSweepThreads = 256;
constexpr int kSweepIPT = 8;
constexpr int kTile = kSweepThreads * kSweepIPT;
constexpr int kFixThreads = 256;
// Sweeps per captured CUDA graph (even, so every graph starts on buffer 0).
constexpr int kSweepsPerGraph = 8;

// Per-precision work buffers and the captured sweep graph.
template <typename T>
struct Plane {
    DeviceArray<T> y[2];         // ping-pong iterate in gather form
    DeviceArray<T> head, tail;   // per-tile partials
    DeviceArray<T> w;            // arc weights in this precision (weighted)
    DeviceArray<T> degw;         // weighted degree in this precision
    DeviceArray<T> tele;         // personalised teleport, relabelled
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // [personal]
    unsigned sweep_ctas = 0;
    unsigned fix_ctas = 0;
};

} // namespace nkg

struct nkg_graph {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t z = 0, n = 0, arcs = 0, n_nonsink = 0, ntiles = 0;
    bool weighted = false, directed = false, reordered = true;
    double ms_create = 0.0;

    nkg::DeviceArray<uint32_t> perm;     // new id -> original id (n)
    nkg::DeviceArray<uint32_t> inv;      // original id -> new id (z), kNone if absent
    nkg::DeviceArray<uint32_t> row_ptr;  // n+1
    nkg::DeviceArray<uint32_t> col;      // arcs
    nkg::DeviceArray<uint32_t> degc;     // out-degree count (n)
    nkg::DeviceArray<double> w64src;     // arc weights (FP64, relabelled order)
    nkg::DeviceArray<double> degw64src;  // weighted degree (FP64)
    nkg::DeviceArray<uint32_t> tile_row, tile_arc;  // ntiles+1

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
