/*
 * nkgpu.h - C ABI of the B200 PageRank library (libnkgpu.so).
 *
 * Drop-in boundary for NetworKit's PageRank path. The reference reaches its
 * C++ through Cython (networkit/centrality.pyx:1989-2037 -> PageRank.hpp:28-75);
 * a Cython class replacing it binds the functions below. Plain pointers and
 * sizes only; host arrays are caller-owned and copied; device buffers are
 * owned by the opaque handle.
 *
 * Return codes: 0 on success, a negative NKG_ERR_* otherwise; the message of
 * the last failure on the calling thread is nkg_last_error(). The Python layer
 * raises RuntimeError(nkg_last_error()) like the reference's `except +`
 * translation of std::runtime_error.
 */
#ifndef NKGPU_H
#define NKGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NKG_ABI_VERSION 2

#if defined(__GNUC__)
#define NKG_API __attribute__((visibility("default")))
#else
#define NKG_API
#endif

enum {
    NKG_OK = 0,
    NKG_ERR_INVALID_ARG = -1, /* bad sizes, pointers, CSR contents */
    NKG_ERR_CUDA = -2,        /* a CUDA runtime call failed */
    NKG_ERR_OOM = -3,         /* device allocation failed */
    NKG_ERR_CANCELLED = -4,   /* nkg_cancel() was called during the run */
    NKG_ERR_TIMEOUT = -5,     /* a bounded device-side wait gave up */
    NKG_ERR_NOT_RUN = -6,     /* result requested before a run */
    NKG_ERR_NO_DEVICE = -7    /* no usable CUDA device */
};

/* PageRank::Norm (PageRank.hpp:31): L1Norm = 0, L2Norm = 1. */
enum { NKG_NORM_L1 = 0, NKG_NORM_L2 = 1 };

/* Arithmetic of the iteration. FP64 keeps the reference's arithmetic
 * (PageRank.cpp:56-66). FP32_REFINE runs the sweeps in FP32 and corrects the
 * iterate with FP64 residual sweeps until the FP64 stopping test holds. */
enum { NKG_PREC_FP64 = 0, NKG_PREC_FP32_REFINE = 1, NKG_PREC_FP32 = 2 };

typedef struct nkg_graph nkg_graph;

/* Flag of nkg_pagerank_run_ex, nkg_graph_set_weights and nkg_pagerank_adjoint:
 * every array argument is DEVICE memory on the graph's device (without it,
 * host memory). */
#define NKG_DEVICE_PTRS 1

/* PageRank(G, damp, tol, normalized) (PageRank.hpp:40, centrality.pyx:2006)
 * plus the public fields norm / maxIterations (PageRank.hpp:64,67) and the
 * distributeSinks flag (redistribute the mass of out-degree-0 nodes uniformly
 * every iteration; 0 keeps the reference's semantics). */
typedef struct {
    double damp;
    double tol;
    int32_t norm;
    int32_t normalized;
    int32_t distribute_sinks;
    int32_t precision;
    uint64_t max_iterations; /* UINT64_MAX = unbounded (the reference default) */
} nkg_pr_params;

/* Per-run statistics (device timings from CUDA events on the handle's stream).
 * Residual trace: before the call the caller may point residual_trace at an
 * array of trace_capacity doubles (NULL / 0: no trace). A PageRank run
 * (nkg_pagerank_run*) then stores there the stopping-test residual of every
 * sweep that the test is applied to, in order (the values `converged()` of
 * PageRank.cpp:41-51 compares with tol): every sweep of the FP64 and FP32
 * power iterations, every FP64 sweep of FP32_REFINE. trace_length receives
 * the number of such sweeps, which may exceed what was stored (at most
 * trace_capacity entries, and at most the first 65,536 sweeps). Every call
 * that fills an nkg_stats keeps residual_trace and trace_capacity as given;
 * the other calls report trace_length 0. A caller that does not use the trace
 * zero-initialises the struct (nkg_stats st = {0};). */
typedef struct {
    uint64_t iterations;       /* numberOfIterations() */
    double residual;           /* last residual norm (L1 sum or L2 sqrt) */
    double sink_mass;          /* sum of scores of out-degree-0 nodes, last iterate */
    double ms_total;           /* device time of the whole run */
    double ms_iterations;      /* device time of the iteration loop */
    uint64_t kernel_launches;  /* kernels this library launched for the run */
    uint64_t fp64_sweeps;      /* SpMV sweeps in FP64 */
    uint64_t fp32_sweeps;      /* SpMV sweeps in FP32 */
    uint64_t bytes_per_sweep_fp64; /* algorithmic bytes of one FP64 sweep */
    uint64_t bytes_per_sweep_fp32; /* algorithmic bytes of one FP32 sweep */
    double *residual_trace;    /* in: caller's array, or NULL */
    uint64_t trace_capacity;   /* in: entries of residual_trace */
    uint64_t trace_length;     /* out: sweeps with a stopping test */
} nkg_stats;

/* Graph shape after upload. */
typedef struct {
    uint64_t z;          /* upperNodeIdBound */
    uint64_t n;          /* numberOfNodes */
    uint64_t arcs;       /* in-arcs traversed per sweep */
    uint64_t sinks;      /* existing nodes with out-degree 0 */
    uint64_t slots;      /* arc slots of the sliced layout (arcs + padding) */
    uint64_t split_rows; /* rows longer than one chunk, summed in pieces */
    int32_t weighted;
    int32_t directed;
    int32_t device;
    int32_t row_order;   /* the relabelling used (nkg_graph_options.row_order, resolved) */
    double ms_create;    /* device time of nkg_graph_create after the copies */
} nkg_graph_info;

/* Options of nkg_graph_create_ex. */
typedef struct {
    int32_t device;      /* CUDA device ordinal (-1: current device) */
    int32_t sweep_shape; /* launch shape of the sweep kernels: threads per CTA and
                            gathers in flight per lane (-1 default = 0: 512
                            threads, 8; 1: 256, 8; 2: 256, 4; 3: 256, 16) */
    int32_t arc_order;   /* 0 (default): keep every in-row in the caller's order,
                            which is the reference's summation order; 1: sort
                            each in-row by source after relabelling (faster
                            gathers, sums rounded in a different order) */
    int32_t row_order;   /* relabelling of the rows for the sliced layout: 0 (default)
                            in-degree, descending; 1 half-octave in-degree buckets,
                            descending, keeping the caller's id order inside a bucket
                            (for numberings that carry locality - geometric, crawl or
                            mesh order: neighbouring rows then gather from neighbouring
                            ids and share sectors; slices pad a little more); -1
                            automatic: 1 when more than 1/4 of 65,536 sampled arcs join
                            ids closer than max(64, z/1024), else 0; nkg_graph_create
                            (no options) uses -1. Results do not depend on it beyond
                            the order of the reductions */
    int32_t hot_tier_kb; /* shared-memory tier of the PageRank sweep: the iterate
                            of the first ids (the most-gathered sources after
                            the relabelling) is copied into this many KB of
                            shared memory per CTA every sweep, and gathers of
                            those ids read it there (1..224 KB; 0: no tier, the
                            whole L1 for the gathers; -1: the library's choice,
                            no tier). Every row sum is the same either way; the
                            residual and sink mass are summed over a different
                            number of CTAs */
} nkg_graph_options;

/* Upload a graph given as its in-adjacency CSR.
 * Replaces constructing NetworKit::Graph + the per-run deg[] setup
 * (PageRank.cpp:29-30) on the GPU side; the in-adjacency is what
 * Graph::forInEdgesOf visits (Graph.hpp:1917-1938): for directed graphs the
 * in-lists, for undirected graphs the neighbour lists (self-loops once).
 *   z           upperNodeIdBound (node ids 0..z-1), 1 <= z < 2^32
 *   arcs        in_row_ptr[z], < 2^32
 *   in_row_ptr  z+1 offsets, non-decreasing, in_row_ptr[0] = 0
 *   in_col      source node of each in-arc, < z and existing
 *   in_w        in-arc weights (NULL: unweighted, every weight 1.0)
 *   out_wdeg    weightedDegree(u) (Graph.cpp:426-452); read only for weighted
 *               graphs (for unweighted graphs it is the out-degree, which
 *               the library counts itself). May be NULL when in_w is NULL.
 *   exists      node-existence mask (NULL: all nodes exist); deleted nodes
 *               must have no arcs
 *   directed    informational (the CSR already encodes the direction) */
NKG_API int nkg_graph_create(nkg_graph **out, uint64_t z, uint64_t arcs, const uint64_t *in_row_ptr,
                     const uint32_t *in_col, const double *in_w, const double *out_wdeg,
                     const uint8_t *exists, int directed);
NKG_API int nkg_graph_create_ex(nkg_graph **out, uint64_t z, uint64_t arcs, const uint64_t *in_row_ptr,
                        const uint32_t *in_col, const double *in_w, const double *out_wdeg,
                        const uint8_t *exists, int directed, const nkg_graph_options *opts);
/* The same graph from its edge list, built on the device: edge e = (src[e],
 * dst[e]) with weight w[e] (w NULL: unweighted), in the order Graph::addEdge
 * was called (Graph.cpp:549-596). The in-adjacency is what Graph stores: for
 * directed graphs row v lists the sources of v's in-edges, for undirected
 * graphs row x lists the other endpoint of every edge at x (a self-loop
 * once), in edge order; weighted degrees are summed in edge order, as the
 * host builder does. Duplicate edges stay (as addEdge keeps them). flags: 0
 * (host arrays) or NKG_DEVICE_PTRS (src, dst, w, exists in device memory).
 * No reference counterpart as a single call (GPU ingest). */
NKG_API int nkg_graph_create_from_edges(nkg_graph **out, uint64_t z, uint64_t m,
                                        const uint32_t *src, const uint32_t *dst, const double *w,
                                        const uint8_t *exists, int directed, int flags,
                                        const nkg_graph_options *opts);
/* NetworkitBinaryReader::read (NetworkitBinaryReader.cpp:19-235) on the GPU:
 * a NetworkitBinaryGraph file (its `size` bytes, host memory or, with flags =
 * NKG_DEVICE_PTRS, device memory) decoded on the device straight into the
 * graph, with the adjacency the reference reader stores (directed: row v = v's
 * transpose list, weighted degree = the sum of v's out-list weights in list
 * order; undirected: row v = v's adjacency list, then its transpose list
 * without self-loops; weighted degree = the row's sum in row order; node flag
 * bit 0 = the node exists). Every weight encoding (none, varint, zigzag,
 * double, float). The decode is fully parallel: a scan finds every varint,
 * one CTA per file chunk walks the list lengths. Malformed files (magic,
 * sections outside the file, chunks not starting at a list length, truncated
 * lists, neighbour ids >= the node count) fail with NKG_ERR_INVALID_ARG.
 * ms_decode_out (nullable): device time of the decode, after the copy of a
 * host file.
 * nkg_graph_create_from_nkbg_file: the same from the file at `path` (what
 * NetworkitBinaryReader::read(path) takes): reader threads read it in pieces
 * of staging_bytes (0: 16 MiB) into page-locked staging blocks and copy each
 * piece to the device as soon as it is read, so reading and copying overlap;
 * s_load_out (nullable): host seconds from opening the file to all of it on
 * the device. A file that cannot be opened or read fails with
 * NKG_ERR_INVALID_ARG.
 * nkg_nkbg_decode: the same decode into caller-owned HOST arrays (any may be
 * NULL; sizes from a first call with all of them NULL: z_out, arcs_out):
 * in_ptr z+1, in_col / in_w arcs, wdeg / outdeg / exists z. */
NKG_API int nkg_graph_create_from_nkbg(nkg_graph **out, const void *file, uint64_t size,
                                       int flags, const nkg_graph_options *opts,
                                       double *ms_decode_out);
NKG_API int nkg_graph_create_from_nkbg_file(nkg_graph **out, const char *path,
                                            uint64_t staging_bytes,
                                            const nkg_graph_options *opts,
                                            double *ms_decode_out, double *s_load_out);
NKG_API int nkg_nkbg_decode(const void *file, uint64_t size, int flags, int device,
                            uint64_t *z_out, uint64_t *arcs_out, int *directed_out,
                            int *weighted_out, uint64_t *in_ptr, uint32_t *in_col, double *in_w,
                            double *wdeg, uint32_t *outdeg, uint8_t *exists,
                            double *ms_decode_out);
NKG_API void nkg_graph_destroy(nkg_graph *g);
NKG_API int nkg_graph_get_info(const nkg_graph *g, nkg_graph_info *info);

/* PageRank::run() (PageRank.cpp:20-104) followed by scores()
 * (Centrality.cpp:43-46) and maximum() (PageRank.cpp:106-108).
 * scores_out: host array of z doubles (non-existent ids get 1/n, as the
 * reference leaves them). Any of iterations_out, max_out, stats may be NULL.
 * Blocks until the run has finished. */
NKG_API int nkg_pagerank_run(nkg_graph *g, const nkg_pr_params *p, double *scores_out,
                     uint64_t *iterations_out, double *max_out, nkg_stats *stats);

/* Same as nkg_pagerank_run, but the z scores are written to DEVICE memory
 * (d_scores_out, on the graph's device); nothing crosses PCIe but the
 * iteration status. */
NKG_API int nkg_pagerank_run_device(nkg_graph *g, const nkg_pr_params *p, double *d_scores_out,
                            uint64_t *iterations_out, double *max_out, nkg_stats *stats);

/* Personalised PageRank with an explicit teleport distribution t (host array
 * of z doubles, summing to 1 over existing nodes): the uniform (1-damp)/n of
 * PageRank.cpp:25,65 becomes (1-damp)*t[u] and, with distribute_sinks, the
 * sink mass is spread along t. Otherwise identical to nkg_pagerank_run. */
NKG_API int nkg_pagerank_run_teleport(nkg_graph *g, const nkg_pr_params *p, const double *teleport,
                              double *scores_out, uint64_t *iterations_out, double *max_out,
                              nkg_stats *stats);

/* nkg_pagerank_run / nkg_pagerank_run_teleport with the array arguments in
 * host or device memory (flags: 0 or NKG_DEVICE_PTRS): teleport (z doubles,
 * NULL for the uniform teleport) and scores_out (z doubles). */
NKG_API int nkg_pagerank_run_ex(nkg_graph *g, const nkg_pr_params *p, const double *teleport,
                                double *scores_out, int flags, uint64_t *iterations_out,
                                double *max_out, nkg_stats *stats);

/* Differentiable form, no reference counterpart.
 *
 * nkg_graph_set_weights: replace the arc weights of a graph created weighted
 * (with arc_order 0): in_w holds `arcs` weights in the order of the in_col
 * given to nkg_graph_create; out_wdeg (z doubles) the new weighted degrees,
 * or NULL to have them summed on the device (over each node's out-arcs, in
 * the order those arcs appear in the in-CSR). The graph keeps its layout and
 * buffers; what differs is the weights only, as if the graph had been created
 * with them.
 *
 * nkg_pagerank_adjoint: the backward pass of PageRank (normalized = 0) for a
 * loss L(scores). Inputs: the parameters and teleport (NULL: uniform) of the
 * forward run, its scores (z doubles, the converged output of
 * nkg_pagerank_run*), and grad_scores = dL/dscores (z doubles). Outputs
 * (each may be NULL): grad_w_out = dL/dw for every arc (`arcs` doubles, the
 * order of in_col; for unweighted graphs the derivative at w = 1), and
 * grad_t_out = dL/dteleport (z doubles; 0 at deleted ids). The adjoint
 * system (I - damp M^T) lam = grad - (grad.scores) 1 is solved to
 * |residual|_1 <= tol * |right-hand side|_1: p->precision FP64 by Jacobi
 * sweeps, FP32_REFINE by FP32 BiCGSTAB with FP64 residual sweeps, FP32 by
 * FP32 BiCGSTAB alone (to max(tol, 3e-7)). iterations_out / stats count the
 * sweeps (fp64_sweeps, fp32_sweeps). flags: 0 or NKG_DEVICE_PTRS. */
NKG_API int nkg_graph_set_weights(nkg_graph *g, const double *in_w, const double *out_wdeg,
                                  int flags);
NKG_API int nkg_pagerank_adjoint(nkg_graph *g, const nkg_pr_params *p, const double *teleport,
                                 const double *scores, const double *grad_scores,
                                 double *grad_w_out, double *grad_t_out, int flags,
                                 uint64_t *iterations_out, nkg_stats *stats);

/* Batched personalised PageRank, no reference counterpart: k <= 256 columns,
 * column j with the teleport t_j = e_{seeds[j]} (seeds are node ids of the
 * caller), solved together as one FP32 SpMM over the shared graph (each
 * column is PageRank.cpp:56-70 with the uniform teleport replaced by t_j;
 * with distribute_sinks the sink mass of column j goes to seeds[j]). Every
 * column starts at 1/n, keeps its own FP64 residual and stops (its values
 * freeze) once that residual is <= tol or max_iterations sweeps are done.
 * Output: column-major k x z floats, column j at scores_out + j*z, in the
 * caller's ids, each column normalised like PageRank.cpp:75-92.
 * scores_out is host memory (out_on_device = 0) or device memory (1).
 * iterations_out (nullable): k sweep counts. Unweighted graphs only. */
NKG_API int nkg_ppr_run(nkg_graph *g, const nkg_pr_params *p, uint32_t k, const uint32_t *seeds,
                        float *scores_out, int out_on_device, uint64_t *iterations_out,
                        nkg_stats *stats);

/* Many-graph batch, no reference counterpart: `count` independent graphs
 * (each PageRank.cpp:20-104 on its own: its own n, teleport (1-damp)/n,
 * residual and stopping test) solved together by one persistent kernel
 * launch, captured in a CUDA graph. The graphs come as one block-diagonal
 * in-CSR: graph i owns the node ids [node_offsets[i], node_offsets[i+1]) and
 * every arc stays inside its graph (checked). Unweighted; all nodes exist.
 * FP32 runs stop at tol, at max_iterations, or at the FP32 rounding floor (a
 * residual that shrinks by less than 0.9x in one sweep, which the exact
 * iteration never does); FP64 runs stop at tol or max_iterations.
 * The kernel's launch shape comes from nkg_batch_tuning: thread-block
 * cluster size, threads per CTA, and the row-split threshold (rows longer
 * than `split` arcs are summed by a whole warp, the others one per lane in
 * 32-row slices). nkg_batch_tune times `sweeps` sweeps of every graph for
 * each candidate (split 32..1024, 256 or 512 threads, clusters 1..16), or
 * with sweeps = 0 the whole run to convergence under *p (the real objective:
 * it sees the largest graphs' critical path), then the kernel variants on
 * the best of those, and keeps the fastest; results (nullable, `capacity`
 * entries) receive every timed candidate, n_results their count.
 * nkg_batch_run: scores_out = the total node count of doubles (caller ids,
 * each graph normalised like PageRank.cpp:75-92), host or device memory
 * (flags 0 / NKG_DEVICE_PTRS); iterations_out (nullable, host) = count sweep
 * counts; floor_stops_out (nullable) = graphs stopped at the FP32 floor. */
typedef struct nkg_batch nkg_batch;
typedef struct {
    uint32_t cluster;  /* CTAs per thread-block cluster: 1, 2, 4, 8 or 16 */
    uint32_t threads;  /* threads per CTA: 128, 256 or 512 */
    uint32_t split;    /* row-split threshold (arcs) */
    uint32_t variant;  /* kernel variant bits: 1 = 16 slots per batch of gathers
                          (else 8), 2 = iterate loads through L2 only */
    double ms;         /* nkg_batch_tune: device time of the timed sweeps */
} nkg_batch_tuning;
NKG_API int nkg_batch_create(nkg_batch **out, uint32_t count, const uint64_t *node_offsets,
                             const uint64_t *in_row_ptr, const uint32_t *in_col, int device);
NKG_API void nkg_batch_destroy(nkg_batch *b);
NKG_API int nkg_batch_get_tuning(const nkg_batch *b, nkg_batch_tuning *t);
NKG_API int nkg_batch_set_tuning(nkg_batch *b, const nkg_batch_tuning *t);
NKG_API int nkg_batch_tune(nkg_batch *b, const nkg_pr_params *p, uint32_t sweeps,
                           nkg_batch_tuning *results, uint32_t capacity, uint32_t *n_results,
                           nkg_batch_tuning *best_out);
NKG_API int nkg_batch_run(nkg_batch *b, const nkg_pr_params *p, double *scores_out, int flags,
                          uint64_t *iterations_out, uint32_t *floor_stops_out, nkg_stats *stats);
/* Diagnostic: when each graph of the last run (or tuning launch) started and
 * converged, in ms from the earliest start (device global timer); count
 * entries each. */
NKG_API int nkg_batch_graph_times(nkg_batch *b, double *start_ms, double *end_ms);

/* EigenvectorCentrality(G, tol).run() + scores() (EigenvectorCentrality.cpp:20-60,
 * centrality.pyx:1950-1968) and KatzCentrality(G, alpha, beta, tol) with
 * edgeDirection 0 (InEdges) or 1 (OutEdges) (KatzCentrality.cpp:20-72,
 * centrality.pyx:1678-1712; alpha 0 = 1 / (1 + maxDegree); a negative alpha
 * is rejected with the reference's message), on the graph's weights, FP64.
 * The reference has no iteration cap; max_iterations (UINT64_MAX = none)
 * bounds the loop. scores_out: z doubles, host or device (flags 0 /
 * NKG_DEVICE_PTRS); deleted ids keep 1.0 as in the reference. */
NKG_API int nkg_eigenvector_run(nkg_graph *g, double tol, uint64_t max_iterations,
                                double *scores_out, int flags, uint64_t *iterations_out,
                                nkg_stats *stats);
NKG_API int nkg_katz_run(nkg_graph *g, double alpha, double beta, double tol, int edge_direction,
                         uint64_t max_iterations, double *scores_out, int flags,
                         uint64_t *iterations_out, nkg_stats *stats);

/* Centrality::ranking() (Centrality.cpp:29-41): existing nodes sorted by score
 * descending, ties by node id ascending. scores: host array of z doubles (any
 * scores, e.g. from nkg_pagerank_run); ids_out / vals_out: n entries each. */
NKG_API int nkg_ranking(nkg_graph *g, const double *scores, uint64_t *ids_out, double *vals_out);

/* Ask the run on this handle to stop (the reference's SIGINT check,
 * PageRank.cpp:55 / SignalHandling.cpp:62-66): the running nkg_pagerank_run*
 * (or eigenvector, Katz, personalised or adjoint run), or, if none is running,
 * the next one, returns NKG_ERR_CANCELLED at its next check (between
 * CUDA-graph chunks of sweeps). A request is cleared when the run it stopped,
 * or any other run on the handle, ends. Safe from any thread or a signal
 * handler (one atomic store). */
NKG_API void nkg_cancel(nkg_graph *g);

/* Aux::SignalHandler (SignalHandling.cpp:29-60) for the runs on g: while
 * enabled, SIGINT calls nkg_cancel(g) instead of reaching the handler that
 * was installed before, which disabling puts back. One handle at a time per
 * process, like the reference's root handler: enabling for a second handle
 * while one holds SIGINT fails with NKG_ERR_INVALID_ARG. *got_sigint_out
 * (nullable, on disable) tells whether a SIGINT arrived while enabled. */
NKG_API int nkg_sigint_cancels(nkg_graph *g, int enable, int *got_sigint_out);

/* Diagnostic, no reference counterpart: run `sweeps` iterations (precision
 * NKG_PREC_FP64 or NKG_PREC_FP32, the stopping test disabled) on the
 * resident graph with CUDA events on the handle's stream around every
 * launch of the sweep kernel. Reports the mean duration of one sweep-kernel
 * launch and of one whole iteration (sweep + fix-up). bench.py derives the
 * roofline figure from it. */
NKG_API int nkg_profile_sweeps(nkg_graph *g, int precision, int sweeps, double *ms_sweep_kernel,
                               double *ms_iteration);

/* Diagnostic, no reference counterpart: only the gathers of one sweep - the
 * sliced layout's column stream in storage order, padding included, read
 * from the current iterate and summed per thread, eight gathers in flight
 * per thread - timed with CUDA events over `reps` launches (after one
 * untimed launch). Its mean launch time is the random-gather bound of this
 * graph on this GPU, the floor under nkg_profile_sweeps' sweep time. */
NKG_API int nkg_profile_gathers(nkg_graph *g, int precision, int reps, double *ms_gather_kernel);

/* Row partition of the PageRank iteration over several GPUs; no counterpart
 * in the reference (whose run is one shared-memory process). The rows of the
 * in-CSR are cut into contiguous slices of about equal arc counts, one slice
 * per GPU (or several). Each slice computes its rows of the next iterate from
 * the whole previous one (PageRank.cpp:56-66 restricted to its rows); between
 * sweeps the caller all-gathers the slices into the shared iterate and
 * all-reduces the residual and sink-mass partial sums, then applies the
 * stopping test (PageRank.cpp:41-51) and the sink term to the reduced sums.
 *
 * The shared iterate (vec_len doubles, device memory of each GPU) holds the
 * slices in gather form (x / deg, or x for out-degree-0 nodes): slice q at
 * [q * stride, q * stride + rows_q) for a stride >= every rows_q, so that an
 * all-gather of equal blocks assembles it, and a last entry (vec_len - 1) that
 * is 0. The caller numbers the in-arc sources of its slice in that layout.
 *
 * nkg_part_create: row_base = the slice's offset in the shared iterate; rows,
 *   arcs, row_ptr (rows + 1, from 0) and col (arcs, positions < vec_len - 1)
 *   its in-CSR (host arrays, each row in the reference's arc order); w
 *   (nullable) the arc weights; out_deg / out_wdeg (rows) the out-degree count
 *   and, for weighted graphs, the weighted out-degree (Graph.cpp:426-452) of
 *   the slice's nodes in the whole graph. device -1: the current device.
 * nkg_part_begin: x = 1 / n_global (PageRank.cpp:26) into d_y_out (rows, the
 *   slice's block of the shared iterate); p gives damp, norm and
 *   distribute_sinks (FP64 only; tol and max_iterations are the caller's).
 * nkg_part_sweep: one sweep of the slice from the shared iterate d_y_in into
 *   d_y_out (rows), with sink_coef added to every row sum before the damping
 *   (distribute_sinks: the previous iterate's sink mass / n_global). Returns
 *   the slice's residual sum (sum of |x' - x|, or of (x' - x)^2 for L2, before
 *   any square root) and its sink mass (sum of x' over out-degree-0 nodes).
 * nkg_part_sums: sum of x, sum of x over out-degree-0 nodes, and max of x over
 *   the slice, for PageRank.cpp:75-102 after reduction across slices.
 * nkg_part_scores: x / factor for the slice rows into d_out (rows).
 * All d_* pointers are device memory on the slice's device; work runs on
 * `stream` (a cudaStream_t, NULL: the handle's own) and every call returns
 * once it has finished. */
typedef struct nkg_part nkg_part;
NKG_API int nkg_part_create(nkg_part **out, uint64_t vec_len, uint64_t row_base, uint64_t rows,
                            uint64_t arcs, const uint64_t *row_ptr, const uint32_t *col,
                            const double *w, const uint32_t *out_deg, const double *out_wdeg,
                            int device);
NKG_API void nkg_part_destroy(nkg_part *p);
NKG_API int nkg_part_begin(nkg_part *p, const nkg_pr_params *prm, uint64_t n_global,
                           double *d_y_out, void *stream);
NKG_API int nkg_part_sweep(nkg_part *p, const double *d_y_in, double sink_coef, double *d_y_out,
                           double *residual_sum_out, double *sink_sum_out, void *stream);
NKG_API int nkg_part_sums(nkg_part *p, const double *d_y, double *sum_out, double *sink_sum_out,
                          double *max_out, void *stream);
NKG_API int nkg_part_scores(nkg_part *p, const double *d_y, double factor, double *d_out,
                            void *stream);

/* PageRank without any device allocation; no counterpart in the reference.
 * For callers that cannot allocate device memory when they call in: a
 * framework whose caching allocator owns the device memory, a service with
 * a memory budget fixed at start-up, a latency-critical loop in which
 * cudaMalloc/cudaFree would synchronise the device. The caller passes the
 * graph and the output in device memory:
 *   d_in_row_ptr  n+1 in-CSR offsets (device), d_in_col  arcs sources (device)
 *   d_scores_out  n doubles (device)
 * FP64 only and unweighted: every arc counts with weight 1.0 and a node's
 * degree is its number of out-arcs in d_in_col, so weighted graphs must use
 * nkg_pagerank_run. n <= 524288 nodes; larger graphs are rejected with
 * NKG_ERR_INVALID_ARG, as are offsets that are not a CSR (row_ptr[0] != 0,
 * decreasing, or row_ptr[n] != arcs) and column ids >= n; both are checked on
 * the device before any sweep reads the graph. All working storage is one
 * 12.1 MB file-scope __device__ array of the library, held by every GPU that
 * loads the library until the process exits. The first call on a device looks
 * up that array's address (cudaGetSymbolAddress, with the device current) and
 * keeps it; make that first call before any stream capture, and make no call
 * on a device after a cudaDeviceReset of it (the kept address is then stale).
 * Calls share the array: calls that overlap on the GPU (other threads, other
 * streams) race and must be serialised by the caller. Work runs on `stream`
 * (a cudaStream_t; NULL = default stream) and the call returns when it has
 * finished. */
NKG_API int nkg_pagerank_csr_noalloc(uint64_t n, uint64_t arcs, const uint64_t *d_in_row_ptr,
                                     const uint32_t *d_in_col, const nkg_pr_params *p,
                                     double *d_scores_out, uint64_t *iterations_out,
                                     void *stream);

/* Local (seeded) PageRank: ApproximatePageRank (scd/ApproximatePageRank.cpp:18-55,
 * scd.pyx:87-136) and PageRankNibble (scd/PageRankNibble.cpp:28-89,
 * scd.pyx:138-151), many independent problems per call.
 *
 * nkg_local_create uploads the neighbour CSR in Graph::forNeighborsOf order
 * (undirected graphs: the neighbour lists, self-loops once; directed graphs:
 * the out-lists in insertion order), weights w (NULL: unweighted), the
 * existence mask (NULL: all exist) and the graph kind. It computes
 * weightedDegree(u, true) of every node (Graph.cpp:427-453) and
 * 2 * totalEdgeWeight() (Graph.cpp:860-868). memory_budget bounds the
 * problems in flight (0: half the free device memory, at most 48 GiB): each
 * holds a hash map of 40 bytes per entry, 1024 entries at first, doubled when
 * half full; the map pool grows past the budget when one problem's support
 * needs it.
 *
 * nkg_local_run: problem k has the seeds seeds[seed_ptr[k] .. seed_ptr[k+1])
 * (ascending, no duplicates: the reference's std::set<node>) and runs
 * ApproximatePageRank(G, alpha, epsilon).run(seeds) in the reference's push
 * order, bit for bit. With NKG_LOCAL_NIBBLE it also runs
 * PageRankNibble::bestSweepSet on each result (ties of p/vol broken by
 * ascending node id). One problem per seed is SelectiveCommunityDetector::run
 * (SelectiveCommunityDetector.cpp:15-23); one problem of all seeds is
 * expandOneCommunity(seeds). max_pushes bounds the pushes of one problem
 * (UINT64_MAX: none); a problem that reaches it fails the call with
 * NKG_ERR_TIMEOUT. epsilon must be > 0, alpha in (0, 1] and the weights
 * non-negative: then the loop ends (each push moves alpha * r >= alpha *
 * epsilon * vol into the values, which sum to at most 1); the reference does
 * not check these, and its loop need not end without them.
 * support_sizes_out / set_sizes_out
 * (nullable, host) receive per-problem counts.
 * nkg_local_support: the supports of the last run (every node the result
 * map holds), problem after problem, each ascending by id, with its value
 * (values_out nullable); sum of support sizes entries.
 * nkg_local_sets: the PageRankNibble sets of the last run, problem after
 * problem, each ascending. */
typedef struct nkg_local nkg_local;
#define NKG_LOCAL_NIBBLE 2
typedef struct {
    uint64_t pushes;          /* pushes over all problems */
    uint64_t arc_visits;      /* arcs the pushes walked (sum of the pushed rows) */
    uint64_t support;         /* sum of the support sizes */
    uint64_t slots;           /* problems in flight (resident warps) */
    uint64_t table_entries;   /* map entries the last push launch took from the pool */
    uint64_t reruns;          /* push launches repeated to grow the map or result pool */
    double ms_push;           /* device time of the (last) push launch */
    double ms_sweep;          /* ms_total - ms_push: re-runs, sorts and the sweep */
    double ms_total;
    uint64_t kernel_launches;
} nkg_local_stats;
NKG_API int nkg_local_create(nkg_local **out, uint64_t z, const uint64_t *row_ptr,
                             const uint32_t *col, const double *w, const uint8_t *exists,
                             int directed, int device, uint64_t memory_budget);
NKG_API void nkg_local_destroy(nkg_local *h);
NKG_API int nkg_local_run(nkg_local *h, double alpha, double epsilon, uint64_t problems,
                          const uint64_t *seed_ptr, const uint32_t *seeds, int flags,
                          uint64_t max_pushes, uint64_t *support_sizes_out,
                          uint64_t *set_sizes_out, nkg_local_stats *stats);
NKG_API int nkg_local_support(nkg_local *h, uint32_t *nodes_out, double *values_out);
NKG_API int nkg_local_sets(nkg_local *h, uint32_t *nodes_out);

/* Device memory: the library keeps the blocks it frees in a per-device
 * cache keyed by size and hands them out again (a block at most 1/8 larger
 * than the request), so that creating and destroying graphs does not map and
 * unmap device memory each time; an allocation that fails first empties the
 * cache. This returns the cached blocks of `device` (-1: the current device)
 * to the driver; blocks still owned by live handles stay. */
NKG_API int nkg_release_cached_memory(int device);

/* Message of the last failure on the calling thread ("" if none). */
NKG_API const char *nkg_last_error(void);

/* Library ABI version (NKG_ABI_VERSION). */
NKG_API int nkg_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* NKGPU_H */
