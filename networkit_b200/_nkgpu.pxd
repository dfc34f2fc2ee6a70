# Cython declarations of the PageRank part of include/nkgpu.h: the .pxd a
# NetworKit build adds beside networkit/centrality.pyx to reach the library.
# Compiled against the header itself, so a field or signature that drifts from
# it is a C compile error.
from libc.stdint cimport uint8_t, int32_t, uint64_t, uint32_t

cdef extern from "nkgpu.h" nogil:
    ctypedef struct nkg_graph:
        pass

    ctypedef struct nkg_pr_params:
        double damp
        double tol
        int32_t norm
        int32_t normalized
        int32_t distribute_sinks
        int32_t precision
        uint64_t max_iterations

    ctypedef struct nkg_stats:
        uint64_t iterations
        double residual
        double sink_mass
        double ms_total
        double ms_iterations
        uint64_t kernel_launches
        uint64_t fp64_sweeps
        uint64_t fp32_sweeps
        uint64_t bytes_per_sweep_fp64
        uint64_t bytes_per_sweep_fp32
        double *residual_trace
        uint64_t trace_capacity
        uint64_t trace_length

    enum:
        NKG_OK
        NKG_ERR_CANCELLED
        NKG_PREC_FP64
        NKG_PREC_FP32_REFINE
        NKG_PREC_FP32
        NKG_NORM_L1
        NKG_NORM_L2

    int nkg_graph_create(nkg_graph **out, uint64_t z, uint64_t arcs, const uint64_t *in_row_ptr,
                         const uint32_t *in_col, const double *in_w, const double *out_wdeg,
                         const uint8_t *exists, int directed)
    void nkg_graph_destroy(nkg_graph *g)
    int nkg_pagerank_run(nkg_graph *g, const nkg_pr_params *p, double *scores_out,
                         uint64_t *iterations_out, double *max_out, nkg_stats *stats)
    int nkg_ranking(nkg_graph *g, const double *scores, uint64_t *ids_out, double *vals_out)
    void nkg_cancel(nkg_graph *g)
    int nkg_sigint_cancels(nkg_graph *g, int enable, int *got_sigint_out)
    const char *nkg_last_error()
