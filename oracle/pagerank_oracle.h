/* Test infrastructure only (the oracle): a plain-C restatement of the
 * reference PageRank path, used by the tests, the smoke check and the CPU
 * baseline of bench.py as the checker. The product never links it.
 *
 * Graph input is the in-adjacency in CSR form, exactly what the reference's
 * Graph::forInEdgesOf visits (include/networkit/graph/Graph.hpp:1917-1938):
 * directed graphs -> inEdges[u], undirected graphs -> outEdges[u] (both
 * directions stored, self-loops once, Graph.cpp:549-596), in storage order.
 */
#ifndef NK_PAGERANK_ORACLE_H
#define NK_PAGERANK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double damp;             /* PageRank.hpp:70 */
    double tol;              /* PageRank.hpp:71 */
    int32_t norm;            /* 0 = L1Norm, 1 = L2Norm (PageRank.hpp:31,67) */
    int32_t normalized;      /* PageRank.hpp:73 */
    int32_t distribute_sinks;/* new: redistribute dangling mass every iteration */
    int32_t nthreads;        /* <= 1: sequential sums in node order */
    uint64_t max_iterations; /* PageRank.hpp:64 */
} nko_params;

/* PageRank::run() (PageRank.cpp:20-104) over the in-CSR.
 *   z         upperNodeIdBound
 *   in_ptr    z+1 row offsets; in_col the source of each in-arc
 *   in_w      in-arc weights or NULL (unweighted: every weight is 1.0)
 *   wdeg      weightedDegree(u) of every node (out-degree / out-weight sum)
 *   outdeg    degree(u) (number of out-arcs) of every node, used by the
 *             normalized branch (PageRank.cpp:84) and the sink set
 *   exists    node-existence mask or NULL (all exist)
 *   teleport  personalised teleport distribution (z entries summing to 1 over
 *             existing nodes) or NULL for the uniform (1-damp)/n
 *   scores    out: z entries; iterations, max_out: out
 *   trace     optional per-iteration residual (before the sqrt for L2 it is
 *             already the norm), up to trace_cap entries
 * Returns 0, or -1 on invalid arguments. */
int nko_pagerank(uint64_t z, const uint64_t *in_ptr, const uint32_t *in_col, const double *in_w,
                 const double *wdeg, const uint32_t *outdeg, const uint8_t *exists,
                 const double *teleport, const nko_params *p, double *scores, uint64_t *iterations,
                 double *max_out, double *trace, uint64_t trace_cap);

/* Centrality::ranking() (Centrality.cpp:29-41): existing nodes sorted by
 * score descending, ties by node id ascending. ids/vals get n entries. */
int nko_ranking(uint64_t z, const double *scores, const uint8_t *exists, uint64_t *ids,
                double *vals);

/* FP64 host adjoint for the differentiable form (no reference counterpart).
 * Forward fixed point, with t the teleport distribution (uniform 1/n when
 * teleport is NULL), m the sink mask and A[u,v] = w(v->u)/wdeg[v]:
 *     x = d*(A x + [distribute_sinks] (m.x) t) + (1-d) t,   p = x / sum(x)
 * (the final division is PageRank.cpp:75-80). For a loss L with g = dL/dp:
 *     gbar = (g - (g.p) 1) / sum(x)
 *     lam  = gbar + d*(A^T lam + [distribute_sinks] m (t.lam))   (Jacobi, L1 tol)
 *     c    = A^T lam
 *     dL/dw(v->u) = d * (x[v]/wdeg[v]) * (lam[u] - c[v])
 *     dL/dt[u]    = (d*[distribute_sinks](m.x) + 1 - d) * lam[u]
 * x is the converged, un-normalised vector. grad_w is indexed like in_col.
 * Returns the number of Jacobi sweeps, or -1 on invalid arguments. */
int64_t nko_pagerank_adjoint(uint64_t z, const uint64_t *in_ptr, const uint32_t *in_col,
                             const double *in_w, const double *wdeg, const uint32_t *outdeg,
                             const double *teleport, double damp, int distribute_sinks,
                             const double *x, const double *g, double tol, uint64_t max_iter,
                             double *lam, double *grad_w, double *grad_t, int nthreads);

/* PageRank.cpp:75-102 on a final iterate (in place): normalisation and
 * maximum(); n = numberOfNodes(). */
void nko_finish(uint64_t z, const uint8_t *exists, const uint32_t *outdeg, double damp,
                int normalized, uint64_t n, double *scores, double *max_out);

/* One sweep of a slice of rows of a row-partitioned run (PageRank.cpp:56-66
 * restricted to the slice); see pagerank_oracle.c. */
int nko_sweep_rows(uint64_t rows, const uint64_t *ptr, const uint32_t *col, const double *w,
                   const double *x, const double *wdeg, const uint32_t *outdeg_rows,
                   uint64_t base, double damp, double teleport_prob, double share, int distribute,
                   int l2, double *x_out, double *res_out, double *sink_out);

/* EigenvectorCentrality::run() (EigenvectorCentrality.cpp:20-60): x = 1 for
 * all z ids; repeat values[u] = sum over in-arcs of w * x[v] (arc order),
 * length = sqrt(sum of values^2 over existing nodes, id order), values /=
 * length, swap; until |length - oldLength| <= tol (NumericTools::equal,
 * NumericTools.cpp:16-18); finally |x| if x[0] < 0. Deleted ids keep 1.
 * Returns the number of iterations (capped at max_iter), -1 on bad input. */
int64_t nko_eigenvector(uint64_t z, const uint64_t *in_ptr, const uint32_t *in_col,
                        const double *in_w, const uint8_t *exists, double tol, uint64_t max_iter,
                        double *scores);

/* KatzCentrality::run() (KatzCentrality.cpp:28-72) over the given adjacency
 * (the in-CSR for EdgeDirection::InEdges, the out-CSR for OutEdges):
 * x = 1; repeat values[u] = sum of w * alpha * (1 + x[v]) + beta, length =
 * sqrt(sum of values^2), x = values; until |length - oldLength| <= tol;
 * finally x /= length on existing nodes (deleted ids keep 1). alpha must
 * already be resolved (the reference's 0 = 1 / (1 + maxDegree)). Returns the
 * number of iterations (capped at max_iter), -1 on bad input. */
int64_t nko_katz(uint64_t z, const uint64_t *ptr, const uint32_t *col, const double *w,
                 const uint8_t *exists, double alpha, double beta, double tol, uint64_t max_iter,
                 double *scores);

/* Graph::weightedDegree(u, true) (Graph.cpp:427-453) over a neighbour CSR
 * in forNeighborsOf order: weighted: sum of w, self-loops counted twice, in
 * row order; unweighted: degree + number of self-loops. Returns 0. */
int nko_volumes(uint64_t z, const uint64_t *ptr, const uint32_t *col, const double *w,
                double *vol);

/* ApproximatePageRank::run(seeds) (ApproximatePageRank.cpp:18-55): the FIFO
 * push of Andersen-Chung-Lang on the lazy walk. Every seed (ascending, no
 * duplicates; a std::set) starts with residual 1/|seeds| and is queued; a
 * push of u adds (1-alpha)*res*w/(2*vol u) to each neighbour's residual in
 * row order, queueing a neighbour whose residual crosses eps*vol from below,
 * then sets (p, r)(u) = (p + alpha*res, (1-alpha)*res/2) (a self-loop's share
 * added during the loop is overwritten) and queues u again while
 * r/vol >= eps. Output: every node the map holds (seeds and neighbours of
 * pushed nodes) with its p, ascending by id, at most `cap` of them. Returns
 * the support size (may exceed cap: nothing past cap is written), -1 on bad
 * input. *pushes = number of pushes. */
int64_t nko_apr(uint64_t z, const uint64_t *ptr, const uint32_t *col, const double *w,
                const double *vol, double alpha, double eps, const uint32_t *seeds,
                uint64_t nseeds, uint64_t cap, uint32_t *nodes, double *values,
                uint64_t *pushes);

/* PageRankNibble::bestSweepSet (PageRankNibble.cpp:28-82) on an APR support:
 * values p/vol, ordered descending (ties: ascending node id - the reference's
 * unstable sort leaves tie order open); prefix sets swept in that order with
 * cut += w for a neighbour outside the prefix (the node itself included),
 * cut -= w inside, volume += the row's weight sum, conductance
 * cut / min(volume, total_volume - volume); the first strict minimum over
 * prefixes smaller than n_nodes wins. Writes the chosen set ascending by id
 * into `set`; returns its size, -1 on bad input. */
int64_t nko_sweep_set(uint64_t z, const uint64_t *ptr, const uint32_t *col, const double *w,
                      const double *vol, double total_volume, uint64_t n_nodes,
                      uint64_t support, const uint32_t *nodes, const double *values,
                      uint32_t *set);

#ifdef __cplusplus
}
#endif
#endif
