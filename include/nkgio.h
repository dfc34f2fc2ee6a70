/* Graph file input for the PageRank path: host-side decoding of the
 * NetworkitBinaryGraph format (networkit/cpp/io/NetworkitBinaryGraph.md) into
 * the in-adjacency CSR that nkg_graph_create takes, and the matching writer.
 * Built into libnkgen.so (C++/OpenMP, one thread per file chunk).
 *
 * nkgen_read_nkbg replaces NetworkitBinaryReader::read
 * (NetworkitBinaryReader.cpp:19-235, graphio.pyx:145-151), without building a
 * Graph: the arrays it returns are exactly the adjacency the reference's
 * reader stores, in storage order:
 *   directed graphs    row v = v's transpose list (in-neighbours),
 *                      wdeg[v] = sum of v's out-list weights in list order,
 *                      outdeg[v] = length of v's out-list;
 *   undirected graphs  row v = v's adjacency list, then its transpose list
 *                      without self-loops; wdeg[v] = the row's weight sum in
 *                      row order; outdeg[v] = the row length.
 * exists[v] = bit 0 of v's flag byte. Weights (w, NULL when the file has
 * none) in the file's encoding: unsigned varint, zigzag varint, double or
 * float. The arrays are malloc'ed; nkgen_graph_free releases them. */
#ifndef NKGIO_H
#define NKGIO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NKGEN_API __attribute__((visibility("default")))

typedef struct {
    uint64_t z;       /* node count of the file (upperNodeIdBound) */
    uint64_t arcs;    /* in_ptr[z] */
    uint64_t *in_ptr; /* z + 1 */
    uint32_t *in_col; /* arcs */
    uint32_t *outdeg; /* z */
    double *w;        /* arcs, NULL when unweighted */
    double *wdeg;     /* z */
    uint8_t *exists;  /* z */
    int directed;
    int weighted;
} nkgen_graph;

/* Decode `path` with `nthreads` OpenMP threads (0: the OpenMP default).
 * Returns 0, or -1 with the message in nkgen_io_last_error(): not the
 * format (magic "nkbg002"), sections outside the file, truncated lists,
 * neighbour ids >= the node count, an unknown weight encoding. */
NKGEN_API int nkgen_read_nkbg(const char *path, int nthreads, nkgen_graph *out);
NKGEN_API void nkgen_graph_free(nkgen_graph *g);

/* NetworkitBinaryWriter(chunks, weights).write(G, path)
 * (NetworkitBinaryWriter.cpp:21-380, graphio.pyx:153-159), byte for byte.
 * The graph: n nodes, all existing (the reference writer numbers only
 * existing nodes, so a graph with deleted nodes does not round trip through
 * it); out_ptr / out_col / out_w its out-lists in outEdges storage order (for
 * undirected graphs the neighbour lists); for directed graphs in_ptr / in_col
 * / in_w its in-lists in inEdges order (NULL for undirected graphs). Weights
 * NULL: unweighted (every weight 1.0). weights: 0 none, 1 unsigned varint,
 * 2 signed varint, 3 double, 4 float, 5 the narrowest that holds every edge
 * weight (the reference's autoDetect). chunks is capped at n. The file is
 * encoded in memory by nthreads OpenMP threads (0: the OpenMP default), one
 * chunk each, and written once. Returns 0, or -1 with the message in
 * nkgen_io_last_error(). */
NKGEN_API int nkgen_write_nkbg(const char *path, uint64_t n, int directed, const uint64_t *out_ptr,
                               const uint32_t *out_col, const double *out_w,
                               const uint64_t *in_ptr, const uint32_t *in_col,
                               const double *in_w, uint64_t chunks, int weights, int nthreads);
NKGEN_API const char *nkgen_io_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
