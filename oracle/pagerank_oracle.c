/* Test infrastructure only (the oracle): plain-C restatement of the reference
 * PageRank path. Each function cites the reference lines it follows. It is
 * the checker for the CUDA path; the product never links it.
 *
 * Parity pin: with distribute_sinks = 0, a uniform teleport and nthreads <= 1
 * this follows PageRank.cpp:20-104 operation for operation, so its scores are
 * bit-identical to the reference library built from the reference sources
 * (oracle/_ref/libnkref.so) run on one OpenMP thread; tests/test_oracle.py
 * checks that on every golden fixture. The distributeSinks term, the
 * personalised teleport and the adjoint have no reference implementation
 * (parity unpinned); they extend the same loop. EigenvectorCentrality and
 * KatzCentrality (EigenvectorCentrality.cpp, KatzCentrality.cpp) are
 * restated the same way and pinned against the reference library. */
#include "pagerank_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static int exists_at(const uint8_t *exists, uint64_t u) { return exists == NULL || exists[u] != 0; }

/* Graph::parallelSumForNodes (Graph.hpp:2123-2134) of |a-b| or (a-b)^2. */
static double residual_sum(uint64_t z, const uint8_t *exists, const double *a, const double *b,
                           int l2, int nthreads) {
    double sum = 0.0;
    if (nthreads > 1) {
#pragma omp parallel for reduction(+ : sum) num_threads(nthreads) schedule(static)
        for (int64_t u = 0; u < (int64_t)z; ++u) {
            if (exists_at(exists, (uint64_t)u)) {
                const double d = a[u] - b[u];
                sum += l2 ? d * d : fabs(d);
            }
        }
    } else {
        for (uint64_t u = 0; u < z; ++u) {
            if (exists_at(exists, u)) {
                const double d = a[u] - b[u];
                sum += l2 ? d * d : fabs(d);
            }
        }
    }
    return sum;
}

static double sink_mass(uint64_t z, const uint8_t *exists, const uint32_t *outdeg,
                        const double *x) {
    double s = 0.0;
    for (uint64_t u = 0; u < z; ++u)
        if (exists_at(exists, u) && outdeg[u] == 0)
            s += x[u];
    return s;
}

/* PageRank.cpp:75-102 on the final iterate `scores` (in place): the
 * normalisation of both modes and maximum(). */
void nko_finish(uint64_t z, const uint8_t *exists, const uint32_t *outdeg, double damp,
                int normalized, uint64_t n, double *scores, double *max_out) {
    /* PageRank.cpp:75-92 */
    if (!normalized) {
        double sum = 0.0;
        for (uint64_t u = 0; u < z; ++u)
            if (exists_at(exists, u))
                sum += scores[u];
        for (uint64_t u = 0; u < z; ++u)
            if (exists_at(exists, u))
                scores[u] /= sum;
    } else {
        double sum = 0.0;
        for (uint64_t u = 0; u < z; ++u)
            if (exists_at(exists, u) && outdeg[u] == 0)
                sum += scores[u];
        const double normFactor = (1.0 / (double)n) * ((1 - damp) + (damp * sum));
        for (uint64_t u = 0; u < z; ++u)
            if (exists_at(exists, u))
                scores[u] /= normFactor;
    }
    /* PageRank.cpp:95-102 */
    if (max_out) {
        if (!normalized) {
            *max_out = 1.0;
        } else {
            double m = scores[0];
            for (uint64_t u = 0; u < z; ++u)
                if (exists_at(exists, u) && scores[u] > m)
                    m = scores[u];
            *max_out = m;
        }
    }
}

/* One Jacobi sweep (PageRank.cpp:56-66) of a slice of rows, the step each
 * rank of a row-partitioned run takes: row r < rows has the in-arcs
 * ptr[r]..ptr[r+1] whose sources are positions col[e] in the shared vectors x
 * (the previous iterate, x itself) and wdeg (weighted degrees); the new value
 * goes to x_out[r]. The sink term adds `share` to the row sum before the
 * damping when distribute is set. Returns the slice's residual sum against
 * x[base + r] (|d| or d^2, PageRank.cpp:34-39) and its sink mass (new x over
 * rows with outdeg_rows[r] == 0), rows in order. */
int nko_sweep_rows(uint64_t rows, const uint64_t *ptr, const uint32_t *col, const double *w,
                   const double *x, const double *wdeg, const uint32_t *outdeg_rows,
                   uint64_t base, double damp, double teleport_prob, double share, int distribute,
                   int l2, double *x_out, double *res_out, double *sink_out) {
    if (!ptr || !x || !wdeg || !outdeg_rows || !x_out || !res_out || !sink_out)
        return -1;
    double res = 0.0, sink = 0.0;
    for (uint64_t r = 0; r < rows; ++r) {
        double acc = 0.0;
        for (uint64_t e = ptr[r]; e < ptr[r + 1]; ++e) {
            const uint32_t v = col[e];
            const double we = w ? w[e] : 1.0;
            acc += x[v] * we / wdeg[v];
        }
        if (distribute)
            acc += share;
        acc *= damp;
        acc += teleport_prob;
        x_out[r] = acc;
        const double d = x[base + r] - acc;
        res += l2 ? d * d : fabs(d);
        if (outdeg_rows[r] == 0)
            sink += acc;
    }
    *res_out = res;
    *sink_out = sink;
    return 0;
}

int nko_pagerank(uint64_t z, const uint64_t *in_ptr, const uint32_t *in_col, const double *in_w,
                 const double *wdeg, const uint32_t *outdeg, const uint8_t *exists,
                 const double *teleport, const nko_params *p, double *scores, uint64_t *iterations,
                 double *max_out, double *trace, uint64_t trace_cap) {
    if (!in_ptr || !wdeg || !outdeg || !p || !scores || z == 0)
        return -1;
    uint64_t n = 0;
    for (uint64_t u = 0; u < z; ++u)
        n += exists_at(exists, u);
    if (n == 0)
        return -1;
    const int nthreads = p->nthreads;
    const double damp = p->damp;
    /* PageRank.cpp:25-27 */
    const double teleportProb = (1.0 - damp) / (double)n;
    double *scoreData = scores;
    for (uint64_t u = 0; u < z; ++u)
        scoreData[u] = 1.0 / (double)n;
    double *pr = (double *)malloc(z * sizeof(double));
    if (!pr)
        return -1;
    memcpy(pr, scoreData, z * sizeof(double));
    /* PageRank.cpp:29-30: deg[u] = weightedDegree(u) is the caller's wdeg. */
    uint64_t iters = 0;
    int converged = 0;
    do {
        /* Sink term (distributeSinks): the mass of dangling nodes of the
         * previous iterate, spread like the teleport. */
        double share = 0.0, S = 0.0;
        if (p->distribute_sinks) {
            S = sink_mass(z, exists, outdeg, scoreData);
            share = S / (double)n;
        }
        /* PageRank.cpp:56-66 (balancedParallelForNodes + forInEdgesOf) */
#pragma omp parallel for schedule(guided) num_threads(nthreads > 1 ? nthreads : 1)
        for (int64_t ui = 0; ui < (int64_t)z; ++ui) {
            const uint64_t u = (uint64_t)ui;
            if (!exists_at(exists, u))
                continue;
            double acc = 0.0;
            for (uint64_t e = in_ptr[u]; e < in_ptr[u + 1]; ++e) {
                const uint32_t v = in_col[e];
                const double w = in_w ? in_w[e] : 1.0;
                acc += scoreData[v] * w / wdeg[v];
            }
            if (p->distribute_sinks)
                acc += teleport ? S * teleport[u] : share;
            acc *= damp;
            acc += teleport ? (1.0 - damp) * teleport[u] : teleportProb;
            pr[u] = acc;
        }
        ++iters;
        /* PageRank.cpp:41-51 */
        double res;
        if (p->norm == 1)
            res = sqrt(residual_sum(z, exists, scoreData, pr, 1, nthreads));
        else
            res = residual_sum(z, exists, scoreData, pr, 0, nthreads);
        if (trace && iters <= trace_cap)
            trace[iters - 1] = res;
        converged = iters >= p->max_iterations || res <= p->tol;
        /* PageRank.cpp:70: std::swap(pr, scoreData) */
        double *t = pr;
        pr = scoreData;
        scoreData = t;
    } while (!converged);

    if (scoreData != scores) {
        memcpy(scores, scoreData, z * sizeof(double));
        pr = scoreData; /* the malloc'd buffer, freed below */
    }
    nko_finish(z, exists, outdeg, damp, p->normalized, n, scores, max_out);
    if (iterations)
        *iterations = iters;
    free(pr);
    return 0;
}

typedef struct {
    uint64_t id;
    double val;
} rank_pair;

/* Centrality.cpp:34-38: score descending, ties by node id ascending. */
static int rank_cmp(const void *a, const void *b) {
    const rank_pair *x = (const rank_pair *)a, *y = (const rank_pair *)b;
    if (x->val == y->val)
        return x->id < y->id ? -1 : (x->id > y->id ? 1 : 0);
    return x->val > y->val ? -1 : 1;
}

int nko_ranking(uint64_t z, const double *scores, const uint8_t *exists, uint64_t *ids,
                double *vals) {
    rank_pair *r = (rank_pair *)malloc((z ? z : 1) * sizeof(rank_pair));
    if (!r)
        return -1;
    uint64_t n = 0;
    for (uint64_t u = 0; u < z; ++u)
        if (exists_at(exists, u)) {
            r[n].id = u;
            r[n].val = scores[u];
            ++n;
        }
    qsort(r, n, sizeof(rank_pair), rank_cmp);
    for (uint64_t i = 0; i < n; ++i) {
        if (ids)
            ids[i] = r[i].id;
        if (vals)
            vals[i] = r[i].val;
    }
    free(r);
    return 0;
}

/* c = A^T lam over the out-lists built from the in-CSR (pull form, rows in
 * parallel): c[v] = sum over the in-arcs (u <- v), u ascending and then in
 * arc order, of (w / wdeg[v]) * lam[u]. That is the order in which a scatter
 * over the in-CSR (u ascending, arcs in order) adds to c[v], so the result is
 * the same bit for bit for any thread count. */
static void adjoint_pull(uint64_t z, const uint64_t *optr, const uint32_t *orow,
                         const uint64_t *oarc, const double *in_w, const double *wdeg,
                         const double *lam, double *c, int nthreads) {
#pragma omp parallel for schedule(guided) num_threads(nthreads > 1 ? nthreads : 1)
    for (int64_t v = 0; v < (int64_t)z; ++v) {
        double acc = 0.0;
        for (uint64_t k = optr[v]; k < optr[v + 1]; ++k) {
            const double w = in_w ? in_w[oarc[k]] : 1.0;
            acc += w / wdeg[v] * lam[orow[k]];
        }
        c[v] = acc;
    }
}

int64_t nko_pagerank_adjoint(uint64_t z, const uint64_t *in_ptr, const uint32_t *in_col,
                             const double *in_w, const double *wdeg, const uint32_t *outdeg,
                             const double *teleport, double damp, int distribute_sinks,
                             const double *x, const double *g, double tol, uint64_t max_iter,
                             double *lam, double *grad_w, double *grad_t, int nthreads) {
    if (!in_ptr || !wdeg || !outdeg || !x || !g || !lam || z == 0)
        return -1;
    const double n = (double)z;
    const uint64_t m = in_ptr[z];
    double sumx = 0.0, S = 0.0;
    for (uint64_t u = 0; u < z; ++u) {
        sumx += x[u];
        if (outdeg[u] == 0)
            S += x[u];
    }
    double gp = 0.0;
    for (uint64_t u = 0; u < z; ++u)
        gp += g[u] * (x[u] / sumx);
    double *gbar = (double *)malloc(z * sizeof(double));
    double *c = (double *)malloc(z * sizeof(double));
    double *lam2 = (double *)malloc(z * sizeof(double));
    /* Out-lists of the in-CSR: for source v, (target u, arc index e) with u
     * ascending and e ascending within u (a stable counting sort). */
    uint64_t *optr = (uint64_t *)calloc(z + 1, sizeof(uint64_t));
    uint32_t *orow = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    uint64_t *oarc = (uint64_t *)malloc((m ? m : 1) * sizeof(uint64_t));
    uint64_t *fill = (uint64_t *)malloc((z + 1) * sizeof(uint64_t));
    if (!gbar || !c || !lam2 || !optr || !orow || !oarc || !fill) {
        free(gbar);
        free(c);
        free(lam2);
        free(optr);
        free(orow);
        free(oarc);
        free(fill);
        return -1;
    }
    for (uint64_t e = 0; e < m; ++e)
        optr[in_col[e] + 1]++;
    for (uint64_t v = 0; v < z; ++v)
        optr[v + 1] += optr[v];
    memcpy(fill, optr, (z + 1) * sizeof(uint64_t));
    for (uint64_t u = 0; u < z; ++u)
        for (uint64_t e = in_ptr[u]; e < in_ptr[u + 1]; ++e) {
            const uint64_t k = fill[in_col[e]]++;
            orow[k] = (uint32_t)u;
            oarc[k] = e;
        }
    for (uint64_t u = 0; u < z; ++u) {
        gbar[u] = (g[u] - gp) / sumx;
        lam[u] = gbar[u];
    }
    int64_t sweeps = 0;
    for (;;) {
        adjoint_pull(z, optr, orow, oarc, in_w, wdeg, lam, c, nthreads);
        double tl = 0.0;
        if (distribute_sinks)
            for (uint64_t u = 0; u < z; ++u)
                tl += (teleport ? teleport[u] : 1.0 / n) * lam[u];
        double res = 0.0;
        for (uint64_t v = 0; v < z; ++v) {
            double s = c[v];
            if (distribute_sinks && outdeg[v] == 0)
                s += tl;
            lam2[v] = gbar[v] + damp * s;
            res += fabs(lam2[v] - lam[v]);
        }
        memcpy(lam, lam2, z * sizeof(double));
        ++sweeps;
        if (res <= tol || (uint64_t)sweeps >= max_iter)
            break;
    }
    /* c for the final lam */
    adjoint_pull(z, optr, orow, oarc, in_w, wdeg, lam, c, nthreads);
    if (grad_w)
        for (uint64_t u = 0; u < z; ++u)
            for (uint64_t e = in_ptr[u]; e < in_ptr[u + 1]; ++e) {
                const uint32_t v = in_col[e];
                grad_w[e] = damp * (x[v] / wdeg[v]) * (lam[u] - c[v]);
            }
    if (grad_t) {
        const double f = (distribute_sinks ? damp * S : 0.0) + 1.0 - damp;
        for (uint64_t u = 0; u < z; ++u)
            grad_t[u] = f * lam[u];
    }
    free(gbar);
    free(c);
    free(lam2);
    free(optr);
    free(orow);
    free(oarc);
    free(fill);
    return sweeps;
}

/* NumericTools::equal (NumericTools.cpp:16-18). */
static int num_equal(double x, double y, double error) {
    return (x <= (y + error)) && (x >= (y - error));
}

static double length_of(uint64_t z, const uint8_t *exists, const double *v) {
    double sum = 0.0;
    for (uint64_t u = 0; u < z; ++u)
        if (exists_at(exists, u))
            sum += v[u] * v[u];
    return sqrt(sum);
}

int64_t nko_eigenvector(uint64_t z, const uint64_t *in_ptr, const uint32_t *in_col,
                        const double *in_w, const uint8_t *exists, double tol, uint64_t max_iter,
                        double *scores) {
    if (!in_ptr || !scores || z == 0)
        return -1;
    double *values = (double *)malloc(z * sizeof(double));
    double *x = (double *)malloc(z * sizeof(double));
    if (!values || !x) {
        free(values);
        free(x);
        return -1;
    }
    for (uint64_t u = 0; u < z; ++u)
        values[u] = x[u] = 1.0;
    double length = 0.0, old_length = 0.0;
    int64_t it = 0;
    do {
        old_length = length;
        for (uint64_t u = 0; u < z; ++u) {
            if (!exists_at(exists, u))
                continue;
            values[u] = 0.0;
            for (uint64_t e = in_ptr[u]; e < in_ptr[u + 1]; ++e)
                values[u] += (in_w ? in_w[e] : 1.0) * x[in_col[e]];
        }
        length = length_of(z, exists, values);
        for (uint64_t u = 0; u < z; ++u)
            if (exists_at(exists, u))
                values[u] /= length;
        double *t = x;
        x = values;
        values = t;
        ++it;
    } while (!num_equal(length, old_length, tol) && (uint64_t)it < max_iter);
    if (x[0] < 0)
        for (uint64_t u = 0; u < z; ++u)
            if (exists_at(exists, u))
                x[u] = fabs(x[u]);
    memcpy(scores, x, z * sizeof(double));
    free(values);
    free(x);
    return it;
}

int64_t nko_katz(uint64_t z, const uint64_t *ptr, const uint32_t *col, const double *w,
                 const uint8_t *exists, double alpha, double beta, double tol, uint64_t max_iter,
                 double *scores) {
    if (!ptr || !scores || z == 0)
        return -1;
    double *values = (double *)malloc(z * sizeof(double));
    if (!values)
        return -1;
    for (uint64_t u = 0; u < z; ++u)
        values[u] = scores[u] = 1.0;
    double length = 0.0, old_length = 0.0;
    int64_t it = 0;
    do {
        old_length = length;
        for (uint64_t u = 0; u < z; ++u) {
            if (!exists_at(exists, u))
                continue;
            values[u] = 0.0;
            for (uint64_t e = ptr[u]; e < ptr[u + 1]; ++e)
                values[u] += (w ? w[e] : 1.0) * alpha * (1 + scores[col[e]]);
            values[u] += beta;
        }
        length = length_of(z, exists, values);
        memcpy(scores, values, z * sizeof(double));
        ++it;
    } while (!num_equal(length, old_length, tol) && (uint64_t)it < max_iter);
    for (uint64_t u = 0; u < z; ++u)
        if (exists_at(exists, u))
            scores[u] /= length;
    free(values);
    return it;
}

/* ---------------------------------------------------------------------------
 * Local PageRank: ApproximatePageRank (ApproximatePageRank.cpp:18-55) and the
 * sweep of PageRankNibble (PageRankNibble.cpp:28-82).
 * ------------------------------------------------------------------------- */

int nko_volumes(uint64_t z, const uint64_t *ptr, const uint32_t *col, const double *w,
                double *vol) {
    for (uint64_t u = 0; u < z; ++u) {
        if (w) {
            double sum = 0.0;
            for (uint64_t k = ptr[u]; k < ptr[u + 1]; ++k)
                sum += (col[k] == u) ? 2. * w[k] : w[k];
            vol[u] = sum;
        } else {
            uint64_t sum = ptr[u + 1] - ptr[u];
            for (uint64_t k = ptr[u]; k < ptr[u + 1]; ++k)
                sum += (col[k] == u);
            vol[u] = (double)sum;
        }
    }
    return 0;
}

typedef struct {
    uint32_t *buf;
    uint64_t cap, head, size;
} fifo_t;

static int fifo_push(fifo_t *q, uint32_t v) {
    if (q->size == q->cap) {
        uint64_t ncap = q->cap ? 2 * q->cap : 64;
        uint32_t *nb = (uint32_t *)malloc(ncap * sizeof(uint32_t));
        if (!nb)
            return -1;
        for (uint64_t i = 0; i < q->size; ++i)
            nb[i] = q->buf[(q->head + i) % q->cap];
        free(q->buf);
        q->buf = nb;
        q->cap = ncap;
        q->head = 0;
    }
    q->buf[(q->head + q->size) % q->cap] = v;
    q->size++;
    return 0;
}

static uint32_t fifo_pop(fifo_t *q) {
    uint32_t v = q->buf[q->head];
    q->head = (q->head + 1) % q->cap;
    q->size--;
    return v;
}

int64_t nko_apr(uint64_t z, const uint64_t *ptr, const uint32_t *col, const double *w,
                const double *vol, double alpha, double eps, const uint32_t *seeds,
                uint64_t nseeds, uint64_t cap, uint32_t *nodes, double *values,
                uint64_t *pushes) {
    if (nseeds == 0)
        return -1;
    for (uint64_t i = 0; i < nseeds; ++i)
        if (seeds[i] >= z || (i && seeds[i] <= seeds[i - 1]))
            return -1;
    double *r = (double *)calloc(z ? z : 1, sizeof(double));
    double *p = (double *)calloc(z ? z : 1, sizeof(double));
    uint8_t *in_map = (uint8_t *)calloc(z ? z : 1, 1);
    fifo_t q = {NULL, 0, 0, 0};
    int64_t ret = -1;
    uint64_t npush = 0;
    if (!r || !p || !in_map)
        goto done;
    const double init_res = 1.0 / (double)nseeds;
    for (uint64_t i = 0; i < nseeds; ++i) {
        const uint32_t s = seeds[i];
        in_map[s] = 1;
        p[s] = 0.0;
        r[s] = init_res;
        if (fifo_push(&q, s))
            goto done;
    }
    while (q.size) {
        const uint32_t u = fifo_pop(&q);
        const double res = r[u];
        const double volume = vol[u];
        for (uint64_t k = ptr[u]; k < ptr[u + 1]; ++k) {
            const uint32_t v = col[k];
            const double wk = w ? w[k] : 1.0;
            const double mass = (1.0 - alpha) * res * wk / (2.0 * volume);
            const double vol_v = vol[v];
            in_map[v] = 1;
            if (r[v] < vol_v * eps && (r[v] + mass) >= eps * vol_v)
                if (fifo_push(&q, v))
                    goto done;
            r[v] += mass;
        }
        p[u] = p[u] + alpha * res;
        r[u] = (1.0 - alpha) * res / 2;
        if ((r[u] / volume) >= eps)
            if (fifo_push(&q, u))
                goto done;
        npush++;
    }
    {
        uint64_t cnt = 0;
        for (uint64_t v = 0; v < z; ++v)
            if (in_map[v]) {
                if (cnt < cap) {
                    nodes[cnt] = (uint32_t)v;
                    values[cnt] = p[v];
                }
                cnt++;
            }
        ret = (int64_t)cnt;
    }
done:
    if (pushes)
        *pushes = npush;
    free(r);
    free(p);
    free(in_map);
    free(q.buf);
    return ret;
}

/* Order-preserving map of a double onto uint64 (sign-magnitude to offset
 * binary): numeric order, -0 before +0, NaNs at the ends. */
static uint64_t order_bits(double d) {
    uint64_t u;
    memcpy(&u, &d, 8);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

typedef struct {
    uint64_t key;
    uint32_t node;
} sweep_item;

static int sweep_cmp(const void *a, const void *b) {
    const sweep_item *x = (const sweep_item *)a, *y = (const sweep_item *)b;
    if (x->key != y->key)
        return x->key > y->key ? -1 : 1;
    return x->node < y->node ? -1 : (x->node > y->node);
}

static int u32_cmp(const void *a, const void *b) {
    const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : (x > y);
}

int64_t nko_sweep_set(uint64_t z, const uint64_t *ptr, const uint32_t *col, const double *w,
                      const double *vol, double total_volume, uint64_t n_nodes,
                      uint64_t support, const uint32_t *nodes, const double *values,
                      uint32_t *set) {
    sweep_item *it = (sweep_item *)malloc((support ? support : 1) * sizeof(sweep_item));
    uint8_t *within = (uint8_t *)calloc(z ? z : 1, 1);
    int64_t ret = -1;
    if (!it || !within)
        goto done;
    for (uint64_t i = 0; i < support; ++i) {
        if (nodes[i] >= z)
            goto done;
        it[i].node = nodes[i];
        it[i].key = order_bits(values[i] / vol[nodes[i]]);
    }
    qsort(it, support, sizeof(sweep_item), sweep_cmp);
    {
        double best_cond = 1.79769313486231570815e+308; /* DBL_MAX */
        double cut = 0.0, volume = 0.0;
        uint64_t best = 0;
        for (uint64_t i = 0; i < support; ++i) {
            const uint32_t v = it[i].node;
            double wdeg = 0.0;
            for (uint64_t k = ptr[v]; k < ptr[v + 1]; ++k) {
                const double wk = w ? w[k] : 1.0;
                wdeg += wk;
                if (!within[col[k]])
                    cut += wk;
                else
                    cut -= wk;
            }
            volume += wdeg;
            within[v] = 1;
            const double other = total_volume - volume;
            const double cond = cut / ((other < volume) ? other : volume); /* std::min */
            if ((cond < best_cond) && (i + 1 < n_nodes)) {
                best_cond = cond;
                best = i + 1;
            }
        }
        for (uint64_t i = 0; i < best; ++i)
            set[i] = it[i].node;
        qsort(set, best, sizeof(uint32_t), u32_cmp);
        ret = (int64_t)best;
    }
done:
    free(it);
    free(within);
    return ret;
}
