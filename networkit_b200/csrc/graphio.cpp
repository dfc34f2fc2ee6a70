// Host-side graph file decoding (C++/OpenMP) into the in-CSR the PageRank
// boundary takes, without building a Graph: the NetworkitBinaryGraph format
// (NetworkitBinaryGraph.md; the layout and the adjacency the reference's
// NetworkitBinaryReader builds, NetworkitBinaryReader.cpp:19-235).
//
// File: a header of ten 64-bit words (magic "nkbg002", checksum, features,
// nodes, chunks, and the absolute offsets of the base data, adjacency lists,
// transpose lists, adjacency weights, transpose weights); base data = one flag
// byte per node (bit 0: the node exists) and the first node of chunks 1..;
// every list section = the (chunks-1) chunk offsets, the list total, then per
// node its length and entries as prefix-length varints (the number of
// trailing zero bits of the first byte is the number of extra bytes; the
// remaining high bits of the first byte are the lowest value bits, the extra
// bytes follow little-endian; a zero first byte means 8 extra bytes).
// Weights: none, unsigned varint, zigzag varint, double or float, per list
// entry, in a section with its own chunk offsets.
//
// The in-CSR it yields is the adjacency the reference reader stores: directed
// graphs: row v = v's transpose list (its in-neighbours), weighted degree =
// sum of v's out-list weights in list order; undirected graphs: row v = v's
// out list, then its transpose list without self-loops; weighted degree = sum
// over that row in row order.
#include "nkgio.h"

#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_io_err;

// One prefix-length varint; returns the bytes consumed (0 past `end`).
inline size_t read_varint(const uint8_t *p, const uint8_t *end, uint64_t &value) {
    if (p >= end)
        return 0;
    const uint8_t first = p[0];
    int extra;
    uint64_t v;
    int shift;
    if (first == 0) {
        extra = 8;
        v = 0;
        shift = 0;
    } else {
        extra = __builtin_ctz(first);
        v = static_cast<uint64_t>(first) >> (extra + 1);
        shift = 7 - extra;
    }
    if (p + 1 + extra > end)
        return 0;
    for (int i = 0; i < extra; ++i) {
        v |= static_cast<uint64_t>(p[1 + i]) << shift;
        shift += 8;
    }
    value = v;
    return static_cast<size_t>(extra) + 1;
}

inline uint64_t load_u64(const uint8_t *p) {
    uint64_t v;
    std::memcpy(&v, p, 8);
    return v;
}

enum WeightFormat { kNone = 0, kVarint = 1, kZigzag = 2, kDouble = 3, kFloat = 4 };

struct Cursor {
    const uint8_t *base, *end;
    size_t off;
    uint64_t next_varint() {
        uint64_t v = 0;
        const size_t k = read_varint(base + off, end, v);
        if (!k)
            throw std::runtime_error("truncated list data");
        off += k;
        return v;
    }
    double next_weight(int fmt) {
        switch (fmt) {
        case kVarint:
            return static_cast<double>(next_varint());
        case kZigzag: {
            const uint64_t u = next_varint();
            return static_cast<double>(static_cast<int64_t>((u >> 1) ^ (~(u & 1) + 1)));
        }
        case kDouble: {
            if (base + off + 8 > end)
                throw std::runtime_error("truncated weights");
            double d;
            std::memcpy(&d, base + off, 8);
            off += 8;
            return d;
        }
        case kFloat: {
            if (base + off + 4 > end)
                throw std::runtime_error("truncated weights");
            float f;
            std::memcpy(&f, base + off, 4);
            off += 4;
            return f;
        }
        default:
            return 1.0;
        }
    }
};

} // namespace

extern "C" {

const char *nkgen_io_last_error(void) { return g_io_err.c_str(); }

void nkgen_graph_free(nkgen_graph *g) {
    if (!g)
        return;
    free(g->in_ptr);
    free(g->in_col);
    free(g->outdeg);
    free(g->w);
    free(g->wdeg);
    free(g->exists);
    std::memset(g, 0, sizeof(*g));
}

// Read-only mapping of a whole file (the reference maps it too,
// MemoryMappedFile.cpp).
struct MappedFile {
    const uint8_t *p = nullptr;
    size_t size = 0;
    int fd = -1;
    explicit MappedFile(const char *path) {
        fd = open(path, O_RDONLY);
        if (fd < 0)
            throw std::runtime_error(std::string("cannot open ") + path);
        struct stat st;
        if (fstat(fd, &st) != 0)
            throw std::runtime_error("stat failed");
        size = static_cast<size_t>(st.st_size);
        if (size) {
            void *m = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
            if (m == MAP_FAILED)
                throw std::runtime_error("mmap failed");
            p = static_cast<const uint8_t *>(m);
            madvise(m, size, MADV_WILLNEED);
        }
    }
    ~MappedFile() {
        if (p)
            munmap(const_cast<uint8_t *>(p), size);
        if (fd >= 0)
            close(fd);
    }
};

// Bytes of the varint at p (0 past end).
inline size_t varint_len(const uint8_t *p, const uint8_t *end) {
    if (p >= end)
        return 0;
    const size_t k = (p[0] == 0) ? 9 : static_cast<size_t>(__builtin_ctz(p[0])) + 1;
    return (p + k <= end) ? k : 0;
}

int nkgen_read_nkbg(const char *path, int nthreads, nkgen_graph *out) {
    try {
        std::memset(out, 0, sizeof(*out));
        MappedFile mf(path);
        const uint8_t *b = mf.p, *end = mf.p + mf.size;
        if (mf.size < 80 || std::memcmp(b, "nkbg002", 8) != 0)
            throw std::runtime_error("not a NetworkitBinaryGraph file (magic nkbg002)");
        const uint64_t features = load_u64(b + 16), nodes = load_u64(b + 24),
                       chunks = load_u64(b + 32), off_base = load_u64(b + 40),
                       off_adj = load_u64(b + 48), off_tr = load_u64(b + 56),
                       off_w = load_u64(b + 64), off_wt = load_u64(b + 72);
        const int directed = static_cast<int>(features & 1u);
        const int fmt = static_cast<int>((features & 0xEu) >> 1);
        if (fmt > kFloat)
            throw std::runtime_error("unknown weight format");
        if (nodes >= 0xffffffffull)
            throw std::runtime_error("node ids must fit in 32 bits");
        if (nodes && chunks == 0)
            throw std::runtime_error("zero chunks");
        auto check_range = [&](uint64_t off, uint64_t len) {
            if (off > mf.size || len > mf.size - off)
                throw std::runtime_error("section outside the file");
        };
        check_range(off_base, nodes + (chunks ? chunks - 1 : 0) * 8);
        std::vector<uint64_t> first(chunks + 1, 0);
        for (uint64_t c = 1; c < chunks; ++c)
            first[c] = load_u64(b + off_base + nodes + (c - 1) * 8);
        first[chunks] = nodes;
        for (uint64_t c = 0; c < chunks; ++c)
            if (first[c] > first[c + 1])
                throw std::runtime_error("chunk boundaries out of order");
        const uint64_t hdr = chunks ? (chunks - 1) * 8 : 0;
        check_range(off_adj, hdr + 8);
        check_range(off_tr, hdr + 8);
        if (fmt != kNone) {
            check_range(off_w, hdr);
            check_range(off_wt, hdr);
        }
        auto chunk_off = [&](uint64_t sec, uint64_t c) -> uint64_t {
            return c ? load_u64(b + sec + (c - 1) * 8) : 0;
        };
        const size_t fixed_w = fmt == kDouble ? 8 : fmt == kFloat ? 4 : 0;
        if (nthreads > 0)
            omp_set_num_threads(nthreads);

        const uint64_t z = nodes;
        out->z = z;
        out->directed = directed;
        out->weighted = fmt != kNone;
        out->in_ptr = static_cast<uint64_t *>(malloc((z + 1) * sizeof(uint64_t)));
        out->outdeg = static_cast<uint32_t *>(malloc(std::max<uint64_t>(z, 1) * 4));
        out->wdeg = static_cast<double *>(malloc(std::max<uint64_t>(z, 1) * 8));
        out->exists = static_cast<uint8_t *>(malloc(std::max<uint64_t>(z, 1)));
        if (!out->in_ptr || !out->outdeg || !out->wdeg || !out->exists)
            throw std::bad_alloc();

        // Pass 1, per file chunk (the chunks are the format's only entry
        // points): row lengths (directed: the transpose count; undirected: the
        // adjacency count plus the transpose entries that are not
        // self-loops), the out-degrees, and where each node's lists and
        // weights start in the four streams. in_ptr[v + 1] holds the chunk's
        // running arc count until the chunk offsets are added.
        std::vector<uint64_t> pos_adj(z), pos_tr(z), pos_wa(fmt ? z : 0), pos_wt(fmt ? z : 0);
        std::vector<uint64_t> chunk_arcs(chunks + 1, 0);
        std::string err;
        auto skip_varints = [&](Cursor &cu, uint64_t n) {
            for (uint64_t j = 0; j < n; ++j) {
                const size_t k = varint_len(cu.base + cu.off, end);
                if (!k)
                    throw std::runtime_error("truncated list data");
                cu.off += k;
            }
        };
        auto skip_weights = [&](Cursor &cu, uint64_t n) {
            if (fmt == kVarint || fmt == kZigzag) {
                skip_varints(cu, n);
            } else if (fixed_w) {
                cu.off += n * fixed_w;
                if (cu.base + cu.off > end)
                    throw std::runtime_error("truncated weights");
            }
        };
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t ci = 0; ci < static_cast<int64_t>(chunks); ++ci) {
            try {
                const uint64_t c = static_cast<uint64_t>(ci);
                Cursor adj{b + off_adj, end, chunk_off(off_adj, c) + hdr + 8};
                Cursor tr{b + off_tr, end, chunk_off(off_tr, c) + hdr + 8};
                Cursor wa{b + off_w, end, fmt ? chunk_off(off_w, c) + hdr : 0};
                Cursor wt{b + off_wt, end, fmt ? chunk_off(off_wt, c) + hdr : 0};
                uint64_t sum = 0;
                for (uint64_t v = first[c]; v < first[c + 1]; ++v) {
                    pos_adj[v] = adj.off;
                    pos_tr[v] = tr.off;
                    if (fmt) {
                        pos_wa[v] = wa.off;
                        pos_wt[v] = wt.off;
                    }
                    const uint64_t n_out = adj.next_varint();
                    const uint64_t n_in = tr.next_varint();
                    uint64_t len;
                    skip_varints(adj, n_out);
                    if (directed) {
                        len = n_in;
                        skip_varints(tr, n_in);
                        out->outdeg[v] = static_cast<uint32_t>(n_out);
                    } else {
                        len = n_out;
                        for (uint64_t j = 0; j < n_in; ++j)
                            len += tr.next_varint() != v;
                        out->outdeg[v] = static_cast<uint32_t>(len);
                    }
                    if (fmt) {
                        skip_weights(wa, n_out);
                        skip_weights(wt, n_in);
                    }
                    sum += len;
                    out->in_ptr[v + 1] = sum;
                }
                chunk_arcs[c + 1] = sum;
            } catch (const std::exception &e) {
#pragma omp critical
                err = e.what();
            }
        }
        if (!err.empty())
            throw std::runtime_error(err);
        for (uint64_t c = 0; c < chunks; ++c)
            chunk_arcs[c + 1] += chunk_arcs[c];
        const uint64_t arcs = chunk_arcs[chunks];
        if (arcs >= 0xffffffffull)
            throw std::runtime_error("arc count must fit in 32 bits");
        out->arcs = arcs;
        out->in_ptr[0] = 0;
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t ci = 0; ci < static_cast<int64_t>(chunks); ++ci) {
            const uint64_t c = static_cast<uint64_t>(ci);
            for (uint64_t v = first[c]; v < first[c + 1]; ++v)
                out->in_ptr[v + 1] += chunk_arcs[c];
        }
        out->in_col = static_cast<uint32_t *>(malloc(std::max<uint64_t>(arcs, 1) * 4));
        if (!out->in_col)
            throw std::bad_alloc();
        if (fmt) {
            out->w = static_cast<double *>(malloc(std::max<uint64_t>(arcs, 1) * 8));
            if (!out->w)
                throw std::bad_alloc();
        }
        // Pass 2: node ranges of about equal arc counts (a power-law graph
        // puts most arcs in a few chunks), each decoded from its recorded
        // stream positions straight to its rows.
        const int threads = std::max(1, omp_get_max_threads());
        const uint64_t parts = std::min<uint64_t>(z, static_cast<uint64_t>(threads) * 16);
        std::vector<uint64_t> cut(parts + 1, z);
        cut[0] = 0;
        for (uint64_t k = 1; k < parts; ++k) {
            const uint64_t target = arcs / parts * k + (arcs % parts) * k / parts;
            cut[k] = static_cast<uint64_t>(
                std::upper_bound(out->in_ptr, out->in_ptr + z + 1, target) - out->in_ptr) - 1;
            cut[k] = std::max(cut[k], cut[k - 1]);
        }
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t pi = 0; pi < static_cast<int64_t>(parts); ++pi) {
            try {
                const uint64_t v0 = cut[pi], v1 = cut[pi + 1];
                if (v0 >= v1)
                    continue;
                Cursor adj{b + off_adj, end, pos_adj[v0]};
                Cursor tr{b + off_tr, end, pos_tr[v0]};
                Cursor wa{b + off_w, end, fmt ? pos_wa[v0] : 0};
                Cursor wt{b + off_wt, end, fmt ? pos_wt[v0] : 0};
                for (uint64_t v = v0; v < v1; ++v) {
                    // A node that starts a chunk: its streams start there.
                    adj.off = pos_adj[v];
                    tr.off = pos_tr[v];
                    if (fmt) {
                        wa.off = pos_wa[v];
                        wt.off = pos_wt[v];
                    }
                    out->exists[v] = b[off_base + v] & 1u;
                    const uint64_t row0 = out->in_ptr[v];
                    uint64_t pos = row0;
                    const uint64_t n_out = adj.next_varint();
                    const uint64_t n_in = tr.next_varint();
                    double osum = 0.0;
                    for (uint64_t j = 0; j < n_out; ++j) {
                        const uint64_t u = adj.next_varint();
                        if (u >= nodes)
                            throw std::runtime_error("neighbour id out of range");
                        const double w = fmt ? wa.next_weight(fmt) : 1.0;
                        osum += w;
                        if (!directed) {
                            out->in_col[pos] = static_cast<uint32_t>(u);
                            if (fmt)
                                out->w[pos] = w;
                            ++pos;
                        }
                    }
                    for (uint64_t j = 0; j < n_in; ++j) {
                        const uint64_t u = tr.next_varint();
                        if (u >= nodes)
                            throw std::runtime_error("neighbour id out of range");
                        const double w = fmt ? wt.next_weight(fmt) : 1.0;
                        if (!directed && u == v)
                            continue;  // a self-loop is stored once
                        out->in_col[pos] = static_cast<uint32_t>(u);
                        if (fmt)
                            out->w[pos] = w;
                        ++pos;
                    }
                    if (pos != out->in_ptr[v + 1])
                        throw std::runtime_error("inconsistent list lengths");
                    if (directed) {
                        out->wdeg[v] = fmt ? osum : static_cast<double>(n_out);
                    } else {
                        double sum = 0.0;
                        for (uint64_t k = row0; k < pos; ++k)
                            sum += fmt ? out->w[k] : 1.0;
                        out->wdeg[v] = sum;
                    }
                }
            } catch (const std::exception &e) {
#pragma omp critical
                err = e.what();
            }
        }
        if (!err.empty())
            throw std::runtime_error(err);
        return 0;
    } catch (const std::exception &e) {
        nkgen_graph_free(out);
        g_io_err = e.what();
        return -1;
    }
}

} // extern "C"

// ---------------------------------------------------------------------------
// Writer: NetworkitBinaryWriter(chunks, weights).write(G, path)
// (NetworkitBinaryWriter.cpp:21-380), byte for byte, from a graph given as
// its out-lists in outEdges order and, for directed graphs, its in-lists in
// inEdges order.

namespace {

inline size_t write_varint(uint64_t value, uint8_t *buf) {
    if (!value) {
        buf[0] = 1;
        return 1;
    }
    int extra;
    if (value >= (1ull << 56)) {
        buf[0] = 0;
        extra = 8;
    } else {
        const int bits = 64 - __builtin_clzll(value);
        extra = (bits - 1) / 7;
        buf[0] = static_cast<uint8_t>((1u << extra) | (value << (extra + 1)));
        value >>= 7 - extra;
    }
    for (int i = 0; i < extra; ++i) {
        buf[i + 1] = static_cast<uint8_t>(value & 0xff);
        value >>= 8;
    }
    return static_cast<size_t>(extra) + 1;
}

inline size_t varint_size(uint64_t value) {
    uint8_t tmp[10];
    return write_varint(value, tmp);
}

inline uint64_t zigzag(int64_t v) {
    return (static_cast<uint64_t>(v) << 1) ^ static_cast<uint64_t>(v < 0 ? -1 : 0);
}

// Encoded size / bytes of one weight in format fmt.
inline size_t weight_size(double w, int fmt) {
    switch (fmt) {
    case kVarint:
        return varint_size(static_cast<uint64_t>(w));
    case kZigzag:
        return varint_size(zigzag(static_cast<int64_t>(w)));
    case kDouble:
        return 8;
    case kFloat:
        return 4;
    default:
        return 0;
    }
}

inline size_t put_weight(double w, int fmt, uint8_t *p) {
    switch (fmt) {
    case kVarint:
        return write_varint(static_cast<uint64_t>(w), p);
    case kZigzag:
        return write_varint(zigzag(static_cast<int64_t>(w)), p);
    case kDouble:
        std::memcpy(p, &w, 8);
        return 8;
    case kFloat: {
        const float f = static_cast<float>(w);
        std::memcpy(p, &f, 4);
        return 4;
    }
    default:
        return 0;
    }
}

struct ListView {
    const uint64_t *ptr;
    const uint32_t *col;
    const double *w;
};

}  // namespace

extern "C" {

int nkgen_write_nkbg(const char *path, uint64_t n, int directed, const uint64_t *out_ptr,
                     const uint32_t *out_col, const double *out_w, const uint64_t *in_ptr,
                     const uint32_t *in_col, const double *in_w, uint64_t chunks, int weights,
                     int nthreads) {
    try {
        if (!path || !out_ptr || (out_ptr[n] && !out_col))
            throw std::runtime_error("NULL argument");
        if (n == 0)
            throw std::runtime_error("the format needs at least one node");
        if (directed && (!in_ptr || (in_ptr[n] && !in_col)))
            throw std::runtime_error("a directed graph needs its in-lists");
        if (weights < 0 || weights > 5)
            throw std::runtime_error("weights must be in 0..5");
        if (chunks == 0)
            throw std::runtime_error("chunks must be >= 1");
        const bool weighted = out_w != nullptr;
        if (weighted && directed && in_ptr[n] && !in_w)
            throw std::runtime_error("a weighted directed graph needs its in-list weights");
        if (nthreads > 0)
            omp_set_num_threads(nthreads);
        // The weight format: as given, or the narrowest that holds every edge
        // weight (forEdges: each undirected edge once, at its larger end).
        int fmt = kNone;
        switch (weights) {
        case 0: fmt = kNone; break;
        case 1: fmt = kVarint; break;
        case 2: fmt = kZigzag; break;
        case 3: fmt = kDouble; break;
        case 4: fmt = kFloat; break;
        default: {
            if (!weighted) {
                fmt = kNone;
                break;
            }
            bool is_unsigned = true, fits_int = true, fits_float = true;
            for (uint64_t u = 0; u < n; ++u)
                for (uint64_t k = out_ptr[u]; k < out_ptr[u + 1]; ++k) {
                    if (!directed && out_col[k] > u)
                        continue;
                    const double w = out_w[k];
                    if (w < 0)
                        is_unsigned = false;
                    if (w != static_cast<double>(static_cast<int64_t>(w)))
                        fits_int = false;
                    if (w != static_cast<double>(static_cast<float>(w)))
                        fits_float = false;
                }
            fmt = fits_int ? (is_unsigned ? kVarint : kZigzag) : (fits_float ? kFloat : kDouble);
        }
        }
        if (chunks > n)
            chunks = n;
        std::vector<uint64_t> first(chunks + 1);
        for (uint64_t c = 0; c < chunks; ++c)
            first[c] = c * (n / chunks);
        first[chunks] = n;
        // Lists: undirected graphs split each neighbour list into v <= u
        // (adjacency) and v >= u (transpose); directed graphs use out- and
        // in-lists as they are.
        const ListView outl{out_ptr, out_col, out_w};
        const ListView inl{directed ? in_ptr : out_ptr, directed ? in_col : out_col,
                           directed ? in_w : out_w};
        auto keep_adj = [&](uint64_t u, uint32_t v) { return directed || v <= u; };
        auto keep_tr = [&](uint64_t u, uint32_t v) { return directed || v >= u; };
        auto wt = [&](const ListView &l, uint64_t k) { return l.w ? l.w[k] : 1.0; };
        // Pass 1: bytes and list lengths per chunk.
        std::vector<uint64_t> adj_b(chunks), tr_b(chunks), adjw_b(chunks), trw_b(chunks),
            adj_n(chunks), tr_n(chunks);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t ci = 0; ci < static_cast<int64_t>(chunks); ++ci) {
            const uint64_t c = static_cast<uint64_t>(ci);
            uint64_t ab = 0, tb = 0, awb = 0, twb = 0, an = 0, tn = 0;
            for (uint64_t u = first[c]; u < first[c + 1]; ++u) {
                uint64_t cnt = 0;
                for (uint64_t k = outl.ptr[u]; k < outl.ptr[u + 1]; ++k)
                    if (keep_adj(u, outl.col[k])) {
                        ++cnt;
                        ab += varint_size(outl.col[k]);
                        awb += weight_size(wt(outl, k), fmt);
                    }
                ab += varint_size(cnt);
                an += cnt;
                cnt = 0;
                for (uint64_t k = inl.ptr[u]; k < inl.ptr[u + 1]; ++k)
                    if (keep_tr(u, inl.col[k])) {
                        ++cnt;
                        tb += varint_size(inl.col[k]);
                        twb += weight_size(wt(inl, k), fmt);
                    }
                tb += varint_size(cnt);
                tn += cnt;
            }
            adj_b[c] = ab, tr_b[c] = tb, adjw_b[c] = awb, trw_b[c] = twb, adj_n[c] = an,
            tr_n[c] = tn;
        }
        auto prefix = [&](const std::vector<uint64_t> &x) {
            std::vector<uint64_t> p(chunks + 1, 0);
            for (uint64_t c = 0; c < chunks; ++c)
                p[c + 1] = p[c] + x[c];
            return p;
        };
        const auto adj_o = prefix(adj_b), tr_o = prefix(tr_b), adjw_o = prefix(adjw_b),
                   trw_o = prefix(trw_b);
        uint64_t adj_total = 0, tr_total = 0;
        for (uint64_t c = 0; c < chunks; ++c)
            adj_total += adj_n[c], tr_total += tr_n[c];
        const uint64_t hdr = (chunks - 1) * 8;
        const uint64_t off_base = 80;
        const uint64_t off_adj = off_base + n + hdr;
        const uint64_t off_tr = off_adj + hdr + 8 + adj_o[chunks];
        const uint64_t off_w = off_tr + hdr + 8 + tr_o[chunks];
        const uint64_t off_wt = off_w + hdr + adjw_o[chunks];
        const uint64_t size = off_wt + hdr + trw_o[chunks];
        std::vector<uint8_t> buf(size, 0);
        uint8_t *b = buf.data();
        auto put64 = [&](uint64_t at, uint64_t v) { std::memcpy(b + at, &v, 8); };
        std::memcpy(b, "nkbg002", 8);
        put64(8, 0);
        put64(16, (directed ? 1u : 0u) | ((static_cast<uint64_t>(fmt) << 1) & 0xEu));
        put64(24, n);
        put64(32, chunks);
        put64(40, off_base);
        put64(48, off_adj);
        put64(56, off_tr);
        put64(64, fmt != kNone ? off_w : 0);
        put64(72, fmt != kNone ? off_wt : 0);
        std::memset(b + off_base, 1, n);  // every node exists
        for (uint64_t c = 1; c < chunks; ++c) {
            put64(off_base + n + (c - 1) * 8, first[c]);
            put64(off_adj + (c - 1) * 8, adj_o[c]);
            put64(off_tr + (c - 1) * 8, tr_o[c]);
            put64(off_w + (c - 1) * 8, adjw_o[c]);
            put64(off_wt + (c - 1) * 8, trw_o[c]);
        }
        put64(off_adj + hdr, adj_total);
        put64(off_tr + hdr, tr_total);
        // Pass 2: the lists, each chunk at its offset.
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t ci = 0; ci < static_cast<int64_t>(chunks); ++ci) {
            const uint64_t c = static_cast<uint64_t>(ci);
            uint8_t *pa = b + off_adj + hdr + 8 + adj_o[c];
            uint8_t *pt = b + off_tr + hdr + 8 + tr_o[c];
            uint8_t *pw = b + off_w + hdr + adjw_o[c];
            uint8_t *ptw = b + off_wt + hdr + trw_o[c];
            for (uint64_t u = first[c]; u < first[c + 1]; ++u) {
                uint64_t cnt = 0;
                for (uint64_t k = outl.ptr[u]; k < outl.ptr[u + 1]; ++k)
                    cnt += keep_adj(u, outl.col[k]);
                pa += write_varint(cnt, pa);
                for (uint64_t k = outl.ptr[u]; k < outl.ptr[u + 1]; ++k)
                    if (keep_adj(u, outl.col[k])) {
                        pa += write_varint(outl.col[k], pa);
                        pw += put_weight(wt(outl, k), fmt, pw);
                    }
                cnt = 0;
                for (uint64_t k = inl.ptr[u]; k < inl.ptr[u + 1]; ++k)
                    cnt += keep_tr(u, inl.col[k]);
                pt += write_varint(cnt, pt);
                for (uint64_t k = inl.ptr[u]; k < inl.ptr[u + 1]; ++k)
                    if (keep_tr(u, inl.col[k])) {
                        pt += write_varint(inl.col[k], pt);
                        ptw += put_weight(wt(inl, k), fmt, ptw);
                    }
            }
        }
        std::ofstream f(path, std::ios::binary | std::ios::trunc);
        if (!f)
            throw std::runtime_error(std::string("cannot open ") + path);
        f.write(reinterpret_cast<const char *>(b), static_cast<std::streamsize>(size));
        if (!f)
            throw std::runtime_error("write failed");
        return 0;
    } catch (const std::exception &e) {
        g_io_err = e.what();
        return -1;
    }
}

}  // extern "C"
