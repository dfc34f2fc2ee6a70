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

#include <omp.h>

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

struct ChunkOut {
    std::vector<uint32_t> rowlen, col, outdeg;
    std::vector<double> w, wdeg;
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

int nkgen_read_nkbg(const char *path, int nthreads, nkgen_graph *out) {
    try {
        std::memset(out, 0, sizeof(*out));
        std::ifstream f(path, std::ios::binary | std::ios::ate);
        if (!f)
            throw std::runtime_error(std::string("cannot open ") + path);
        const std::streamsize size = f.tellg();
        f.seekg(0);
        std::vector<uint8_t> buf(static_cast<size_t>(size));
        if (size && !f.read(reinterpret_cast<char *>(buf.data()), size))
            throw std::runtime_error("read failed");
        const uint8_t *b = buf.data(), *end = b + buf.size();
        if (buf.size() < 80 || std::memcmp(b, "nkbg002", 8) != 0)
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
            if (off > buf.size() || len > buf.size() - off)
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

        if (nthreads > 0)
            omp_set_num_threads(nthreads);
        std::vector<ChunkOut> parts(chunks);
        std::string err;
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t ci = 0; ci < static_cast<int64_t>(chunks); ++ci) {
            try {
                const uint64_t c = static_cast<uint64_t>(ci);
                ChunkOut &o = parts[c];
                Cursor adj{b + off_adj, end, chunk_off(off_adj, c) + hdr + 8};
                Cursor tr{b + off_tr, end, chunk_off(off_tr, c) + hdr + 8};
                Cursor wa{b + off_w, end, fmt ? chunk_off(off_w, c) + hdr : 0};
                Cursor wt{b + off_wt, end, fmt ? chunk_off(off_wt, c) + hdr : 0};
                const uint64_t cnt = first[c + 1] - first[c];
                o.rowlen.resize(cnt);
                o.outdeg.resize(cnt);
                o.wdeg.resize(cnt);
                std::vector<uint32_t> tmp_col;
                std::vector<double> tmp_w;
                for (uint64_t i = 0; i < cnt; ++i) {
                    const uint64_t v = first[c] + i;
                    const uint64_t n_out = adj.next_varint();
                    const uint64_t n_in = tr.next_varint();
                    const size_t row0 = o.col.size();
                    double osum = 0.0;
                    // out list
                    tmp_col.clear();
                    tmp_w.clear();
                    for (uint64_t j = 0; j < n_out; ++j) {
                        const uint64_t u = adj.next_varint();
                        if (u >= nodes)
                            throw std::runtime_error("neighbour id out of range");
                        const double wt_ = fmt ? wa.next_weight(fmt) : 1.0;
                        osum += wt_;
                        tmp_col.push_back(static_cast<uint32_t>(u));
                        tmp_w.push_back(wt_);
                    }
                    if (!directed) {
                        o.col.insert(o.col.end(), tmp_col.begin(), tmp_col.end());
                        if (fmt)
                            o.w.insert(o.w.end(), tmp_w.begin(), tmp_w.end());
                    }
                    // transpose list
                    for (uint64_t j = 0; j < n_in; ++j) {
                        const uint64_t u = tr.next_varint();
                        if (u >= nodes)
                            throw std::runtime_error("neighbour id out of range");
                        const double wt_ = fmt ? wt.next_weight(fmt) : 1.0;
                        if (!directed && u == v)
                            continue;  // a self-loop is stored once
                        o.col.push_back(static_cast<uint32_t>(u));
                        if (fmt)
                            o.w.push_back(wt_);
                    }
                    const uint64_t len = o.col.size() - row0;
                    o.rowlen[i] = static_cast<uint32_t>(len);
                    if (directed) {
                        o.outdeg[i] = static_cast<uint32_t>(n_out);
                        o.wdeg[i] = fmt ? osum : static_cast<double>(n_out);
                    } else {
                        o.outdeg[i] = static_cast<uint32_t>(len);
                        double s = 0.0;
                        for (size_t k = row0; k < o.col.size(); ++k)
                            s += fmt ? o.w[k] : 1.0;
                        o.wdeg[i] = s;
                    }
                }
            } catch (const std::exception &e) {
#pragma omp critical
                err = e.what();
            }
        }
        if (!err.empty())
            throw std::runtime_error(err);

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
        std::vector<uint64_t> arc0(chunks + 1, 0);
        for (uint64_t c = 0; c < chunks; ++c)
            arc0[c + 1] = arc0[c] + parts[c].col.size();
        const uint64_t arcs = arc0[chunks];
        out->arcs = arcs;
        out->in_col = static_cast<uint32_t *>(malloc(std::max<uint64_t>(arcs, 1) * 4));
        if (!out->in_col)
            throw std::bad_alloc();
        if (fmt) {
            out->w = static_cast<double *>(malloc(std::max<uint64_t>(arcs, 1) * 8));
            if (!out->w)
                throw std::bad_alloc();
        }
        for (uint64_t v = 0; v < z; ++v)
            out->exists[v] = b[off_base + v] & 1u;
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t ci = 0; ci < static_cast<int64_t>(chunks); ++ci) {
            const uint64_t c = static_cast<uint64_t>(ci);
            const ChunkOut &o = parts[c];
            uint64_t pos = arc0[c];
            for (uint64_t i = 0; i < o.rowlen.size(); ++i) {
                const uint64_t v = first[c] + i;
                out->in_ptr[v] = pos;
                pos += o.rowlen[i];
                out->outdeg[v] = o.outdeg[i];
                out->wdeg[v] = o.wdeg[i];
            }
            std::copy(o.col.begin(), o.col.end(), out->in_col + arc0[c]);
            if (fmt)
                std::copy(o.w.begin(), o.w.end(), out->w + arc0[c]);
        }
        out->in_ptr[z] = arcs;
        return 0;
    } catch (const std::exception &e) {
        nkgen_graph_free(out);
        g_io_err = e.what();
        return -1;
    }
}

} // extern "C"
