// NetworkitBinaryGraph decoded on the device (nkg_graph_create_from_nkbg,
// nkg_nkbg_decode): NetworkitBinaryReader::read (NetworkitBinaryReader.cpp:
// 19-235) without a Graph, from the file's bytes in device memory straight to
// the in-CSR the PageRank upload takes.
//
// File layout (NetworkitBinaryGraph.hpp / NetworkitBinaryGraph.md): a header
// of ten 64-bit words (magic "nkbg002", checksum, features, nodes, chunks and
// the offsets of the base data, adjacency lists, transpose lists, adjacency
// weights, transpose weights); the base data = one flag byte per node (bit 0:
// the node exists) and the first node of chunks 1..; every list section = the
// (chunks - 1) chunk offsets, the list total, then per node its length and
// its entries as prefix-length varints (the trailing zero bits of the first
// byte count the extra bytes, a zero first byte means 8); weight sections =
// chunk offsets, then per list entry a varint, zigzag varint, double or float.
//
// The adjacency it yields is the reference reader's: directed graphs, row v =
// v's transpose list, weighted degree = the sum of v's out-list weights in
// list order; undirected graphs, row v = v's adjacency list, then its
// transpose list without self-loops, weighted degree = the row's sum in row
// order.
//
// A varint stream has a sequential structure twice over: where a varint
// starts depends on every earlier one, and which varints are list lengths
// depends on every earlier length. The decoder breaks the first with a scan:
// a varint is at most 9 bytes, so a 64-byte segment is a function of how many
// of its first bytes belong to a varint begun earlier (0..8) to how many of
// the next segment's do, plus how many varints start in it. Those 9-entry
// maps compose associatively, so one device scan over all segments gives each
// segment its entry offset and the global index of its first varint, and
// every segment then decodes its varints in parallel into one array. The
// second is a walk over that array: one CTA per file chunk (the format's own
// entry points) hops from length to length through a shared-memory window,
// one step per node. The rest (row lengths, offsets, the entries' places in
// the rows, weights, degrees) is scans and scatter/gather passes.
#include <cub/cub.cuh>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "graph.hpp"
#include "host.hpp"

namespace nkg {
namespace {

constexpr uint32_t kSeg = 64;            // bytes per scan segment
constexpr uint32_t kBad = 0xffffffffu;   // a decoded value that does not fit 32 bits

enum WeightFormat { kWNone = 0, kWVarint = 1, kWZigzag = 2, kWDouble = 3, kWFloat = 4 };

// Segment map: entry offset e (bytes of the segment that continue a varint
// begun before it) -> exit offset into the next segment and varints begun
// inside the segment.
struct SegMap {
    uint32_t cnt[9];
    uint8_t exit[9];
    uint8_t pad[3];
};

struct ComposeMaps {
    __host__ __device__ SegMap operator()(const SegMap &a, const SegMap &b) const {
        SegMap r;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const int m = a.exit[e];
            r.exit[e] = b.exit[m];
            r.cnt[e] = a.cnt[e] + b.cnt[m];
        }
        r.pad[0] = r.pad[1] = r.pad[2] = 0;
        return r;
    }
};

__host__ __device__ inline SegMap identity_map() {
    SegMap r;
    for (int e = 0; e < 9; ++e) {
        r.exit[e] = static_cast<uint8_t>(e);
        r.cnt[e] = 0;
    }
    r.pad[0] = r.pad[1] = r.pad[2] = 0;
    return r;
}

__host__ __device__ inline SegMap compose(const SegMap &a, const SegMap &b) {
    return ComposeMaps()(a, b);
}

// Exclusive scan of n segment maps (composition: earlier then later), in
// three launches: every block scans kScanItems consecutive maps (each thread
// composes kScanPer of them in order, the block combines the thread totals in
// shared memory), one thread scans the block totals, every map then takes its
// block's prefix. Reads and writes stay below n and below the block count.
constexpr int kScanThreads = 256;
constexpr int kScanPer = 8;
constexpr uint64_t kScanItems = static_cast<uint64_t>(kScanThreads) * kScanPer;

__global__ void __launch_bounds__(kScanThreads)
    maps_block_scan(const SegMap *__restrict__ in, uint64_t n, SegMap *__restrict__ out,
                    SegMap *__restrict__ block_total) {
    __shared__ SegMap sm[kScanThreads];
    const uint64_t b0 = static_cast<uint64_t>(blockIdx.x) * kScanItems;
    const uint64_t t0 = b0 + static_cast<uint64_t>(threadIdx.x) * kScanPer;
    SegMap acc = identity_map();
    for (int i = 0; i < kScanPer; ++i)
        if (t0 + i < n)
            acc = compose(acc, in[t0 + i]);
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {
        const SegMap mine = sm[threadIdx.x];
        SegMap v = mine;
        if (threadIdx.x >= off)
            v = compose(sm[threadIdx.x - off], mine);
        __syncthreads();
        sm[threadIdx.x] = v;
        __syncthreads();
    }
    // sm[t] is now the inclusive total of threads 0..t.
    SegMap run = threadIdx.x ? sm[threadIdx.x - 1] : identity_map();
    for (int i = 0; i < kScanPer; ++i)
        if (t0 + i < n) {
            out[t0 + i] = run;
            run = compose(run, in[t0 + i]);
        }
    if (threadIdx.x == kScanThreads - 1)
        block_total[blockIdx.x] = sm[kScanThreads - 1];
}

// Exclusive prefix of the block totals, in place: one block stages tiles of
// kScanThreads totals in shared memory, its first thread composes them in order.
__global__ void __launch_bounds__(kScanThreads) maps_total_scan(SegMap *__restrict__ total,
                                                               uint64_t blocks) {
    __shared__ SegMap tile[kScanThreads];
    SegMap run = identity_map();  // meaningful in thread 0
    for (uint64_t t0 = 0; t0 < blocks; t0 += kScanThreads) {
        const uint64_t b = t0 + threadIdx.x;
        if (b < blocks)
            tile[threadIdx.x] = total[b];
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint64_t m = blocks - t0 < kScanThreads ? blocks - t0 : kScanThreads;
            for (uint64_t i = 0; i < m; ++i) {
                const SegMap t = tile[i];
                tile[i] = run;
                run = compose(run, t);
            }
        }
        __syncthreads();
        if (b < blocks)
            total[b] = tile[threadIdx.x];
        __syncthreads();
    }
}

__global__ void maps_apply(SegMap *__restrict__ out, uint64_t n,
                           const SegMap *__restrict__ block_prefix) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        out[i] = compose(block_prefix[i / kScanItems], out[i]);
}

__device__ __forceinline__ uint32_t varint_bytes(uint8_t first) {
    return first == 0 ? 9u : static_cast<uint32_t>(__ffs(first));
}

// Bytes [begin, end) of the file hold one varint stream starting at begin.
__global__ void seg_maps(const uint8_t *__restrict__ file, uint64_t begin, uint64_t end,
                         uint64_t segs, SegMap *__restrict__ maps) {
    const uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (s >= segs)
        return;
    const uint64_t s0 = begin + s * kSeg;
    const uint64_t s1 = min(s0 + kSeg, end);
    SegMap m;
#pragma unroll 1
    for (int e = 0; e < 9; ++e) {
        uint64_t pos = s0 + e;
        uint32_t cnt = 0;
        while (pos < s1) {
            pos += varint_bytes(file[pos]);
            ++cnt;
        }
        m.cnt[e] = cnt;
        // A walk that leaves the last segment ends the stream: nothing follows.
        m.exit[e] = static_cast<uint8_t>(pos - s1 < 8 ? pos - s1 : 8);
    }
    m.pad[0] = m.pad[1] = m.pad[2] = 0;
    maps[s] = m;
}

__device__ __forceinline__ uint64_t read_varint(const uint8_t *__restrict__ file, uint64_t pos,
                                                uint64_t end, uint32_t &len, bool &ok) {
    const uint8_t first = file[pos];
    len = varint_bytes(first);
    ok = pos + len <= end;
    if (!ok)
        return 0;
    const uint32_t extra = len - 1;
    uint64_t v = first == 0 ? 0 : static_cast<uint64_t>(first) >> len;
    uint32_t shift = first == 0 ? 0 : 8 - len;
    for (uint32_t i = 0; i < extra; ++i) {
        v |= static_cast<uint64_t>(file[pos + 1 + i]) << shift;
        shift += 8;
    }
    return v;
}

// Decode every varint of the stream: value k of the stream to vals[k] (32-bit
// lists) or vals64[k] (varint weights). A varint cut off by the stream's end
// decodes to kBad.
__global__ void seg_decode(const uint8_t *__restrict__ file, uint64_t begin, uint64_t end,
                           uint64_t segs, const SegMap *__restrict__ prefix,
                           uint32_t *__restrict__ vals, uint64_t *__restrict__ vals64) {
    const uint64_t s = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (s >= segs)
        return;
    const uint64_t s0 = begin + s * kSeg;
    const uint64_t s1 = min(s0 + kSeg, end);
    const SegMap &p = prefix[s];
    uint64_t pos = s0 + p.exit[0];
    uint64_t k = p.cnt[0];
    while (pos < s1) {
        uint32_t len;
        bool ok;
        const uint64_t v = read_varint(file, pos, end, len, ok);
        if (vals)
            vals[k] = ok && v <= 0xfffffffeull ? static_cast<uint32_t>(v) : kBad;
        if (vals64)
            vals64[k] = ok ? v : ~0ull;
        pos += len;
        ++k;
    }
}

// The varint index of every chunk's first byte (chunk_pos, file offsets);
// err = 1 when one does not start a varint.
__global__ void chunk_index(const uint8_t *__restrict__ file, uint64_t begin,
                            const uint64_t *__restrict__ chunk_pos, uint32_t chunks,
                            const SegMap *__restrict__ prefix, uint64_t segs,
                            uint64_t *__restrict__ chunk_base, int *err) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= chunks)
        return;
    const uint64_t o = chunk_pos[c];
    const uint64_t s = (o - begin) / kSeg;
    if (s >= segs) {
        // Only an empty chunk may start at the stream's end.
        chunk_base[c] = prefix[segs - 1].cnt[0];  // patched by the host for empty chunks
        atomicExch(err, 1);
        return;
    }
    uint64_t pos = begin + s * kSeg + prefix[s].exit[0];
    uint64_t k = prefix[s].cnt[0];
    while (pos < o) {
        pos += varint_bytes(file[pos]);
        ++k;
    }
    if (pos != o)
        atomicExch(err, 1);
    chunk_base[c] = k;
}

// One CTA per chunk and list stream walks the chunk's list lengths: node
// first_c + j has its length at index hdr[first_c + j] of vals, the next length
// follows its entries. The walk reads vals through a shared-memory window that
// the whole CTA fills with 16-byte loads, and records the lengths' indices in a
// shared list that the whole CTA then writes out (hdr, and the is_hdr marks),
// so the walking thread's steps touch shared memory only. CTAs
// [0, chunks) walk stream 0, [chunks, 2 chunks) stream 1. err = 2 when a walk
// leaves the stream or a length does not fit.
constexpr uint32_t kWin = 24576;  // window and list: 2 x 96 KB of dynamic shared memory
constexpr int kWalkThreads = 256;

struct WalkStream {
    const uint32_t *vals;  // K values
    uint64_t K;
    const uint64_t *chunk_base;
    uint32_t *hdr;
    uint8_t *is_hdr;
    uint64_t *chunk_end;
};

__global__ void __launch_bounds__(kWalkThreads)
    walk_headers(WalkStream s0, WalkStream s1, uint32_t chunks, const uint64_t *__restrict__ first,
                 int *err) {
    extern __shared__ uint4 s_dyn4[];
    uint32_t *win = reinterpret_cast<uint32_t *>(s_dyn4);
    uint32_t *hl = win + kWin;
    __shared__ uint64_t s_h, s_j;
    __shared__ uint32_t s_cnt;
    __shared__ int s_bad;
    const WalkStream &S = blockIdx.x < chunks ? s0 : s1;
    const uint32_t c = blockIdx.x < chunks ? blockIdx.x : blockIdx.x - chunks;
    const uint64_t nodes = first[c + 1] - first[c];
    const uint64_t K = S.K;
    uint64_t h = S.chunk_base[c], j = 0;
    if (threadIdx.x == 0)
        s_bad = 0;
    __syncthreads();
    while (j < nodes) {
        const uint64_t ws = h & ~3ull;  // 16-byte aligned start (vals is 256-byte aligned)
        const uint4 *src = reinterpret_cast<const uint4 *>(S.vals + ws);
        uint4 *dst = reinterpret_cast<uint4 *>(win);
        if (ws + kWin <= K) {  // asynchronous 16-byte copies, all in flight at once
            const uint32_t d0 = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
            for (uint32_t i = threadIdx.x; i < kWin / 4; i += kWalkThreads)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d0 + 16 * i),
                             "l"(src + i)
                             : "memory");
            asm volatile("cp.async.wait_all;\n" ::: "memory");
        } else {
            for (uint32_t i = threadIdx.x; i < kWin / 4; i += kWalkThreads) {
                const uint64_t idx = ws + 4ull * i;  // entries at K and beyond read as kBad
                if (idx + 4 <= K) {
                    dst[i] = src[i];
                } else {
                    uint32_t *d = win + 4 * i;
                    for (uint32_t e = 0; e < 4; ++e)
                        d[e] = idx + e < K ? S.vals[idx + e] : kBad;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            // The walk keeps 32-bit offsets into the window; a step is clamped
            // to 2^31, which leaves the window, and the exact position after
            // the last list is worked out once from that list's length. A
            // length of kBad (an entry at K or beyond) puts it past K, so one
            // test catches that and any list that ends past K.
            const uint32_t lim = nodes - j < kWin ? static_cast<uint32_t>(nodes - j) : kWin;
            uint32_t p = static_cast<uint32_t>(h - ws), cnt = 0;
            while (cnt < lim && p < kWin) {
                const uint32_t len = win[p];
                hl[cnt++] = p;
                p += 1u + (len < 0x7fffffffu ? len : 0x7fffffffu);
            }
            const uint32_t last = hl[cnt - 1];  // cnt >= 1: the first step starts inside
            const uint64_t hh = ws + last + 1 + static_cast<uint64_t>(win[last]);
            const bool bad = hh > K;
            if (bad)
                s_bad = 1;
            s_h = hh;
            s_j = bad ? nodes : j + cnt;
            s_cnt = bad ? 0 : cnt;  // a failed walk writes nothing
        }
        __syncthreads();
        const uint32_t cnt = s_cnt;
        const uint64_t out0 = first[c] + j;
        for (uint32_t i = threadIdx.x; i < cnt; i += kWalkThreads) {
            const uint32_t hi = static_cast<uint32_t>(ws + hl[i]);
            S.hdr[out0 + i] = hi;
            S.is_hdr[hi] = 1;
        }
        h = s_h;
        j = s_j;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        S.chunk_end[c] = h;
        if (s_bad)
            atomicExch(err, 2);
    }
}

// Per node: out-degree count, row length and (undirected) self-loops of the
// transpose list. Directed: row = transpose list. Undirected: row = the
// adjacency list, then the transpose list without self-loops.
__global__ void node_lengths(const uint32_t *__restrict__ va, const uint32_t *__restrict__ vt,
                             const uint32_t *__restrict__ ha, const uint32_t *__restrict__ ht,
                             const uint32_t *__restrict__ keep_t, uint64_t z, int directed,
                             uint64_t *__restrict__ rowlen, uint32_t *__restrict__ outdeg) {
    const uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (v >= z)
        return;
    const uint32_t n_out = va[ha[v]], n_in = vt[ht[v]];
    if (directed) {
        rowlen[v] = n_in;
        outdeg[v] = n_out;
    } else {
        // keep_t is the inclusive prefix of kept transpose entries.
        const uint32_t kept = keep_t[ht[v] + n_in] - keep_t[ht[v]];
        rowlen[v] = static_cast<uint64_t>(n_out) + kept;
        outdeg[v] = n_out + kept;
    }
}

// Which chunk varint k of a stream lies in, or -1 outside every chunk's lists.
__device__ __forceinline__ int chunk_of(uint64_t k, const uint64_t *__restrict__ base,
                                        const uint64_t *__restrict__ cend, uint32_t chunks) {
    uint32_t lo = 0, hi = chunks;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (base[mid] <= k)
            lo = mid;
        else
            hi = mid;
    }
    return k >= base[lo] && k < cend[lo] ? static_cast<int>(lo) : -1;
}

// keep[k] = 1 for a transpose-list entry whose value is not its own node
// (the entries an undirected row takes), 0 for lengths, self-loops and bytes
// outside the chunks. hcount is the inclusive prefix of is_hdr.
__global__ void keep_flags(const uint32_t *__restrict__ vt, const uint8_t *__restrict__ is_hdr,
                           const uint32_t *__restrict__ hcount, uint64_t K,
                           const uint64_t *__restrict__ base, const uint64_t *__restrict__ cend,
                           const uint64_t *__restrict__ first, uint32_t chunks,
                           uint32_t *__restrict__ keep) {
    const uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (k >= K)
        return;
    uint32_t f = 0;
    if (!is_hdr[k]) {
        const int c = chunk_of(k, base, cend, chunks);
        if (c >= 0) {
            const uint64_t before = base[c] ? hcount[base[c] - 1] : 0;
            const uint64_t node = first[c] + (hcount[k] - before) - 1;
            f = vt[k] != node ? 1u : 0u;
        }
    }
    keep[k] = f;
}

// Scatter the list entries of one stream to their row positions (and their
// weights): entry k of node v, j-th of v's list, goes to
// row_ptr[v] + offset + j (adjacency lists, or directed transpose lists) or,
// for undirected transpose lists, to row_ptr[v] + n_out(v) + its rank among
// v's kept entries. Weight of the entry: its index among the chunk's entries
// in the chunk's weight stream.
struct Scatter {
    const uint32_t *vals;
    const uint8_t *is_hdr;
    const uint32_t *hcount;
    uint64_t K;
    const uint64_t *base, *cend, *first;
    uint32_t chunks;
    const uint32_t *hdr;        // per node: index of its length
    const uint32_t *keep;       // undirected transpose: inclusive prefix of kept entries
    const uint32_t *n_out_from; // undirected transpose: adjacency vals / headers for n_out
    const uint32_t *hdr_out;
    const uint64_t *row_ptr;
    int mode;                   // 0: row starts at row_ptr[v]; 1: after n_out, kept only
    uint64_t z;
    // weights
    int wfmt;
    const uint8_t *file;
    const uint64_t *wchunk_pos;  // byte offset of chunk c's weights (fixed formats)
    const uint64_t *wvals;       // decoded varint weights (varint formats)
    const uint64_t *wbase;       // index of chunk c's first weight in wvals
    uint64_t wK;                 // decoded varint weights
    uint32_t *col;
    double *w;
    int *err;
};

__device__ __forceinline__ double weight_of(const Scatter &a, int c, uint64_t e) {
    if ((a.wfmt == kWVarint || a.wfmt == kWZigzag) && a.wbase[c] + e >= a.wK) {
        atomicExch(a.err, 4);  // the weight section ends early
        return 0.0;
    }
    switch (a.wfmt) {
    case kWVarint:
        return static_cast<double>(a.wvals[a.wbase[c] + e]);
    case kWZigzag: {
        const uint64_t u = a.wvals[a.wbase[c] + e];
        return static_cast<double>(static_cast<int64_t>((u >> 1) ^ (~(u & 1) + 1)));
    }
    case kWDouble: {
        double d;
        memcpy(&d, a.file + a.wchunk_pos[c] + 8 * e, 8);
        return d;
    }
    case kWFloat: {
        float f;
        memcpy(&f, a.file + a.wchunk_pos[c] + 4 * e, 4);
        return static_cast<double>(f);
    }
    default:
        return 1.0;
    }
}

__global__ void scatter_entries(Scatter a) {
    const uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (k >= a.K || a.is_hdr[k])
        return;
    const int c = chunk_of(k, a.base, a.cend, a.chunks);
    if (c < 0)
        return;
    const uint64_t before = a.base[c] ? a.hcount[a.base[c] - 1] : 0;
    const uint64_t hc = a.hcount[k] - before;  // lengths of the chunk up to k
    const uint64_t v = a.first[c] + hc - 1;
    const uint32_t val = a.vals[k];
    if (val >= a.z) {
        atomicExch(a.err, 3);
        return;
    }
    const uint64_t j = k - a.hdr[v] - 1;       // place in v's list
    const uint64_t e = (k - a.base[c]) - hc;   // place among the chunk's entries
    uint64_t pos;
    if (a.mode == 0) {
        pos = a.row_ptr[v] + j;
    } else {
        if (val == v)
            return;  // a self-loop is stored once, from the adjacency list
        const uint32_t n_out = a.n_out_from[a.hdr_out[v]];
        pos = a.row_ptr[v] + n_out + (a.keep[k] - a.keep[a.hdr[v]]) - 1;
    }
    a.col[pos] = val;
    if (a.w)
        a.w[pos] = weight_of(a, c, e);
}

// Every list entry of a stream (not a length, inside a chunk's lists) must be
// a node id < z (the adjacency lists of a directed graph, which no row takes).
__global__ void check_ids(const uint32_t *__restrict__ vals, const uint8_t *__restrict__ is_hdr,
                          uint64_t K, const uint64_t *__restrict__ base,
                          const uint64_t *__restrict__ cend, uint32_t chunks, uint64_t z,
                          int *err) {
    const uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (k >= K || is_hdr[k] || vals[k] < z)
        return;
    if (chunk_of(k, base, cend, chunks) >= 0)
        atomicExch(err, 3);
}

__global__ void widen_flags(const uint8_t *__restrict__ f, uint64_t K, uint32_t *__restrict__ out) {
    const uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (k < K)
        out[k] = f[k];
}

// Directed: weighted degree = the out-list weights of v in list order.
__global__ void out_weight_sums(Scatter a, const uint32_t *__restrict__ ha, uint64_t z,
                                const uint64_t *__restrict__ node_chunk_base,
                                double *__restrict__ wdeg) {
    const uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (v >= z)
        return;
    // Chunk of v by its first node.
    uint32_t lo = 0, hi = a.chunks;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.first[mid] <= v)
            lo = mid;
        else
            hi = mid;
    }
    const uint64_t h = ha[v];
    const uint32_t n = a.vals[h];
    // Entries of the chunk before v's list: (h + 1 - base) minus the lengths
    // up to and including v's.
    const uint64_t e0 = (h + 1 - a.base[lo]) - (v - a.first[lo] + 1);
    double sum = 0.0;
    for (uint32_t j = 0; j < n; ++j)
        sum += weight_of(a, static_cast<int>(lo), e0 + j);
    wdeg[v] = sum;
    (void)node_chunk_base;
}

// Undirected: weighted degree = the row's weights in row order.
__global__ void row_weight_sums(const uint64_t *__restrict__ row_ptr, const double *__restrict__ w,
                                uint64_t z, double *__restrict__ wdeg) {
    const uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (v >= z)
        return;
    double sum = 0.0;
    for (uint64_t k = row_ptr[v]; k < row_ptr[v + 1]; ++k)
        sum += w[k];
    wdeg[v] = sum;
}

__global__ void count_degrees(const uint32_t *__restrict__ outdeg, const uint64_t *__restrict__ rowlen,
                              uint64_t z, int directed, double *__restrict__ wdeg) {
    const uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (v < z)
        wdeg[v] = directed ? static_cast<double>(outdeg[v]) : static_cast<double>(rowlen[v]);
}

__global__ void node_flags(const uint8_t *__restrict__ base, uint64_t z, uint8_t *__restrict__ ex,
                           unsigned long long *__restrict__ missing) {
    const uint64_t v = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (v >= z)
        return;
    const uint8_t f = base[v] & 1u;
    ex[v] = f;
    if (!f)
        atomicAdd(missing, 1ull);
}

inline uint64_t load_u64(const uint8_t *p) {
    uint64_t v;
    std::memcpy(&v, p, 8);
    return v;
}

template <typename T>
void inclusive_scan(const T *in, T *out, uint64_t n, cudaStream_t s) {
    size_t tb = 0;
    NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, in, out, static_cast<int64_t>(n), s));
    DeviceArray<unsigned char> tmp(std::max<size_t>(tb, 1));
    NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb, in, out, static_cast<int64_t>(n), s));
}

// One varint stream of the file decoded on the device.
struct Stream {
    uint64_t begin = 0, end = 0, segs = 0, K = 0;
    DeviceArray<SegMap> prefix;
    DeviceArray<uint32_t> vals;
    DeviceArray<uint64_t> vals64;
    DeviceArray<uint64_t> chunk_base;  // varint index of each chunk's first byte
};

void decode_stream(const uint8_t *d_file, uint64_t begin, uint64_t end,
                   const std::vector<uint64_t> &chunk_pos, bool wide, Stream &S, int *d_err,
                   cudaStream_t s) {
    S.begin = begin;
    S.end = end;
    S.segs = end > begin ? (end - begin + kSeg - 1) / kSeg : 0;
    const uint32_t chunks = static_cast<uint32_t>(chunk_pos.size());
    S.chunk_base.alloc(std::max<uint32_t>(chunks, 1));
    if (S.segs == 0) {
        S.K = 0;
        NKG_CUDA(cudaMemsetAsync(S.chunk_base.get(), 0, chunks * sizeof(uint64_t), s));
        return;
    }
    DeviceArray<SegMap> maps(S.segs);
    S.prefix.alloc(S.segs);
    seg_maps<<<ceil_div(S.segs, 256), 256, 0, s>>>(d_file, begin, end, S.segs, maps.get());
    NKG_CUDA(cudaGetLastError());
    const uint64_t blocks = (S.segs + kScanItems - 1) / kScanItems;
    DeviceArray<SegMap> totals(blocks);
    maps_block_scan<<<static_cast<unsigned>(blocks), kScanThreads, 0, s>>>(
        maps.get(), S.segs, S.prefix.get(), totals.get());
    maps_total_scan<<<1, kScanThreads, 0, s>>>(totals.get(), blocks);
    maps_apply<<<ceil_div(S.segs, 256), 256, 0, s>>>(S.prefix.get(), S.segs, totals.get());
    NKG_CUDA(cudaGetLastError());
    SegMap last, lastp;
    NKG_CUDA(cudaMemcpyAsync(&last, maps.get() + S.segs - 1, sizeof(SegMap),
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaMemcpyAsync(&lastp, S.prefix.get() + S.segs - 1, sizeof(SegMap),
                             cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    S.K = static_cast<uint64_t>(lastp.cnt[0]) + last.cnt[lastp.exit[0]];
    if (wide)
        S.vals64.alloc(std::max<uint64_t>(S.K, 1));
    else
        S.vals.alloc(std::max<uint64_t>(S.K, 1) + 1);
    seg_decode<<<ceil_div(S.segs, 256), 256, 0, s>>>(d_file, begin, end, S.segs, S.prefix.get(),
                                                     wide ? nullptr : S.vals.get(),
                                                     wide ? S.vals64.get() : nullptr);
    NKG_CUDA(cudaGetLastError());
    if (!wide)  // one sentinel past the last value
        NKG_CUDA(cudaMemsetAsync(S.vals.get() + S.K, 0xff, sizeof(uint32_t), s));
    DeviceArray<uint64_t> d_pos(std::max<uint32_t>(chunks, 1));
    // Empty trailing chunks may start at the stream's end: their base is K.
    std::vector<uint64_t> pos = chunk_pos;
    std::vector<int> at_end(chunks, 0);
    for (uint32_t c = 0; c < chunks; ++c)
        if (pos[c] >= end) {
            at_end[c] = 1;
            pos[c] = begin;
        }
    NKG_CUDA(cudaMemcpyAsync(d_pos.get(), pos.data(), chunks * sizeof(uint64_t),
                             cudaMemcpyHostToDevice, s));
    chunk_index<<<ceil_div(chunks, 64), 64, 0, s>>>(d_file, begin, d_pos.get(), chunks,
                                                   S.prefix.get(), S.segs, S.chunk_base.get(),
                                                   d_err);
    NKG_CUDA(cudaGetLastError());
    for (uint32_t c = 0; c < chunks; ++c)
        if (at_end[c])
            NKG_CUDA(cudaMemcpyAsync(S.chunk_base.get() + c, &S.K, sizeof(uint64_t),
                                     cudaMemcpyHostToDevice, s));
    NKG_CUDA(cudaStreamSynchronize(s));
}

// The decoded in-CSR in device memory.
struct DeviceCsr {
    uint64_t z = 0, arcs = 0;
    int directed = 0, weighted = 0;
    DeviceArray<uint64_t> ptr;
    DeviceArray<uint32_t> col, outdeg;
    DeviceArray<double> w, wdeg;
    DeviceArray<uint8_t> ex;
    std::vector<uint8_t> ex_host;  // filled when some node is absent
    double ms_decode = 0.0;
};

void decode_nkbg(const uint8_t *file_any, uint64_t size, bool on_device, int device,
                 cudaStream_t s, DeviceCsr &G) {
    require(file_any != nullptr, "file is NULL");
    require(size >= 80, "not a NetworkitBinaryGraph file (shorter than its header)");
    uint8_t hdr[80];
    NKG_CUDA(cudaMemcpy(hdr, file_any, 80, on_device ? cudaMemcpyDeviceToHost
                                                     : cudaMemcpyHostToHost));
    require(std::memcmp(hdr, "nkbg002", 8) == 0,
            "not a NetworkitBinaryGraph file (magic nkbg002)");
    const uint64_t features = load_u64(hdr + 16), nodes = load_u64(hdr + 24),
                   chunks = load_u64(hdr + 32), off_base = load_u64(hdr + 40),
                   off_adj = load_u64(hdr + 48), off_tr = load_u64(hdr + 56),
                   off_w = load_u64(hdr + 64), off_wt = load_u64(hdr + 72);
    const int directed = static_cast<int>(features & 1u);
    const int fmt = static_cast<int>((features & 0xEu) >> 1);
    require(fmt <= kWFloat, "unknown weight format");
    require(nodes >= 1 && nodes < 0xffffffffull, "node count must be in [1, 2^32 - 1)");
    require(chunks >= 1 && chunks <= nodes, "chunk count must be in [1, nodes]");
    auto check_range = [&](uint64_t off, uint64_t len) {
        require(off <= size && len <= size - off, "section outside the file");
    };
    const uint64_t hdr_b = (chunks - 1) * 8;
    check_range(off_base, nodes + hdr_b);
    check_range(off_adj, hdr_b + 8);
    check_range(off_tr, hdr_b + 8);
    if (fmt != kWNone) {
        check_range(off_w, hdr_b);
        check_range(off_wt, hdr_b);
    }
    // The file in device memory.
    DeviceArray<uint8_t> d_copy;
    const uint8_t *d_file = file_any;
    if (!on_device) {
        d_copy.alloc(size, 16);
        NKG_CUDA(cudaMemcpyAsync(d_copy.get(), file_any, size, cudaMemcpyHostToDevice, s));
        d_file = d_copy.get();
    }
    cudaEvent_t e0, e1;
    NKG_CUDA(cudaEventCreate(&e0));
    NKG_CUDA(cudaEventCreate(&e1));
    NKG_CUDA(cudaEventRecord(e0, s));
    // Chunk tables (small): first node of every chunk, chunk offsets per section.
    auto read_table = [&](uint64_t off, uint64_t count) {
        std::vector<uint64_t> v(count);
        if (count)
            NKG_CUDA(cudaMemcpyAsync(v.data(), d_file + off, count * 8, cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        return v;
    };
    std::vector<uint64_t> first(chunks + 1, 0);
    {
        const std::vector<uint64_t> t = read_table(off_base + nodes, chunks - 1);
        for (uint64_t c = 1; c < chunks; ++c)
            first[c] = t[c - 1];
        first[chunks] = nodes;
        for (uint64_t c = 0; c < chunks; ++c)
            require(first[c] <= first[c + 1], "chunk boundaries out of order");
    }
    // Where each section's data may end: the next section's start, else the file's end.
    // (the writer lays out the weight offset tables even without weights).
    std::vector<uint64_t> starts = {off_base, off_adj, off_tr, off_w, off_wt, size};
    auto section_end = [&](uint64_t off) {
        uint64_t e = size;
        for (uint64_t x : starts)
            if (x > off && x < e)
                e = x;
        return e;
    };
    auto chunk_positions = [&](uint64_t sec, uint64_t data_skip) {
        const std::vector<uint64_t> t = read_table(sec, chunks - 1);
        std::vector<uint64_t> pos(chunks);
        for (uint64_t c = 0; c < chunks; ++c) {
            const uint64_t rel = c ? t[c - 1] : 0;
            require(rel <= size, "chunk offset outside the file");
            pos[c] = sec + rel + hdr_b + data_skip;
        }
        return pos;
    };
    const std::vector<uint64_t> pos_a = chunk_positions(off_adj, 8), pos_t = chunk_positions(off_tr, 8);
    DeviceArray<int> d_err(1);
    NKG_CUDA(cudaMemsetAsync(d_err.get(), 0, sizeof(int), s));
    Stream A, T;
    decode_stream(d_file, pos_a[0], section_end(off_adj), pos_a, false, A, d_err.get(), s);
    decode_stream(d_file, pos_t[0], section_end(off_tr), pos_t, false, T, d_err.get(), s);
    require(read_scalar(d_err.get(), s) == 0, "a chunk does not start at a list length");
    const uint64_t z = nodes;
    require(A.K < 0xffffffffull && T.K < 0xffffffffull, "list sections of 2^32 varints or more");
    // Walk the lengths.
    DeviceArray<uint64_t> d_first(chunks + 1), cend_a(chunks), cend_t(chunks);
    NKG_CUDA(cudaMemcpyAsync(d_first.get(), first.data(), (chunks + 1) * 8, cudaMemcpyHostToDevice,
                             s));
    DeviceArray<uint32_t> ha(z), ht(z);
    DeviceArray<uint8_t> ia(std::max<uint64_t>(A.K, 1)), it(std::max<uint64_t>(T.K, 1));
    NKG_CUDA(cudaMemsetAsync(ia.get(), 0, std::max<uint64_t>(A.K, 1), s));
    NKG_CUDA(cudaMemsetAsync(it.get(), 0, std::max<uint64_t>(T.K, 1), s));
    {
        const size_t smem = 2 * kWin * sizeof(uint32_t);
        NKG_CUDA(cudaFuncSetAttribute(walk_headers, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(smem)));
        const WalkStream wa{A.vals.get(), A.K, A.chunk_base.get(), ha.get(), ia.get(),
                            cend_a.get()};
        const WalkStream wt{T.vals.get(), T.K, T.chunk_base.get(), ht.get(), it.get(),
                            cend_t.get()};
        walk_headers<<<2 * static_cast<unsigned>(chunks), kWalkThreads, smem, s>>>(
            wa, wt, static_cast<uint32_t>(chunks), d_first.get(), d_err.get());
    }
    NKG_CUDA(cudaGetLastError());
    require(read_scalar(d_err.get(), s) == 0, "truncated or inconsistent list data");
    // Inclusive prefixes of the length flags (as 32-bit counts).
    DeviceArray<uint32_t> hca(std::max<uint64_t>(A.K, 1)), hct(std::max<uint64_t>(T.K, 1));
    {
        DeviceArray<uint32_t> f32(std::max(A.K, T.K) + 1);
        auto widen = [&](const uint8_t *f, uint64_t K, uint32_t *out) {
            if (!K)
                return;
            widen_flags<<<ceil_div(K, 256), 256, 0, s>>>(f, K, f32.get());
            NKG_CUDA(cudaGetLastError());
            inclusive_scan(f32.get(), out, K, s);
        };
        widen(ia.get(), A.K, hca.get());
        widen(it.get(), T.K, hct.get());
    }
    // Kept transpose entries (undirected rows).
    DeviceArray<uint32_t> keep;
    if (!directed && T.K) {
        DeviceArray<uint32_t> flags(T.K);
        keep.alloc(T.K + 1);
        keep_flags<<<ceil_div(T.K, 256), 256, 0, s>>>(T.vals.get(), it.get(), hct.get(), T.K,
                                                      T.chunk_base.get(), cend_t.get(),
                                                      d_first.get(), static_cast<uint32_t>(chunks),
                                                      flags.get());
        NKG_CUDA(cudaGetLastError());
        inclusive_scan(flags.get(), keep.get(), T.K, s);
    }
    // Row lengths, out-degrees, offsets.
    DeviceArray<uint64_t> rowlen(z);
    G.outdeg.alloc(z);
    node_lengths<<<ceil_div(z, 256), 256, 0, s>>>(A.vals.get(), T.vals.get(), ha.get(), ht.get(),
                                                  keep.get(), z, directed, rowlen.get(),
                                                  G.outdeg.get());
    NKG_CUDA(cudaGetLastError());
    G.ptr.alloc(z + 1);
    NKG_CUDA(cudaMemsetAsync(G.ptr.get(), 0, sizeof(uint64_t), s));
    inclusive_scan(rowlen.get(), G.ptr.get() + 1, z, s);
    const uint64_t arcs = read_scalar(G.ptr.get() + z, s);
    require(arcs < 0xffffffffull, "arc count must fit in 32 bits");
    G.z = z;
    G.arcs = arcs;
    G.directed = directed;
    G.weighted = fmt != kWNone;
    G.col.alloc(std::max<uint64_t>(arcs, 1), 4);
    if (G.weighted)
        G.w.alloc(std::max<uint64_t>(arcs, 1), 4);
    G.wdeg.alloc(z);
    // Weight streams: fixed-size formats are read in place; varint formats
    // decode like the lists.
    Stream WA, WT;
    DeviceArray<uint64_t> wpos_a, wpos_t;
    if (G.weighted) {
        const std::vector<uint64_t> pa = chunk_positions(off_w, 0), pt = chunk_positions(off_wt, 0);
        wpos_a.alloc(chunks);
        wpos_t.alloc(chunks);
        NKG_CUDA(cudaMemcpyAsync(wpos_a.get(), pa.data(), chunks * 8, cudaMemcpyHostToDevice, s));
        NKG_CUDA(cudaMemcpyAsync(wpos_t.get(), pt.data(), chunks * 8, cudaMemcpyHostToDevice, s));
        if (fmt == kWVarint || fmt == kWZigzag) {
            decode_stream(d_file, pa[0], section_end(off_w), pa, true, WA, d_err.get(), s);
            decode_stream(d_file, pt[0], section_end(off_wt), pt, true, WT, d_err.get(), s);
            require(read_scalar(d_err.get(), s) == 0, "a weight chunk does not start at a weight");
        }
        // Fixed-size weights must lie inside the file: the last weight of
        // every chunk is checked through the chunk's entry count on the host.
    }
    auto make_scatter = [&](Stream &S, DeviceArray<uint8_t> &is, DeviceArray<uint32_t> &hc,
                            DeviceArray<uint64_t> &cend, DeviceArray<uint32_t> &h,
                            DeviceArray<uint64_t> &wpos, Stream &W) {
        Scatter a{};
        a.vals = S.vals.get();
        a.is_hdr = is.get();
        a.hcount = hc.get();
        a.K = S.K;
        a.base = S.chunk_base.get();
        a.cend = cend.get();
        a.first = d_first.get();
        a.chunks = static_cast<uint32_t>(chunks);
        a.hdr = h.get();
        a.row_ptr = G.ptr.get();
        a.z = z;
        a.wfmt = fmt;
        a.file = d_file;
        a.wchunk_pos = wpos.get();
        a.wvals = W.vals64.get();
        a.wbase = W.chunk_base.get();
        a.wK = W.K;
        a.col = G.col.get();
        a.w = G.weighted ? G.w.get() : nullptr;
        a.err = d_err.get();
        return a;
    };
    if (G.weighted && (fmt == kWDouble || fmt == kWFloat)) {
        // Bounds of the fixed-size weight streams: entries per chunk.
        std::vector<uint64_t> ba(chunks), ea(chunks), bt(chunks), et(chunks);
        NKG_CUDA(cudaMemcpyAsync(ba.data(), A.chunk_base.get(), chunks * 8, cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaMemcpyAsync(ea.data(), cend_a.get(), chunks * 8, cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaMemcpyAsync(bt.data(), T.chunk_base.get(), chunks * 8, cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaMemcpyAsync(et.data(), cend_t.get(), chunks * 8, cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        const uint64_t ws = fmt == kWDouble ? 8 : 4;
        const std::vector<uint64_t> pa = chunk_positions(off_w, 0), pt = chunk_positions(off_wt, 0);
        for (uint64_t c = 0; c < chunks; ++c) {
            const uint64_t nodes_c = first[c + 1] - first[c];
            check_range(pa[c], (ea[c] - ba[c] - nodes_c) * ws);
            check_range(pt[c], (et[c] - bt[c] - nodes_c) * ws);
        }
    }
    if (directed) {
        if (T.K) {
            Scatter a = make_scatter(T, it, hct, cend_t, ht, wpos_t, WT);
            a.mode = 0;
            scatter_entries<<<ceil_div(T.K, 256), 256, 0, s>>>(a);
        }
        // Adjacency entries are checked too (ids < nodes), and give the
        // weighted degrees.
        if (A.K)
            check_ids<<<ceil_div(A.K, 256), 256, 0, s>>>(A.vals.get(), ia.get(), A.K,
                                                         A.chunk_base.get(), cend_a.get(),
                                                         static_cast<uint32_t>(chunks), z,
                                                         d_err.get());
        Scatter b = make_scatter(A, ia, hca, cend_a, ha, wpos_a, WA);
        if (G.weighted) {
            out_weight_sums<<<ceil_div(z, 256), 256, 0, s>>>(b, ha.get(), z, nullptr,
                                                             G.wdeg.get());
        } else {
            count_degrees<<<ceil_div(z, 256), 256, 0, s>>>(G.outdeg.get(), rowlen.get(), z, 1,
                                                           G.wdeg.get());
        }
    } else {
        if (A.K) {
            Scatter a = make_scatter(A, ia, hca, cend_a, ha, wpos_a, WA);
            a.mode = 0;
            scatter_entries<<<ceil_div(A.K, 256), 256, 0, s>>>(a);
        }
        if (T.K) {
            Scatter b = make_scatter(T, it, hct, cend_t, ht, wpos_t, WT);
            b.mode = 1;
            b.keep = keep.get();
            b.n_out_from = A.vals.get();
            b.hdr_out = ha.get();
            scatter_entries<<<ceil_div(T.K, 256), 256, 0, s>>>(b);
        }
        if (G.weighted)
            row_weight_sums<<<ceil_div(z, 256), 256, 0, s>>>(G.ptr.get(), G.w.get(), z,
                                                              G.wdeg.get());
        else
            count_degrees<<<ceil_div(z, 256), 256, 0, s>>>(G.outdeg.get(), rowlen.get(), z, 0,
                                                           G.wdeg.get());
    }
    NKG_CUDA(cudaGetLastError());
    const int h_err = read_scalar(d_err.get(), s);
    require(h_err != 4, "truncated weights");
    require(h_err == 0, "neighbour id out of range");
    // Node flags.
    G.ex.alloc(z);
    DeviceArray<unsigned long long> missing(1);
    NKG_CUDA(cudaMemsetAsync(missing.get(), 0, sizeof(unsigned long long), s));
    node_flags<<<ceil_div(z, 256), 256, 0, s>>>(d_file + off_base, z, G.ex.get(), missing.get());
    NKG_CUDA(cudaGetLastError());
    NKG_CUDA(cudaEventRecord(e1, s));
    if (read_scalar(missing.get(), s)) {
        G.ex_host.resize(z);
        NKG_CUDA(cudaMemcpyAsync(G.ex_host.data(), G.ex.get(), z, cudaMemcpyDeviceToHost, s));
    }
    NKG_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    NKG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    G.ms_decode = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    (void)device;
}

int option_device_of(const nkg_graph_options *opt) {
    int dev = opt && opt->device >= 0 ? opt->device : -1;
    if (dev < 0)
        NKG_CUDA(cudaGetDevice(&dev));
    return dev;
}

// A graph handle from the file's bytes (host, or device with on_device):
// the decode, then the build nkg_graph_create does, on the handle's stream.
nkg_graph *create_from_nkbg(const void *file, uint64_t size, bool on_device,
                            const nkg_graph_options *opts, double *ms_decode_out) {
    DeviceGuard guard(option_device_of(opts));
    // Read the header first for the shell's z / kind.
    uint8_t hdr[80];
    require(file != nullptr && size >= 80, "not a NetworkitBinaryGraph file");
    NKG_CUDA(cudaMemcpy(hdr, file, 80,
                        on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
    const uint64_t features = load_u64(hdr + 16), nodes = load_u64(hdr + 24);
    require(std::memcmp(hdr, "nkbg002", 8) == 0, "not a NetworkitBinaryGraph file (magic nkbg002)");
    std::unique_ptr<nkg_graph> g = device_graph_shell(
        opts, nodes, ((features & 0xEu) >> 1) != 0, static_cast<int>(features & 1u));
    DeviceCsr G;
    decode_nkbg(static_cast<const uint8_t *>(file), size, on_device, g->device, g->stream, G);
    if (ms_decode_out)
        *ms_decode_out = G.ms_decode;
    // As nkg_graph_create takes them: weights and weighted degrees for
    // weighted graphs only, the existence mask only when a node is absent.
    DeviceArray<uint8_t> ex;
    if (!G.ex_host.empty())
        ex = std::move(G.ex);
    DeviceArray<double> w, wdeg;
    if (G.weighted) {
        w = std::move(G.w);
        wdeg = std::move(G.wdeg);
    }
    return device_graph_build(std::move(g), G.arcs, G.ptr, G.col, w, wdeg, ex,
                              G.ex_host.empty() ? nullptr : G.ex_host.data(), opts);
}

// The file at `path` into device memory (d_file, size bytes plus 16 of
// padding): reader threads pread it in pieces of `piece` bytes into their own
// two page-locked staging blocks, each thread on its own stream, so that the
// reads, the copies over PCIe and the other threads' work overlap; a staging
// block is refilled once the copy out of it has finished. Returns the size.
uint64_t load_file_to_device(const char *path, uint64_t piece, int dev,
                             DeviceArray<uint8_t> &d_file) {
    require(path != nullptr, "path is NULL");
    const int fd = open(path, O_RDONLY);
    if (fd < 0)
        throw Error(NKG_ERR_INVALID_ARG, std::string("cannot open ") + path + ": " +
                                             std::strerror(errno));
    struct FdGuard {
        int fd;
        ~FdGuard() { close(fd); }
    } fg{fd};
    struct stat st;
    require(fstat(fd, &st) == 0 && S_ISREG(st.st_mode), "not a regular file");
    const uint64_t size = static_cast<uint64_t>(st.st_size);
    require(size >= 80, "not a NetworkitBinaryGraph file");
    if (piece == 0)
        piece = 16ull << 20;
    const uint64_t pieces = (size + piece - 1) / piece;
    d_file.alloc(size, 16);
    uint8_t *dst = d_file.get();
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int threads =
        static_cast<int>(std::min<uint64_t>(pieces, std::min<unsigned>(8u, std::max(1u, hw / 2))));
    std::vector<std::string> errs(threads);
    auto reader = [&](int t) {
        cudaStream_t s = nullptr;
        void *slot[2] = {nullptr, nullptr};
        cudaEvent_t ev[2] = {nullptr, nullptr};
        try {
            NKG_CUDA(cudaSetDevice(dev));
            s = stream_acquire(dev);
            for (int k = 0; k < 2; ++k) {
                slot[k] = pinned_alloc(piece);
                NKG_CUDA(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
            }
            bool used[2] = {false, false};
            int k = 0;
            for (uint64_t c = t; c < pieces; c += threads, k ^= 1) {
                if (used[k])
                    NKG_CUDA(cudaEventSynchronize(ev[k]));
                const uint64_t off = c * piece, len = std::min(piece, size - off);
                uint64_t got = 0;
                while (got < len) {
                    const ssize_t r = pread(fd, static_cast<uint8_t *>(slot[k]) + got, len - got,
                                            static_cast<off_t>(off + got));
                    if (r < 0 && errno == EINTR)
                        continue;
                    require(r > 0, "the file could not be read to its end");
                    got += static_cast<uint64_t>(r);
                }
                NKG_CUDA(cudaMemcpyAsync(dst + off, slot[k], len, cudaMemcpyHostToDevice, s));
                NKG_CUDA(cudaEventRecord(ev[k], s));
                used[k] = true;
            }
            NKG_CUDA(cudaStreamSynchronize(s));
        } catch (const std::exception &e) {
            errs[t] = e.what();
            if (s)
                cudaStreamSynchronize(s);
        }
        for (int k = 0; k < 2; ++k) {
            if (ev[k])
                cudaEventDestroy(ev[k]);
            pinned_free(slot[k], piece);
        }
        stream_release(dev, s);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t)
        pool.emplace_back(reader, t);
    reader(0);
    for (auto &th : pool)
        th.join();
    for (const std::string &e : errs)
        if (!e.empty())
            throw Error(NKG_ERR_INVALID_ARG, e);
    return size;
}

} // namespace
} // namespace nkg

extern "C" {

int nkg_graph_create_from_nkbg_file(nkg_graph **out, const char *path, uint64_t staging_bytes,
                                    const nkg_graph_options *opts, double *ms_decode_out,
                                    double *s_load_out) {
    using namespace nkg;
    return guarded([&] {
        require(out != nullptr, "out is NULL");
        *out = nullptr;
        const int dev = option_device_of(opts);
        DeviceGuard guard(dev);
        const auto t0 = std::chrono::steady_clock::now();
        DeviceArray<uint8_t> d_file;
        const uint64_t size = load_file_to_device(path, staging_bytes, dev, d_file);
        if (s_load_out)
            *s_load_out =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        *out = create_from_nkbg(d_file.get(), size, true, opts, ms_decode_out);
    });
}

int nkg_graph_create_from_nkbg(nkg_graph **out, const void *file, uint64_t size, int flags,
                               const nkg_graph_options *opts, double *ms_decode_out) {
    using namespace nkg;
    return guarded([&] {
        require(out != nullptr, "out is NULL");
        require((flags & ~NKG_DEVICE_PTRS) == 0, "unknown flags");
        *out = nullptr;
        *out = create_from_nkbg(file, size, (flags & NKG_DEVICE_PTRS) != 0, opts, ms_decode_out);
    });
}

int nkg_nkbg_decode(const void *file, uint64_t size, int flags, int device, uint64_t *z_out,
                    uint64_t *arcs_out, int *directed_out, int *weighted_out, uint64_t *in_ptr,
                    uint32_t *in_col, double *in_w, double *wdeg, uint32_t *outdeg,
                    uint8_t *exists, double *ms_decode_out) {
    using namespace nkg;
    return guarded([&] {
        require((flags & ~NKG_DEVICE_PTRS) == 0, "unknown flags");
        int dev = device;
        if (dev < 0)
            NKG_CUDA(cudaGetDevice(&dev));
        DeviceGuard guard(dev);
        cudaStream_t s = stream_acquire(dev);
        struct StreamGuard {
            int dev;
            cudaStream_t s;
            ~StreamGuard() { stream_release(dev, s); }
        } sg{dev, s};
        DeviceCsr G;
        decode_nkbg(static_cast<const uint8_t *>(file), size, (flags & NKG_DEVICE_PTRS) != 0, dev,
                    s, G);
        if (z_out)
            *z_out = G.z;
        if (arcs_out)
            *arcs_out = G.arcs;
        if (directed_out)
            *directed_out = G.directed;
        if (weighted_out)
            *weighted_out = G.weighted;
        if (ms_decode_out)
            *ms_decode_out = G.ms_decode;
        auto get = [&](void *dst, const void *src, size_t bytes) {
            if (dst && bytes)
                NKG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
        };
        get(in_ptr, G.ptr.get(), (G.z + 1) * sizeof(uint64_t));
        get(in_col, G.col.get(), G.arcs * sizeof(uint32_t));
        if (G.weighted)
            get(in_w, G.w.get(), G.arcs * sizeof(double));
        get(wdeg, G.wdeg.get(), G.z * sizeof(double));
        get(outdeg, G.outdeg.get(), G.z * sizeof(uint32_t));
        get(exists, G.ex.get(), G.z);
        NKG_CUDA(cudaStreamSynchronize(s));
    });
}

} // extern "C"
