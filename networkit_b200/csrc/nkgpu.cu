// libnkgpu: B200 PageRank behind the C ABI of include/nkgpu.h.
//
// Graph upload (nkg_graph_create*) relabels the nodes by in-degree,
// descending (stable), and builds the sliced layout of sweep.cuh; the arc
// order inside every row (the reference's summation order) is kept. Results
// are mapped back to the caller's ids on the way out.
#include <cub/cub.cuh>

#include <signal.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <unordered_map>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <type_traits>
#include <vector>

#include "graph.hpp"
#include "host.hpp"
#include "refine.cuh"

using namespace nkg;

namespace nkg {

static thread_local std::string g_last_error;
void set_last_error(const std::string &m) { g_last_error = m; }

namespace {

constexpr int kMaxDevices = 64;
std::unordered_map<void *, size_t> g_block_size;  // every block the cache handed out

// Freed blocks kept for reuse, per device, by size: an allocation takes the
// smallest cached block of at least its size and at most 1/8 larger, so a
// graph created and destroyed in a loop gets the same blocks back.
struct BlockCache {
    std::multimap<size_t, void *> free_blocks;
    size_t cached_bytes = 0;
};

std::mutex g_cache_mutex;
BlockCache g_cache[kMaxDevices];

void release_blocks(BlockCache &c) {
    for (auto &kv : c.free_blocks) {
        g_block_size.erase(kv.second);
        cudaFree(kv.second);
    }
    c.free_blocks.clear();
    c.cached_bytes = 0;
}

}  // namespace

void *device_alloc(size_t bytes, int &device) {
    NKG_CUDA(cudaGetDevice(&device));
    require(device >= 0 && device < kMaxDevices, "device ordinal out of range");
    {
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        BlockCache &c = g_cache[device];
        auto it = c.free_blocks.lower_bound(bytes);
        if (it != c.free_blocks.end() && it->first <= bytes + bytes / 8) {
            void *p = it->second;
            c.cached_bytes -= it->first;
            c.free_blocks.erase(it);
            return p;
        }
    }
    // Blocks carry their size in a side table so that a free files them
    // under the size they were allocated with.
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        release_blocks(g_cache[device]);
        e = cudaMalloc(&p, bytes);
    }
    NKG_CUDA(e);
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    g_block_size[p] = bytes;
    return p;
}

void device_free(void *p, int device) {
    if (!p)
        return;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device)
        cudaSetDevice(device);
    // As cudaFree: no work still in flight may use the block.
    cudaDeviceSynchronize();
    {
        std::lock_guard<std::mutex> lock(g_cache_mutex);
        auto it = g_block_size.find(p);
        if (it != g_block_size.end()) {
            g_cache[device].free_blocks.emplace(it->second, p);
            g_cache[device].cached_bytes += it->second;
        } else {
            cudaFree(p);
        }
    }
    if (prev != device && prev >= 0)
        cudaSetDevice(prev);
}

namespace {
std::mutex g_pinned_mutex;
std::multimap<size_t, void *> g_pinned_free;  // cached page-locked blocks by size
std::mutex g_stream_mutex;
std::vector<cudaStream_t> g_streams[kMaxDevices];  // idle streams per device
}  // namespace

void *pinned_alloc(size_t bytes) {
    bytes = std::max<size_t>(bytes, 1);
    {
        std::lock_guard<std::mutex> lock(g_pinned_mutex);
        auto it = g_pinned_free.lower_bound(bytes);
        if (it != g_pinned_free.end() && it->first <= 2 * bytes) {
            void *p = it->second;
            g_pinned_free.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    NKG_CUDA(cudaHostAlloc(&p, bytes, cudaHostAllocDefault));
    return p;
}

void pinned_free(void *p, size_t bytes) {
    if (!p)
        return;
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    g_pinned_free.emplace(std::max<size_t>(bytes, 1), p);
}

cudaStream_t stream_acquire(int device) {
    require(device >= 0 && device < kMaxDevices, "device ordinal out of range");
    {
        std::lock_guard<std::mutex> lock(g_stream_mutex);
        if (!g_streams[device].empty()) {
            cudaStream_t s = g_streams[device].back();
            g_streams[device].pop_back();
            return s;
        }
    }
    cudaStream_t s = nullptr;
    NKG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
}

void stream_release(int device, cudaStream_t s) {
    if (!s)
        return;
    if (cudaStreamSynchronize(s) != cudaSuccess) {  // a stream in a failed state is not kept
        cudaGetLastError();
        cudaStreamDestroy(s);
        return;
    }
    std::lock_guard<std::mutex> lock(g_stream_mutex);
    g_streams[device].push_back(s);
}

// ---------------------------------------------------------------------------
// Graph build kernels

// Checks the caller's CSR: monotone offsets, columns in range and pointing at
// existing nodes, deleted nodes without arcs. Sets *err on the first problem
// (1: offsets, 2: column range, 3: column to deleted node, 4: deleted node
// with in-arcs) and counts out-degrees.
__global__ void validate_and_count(const uint64_t *__restrict__ in_ptr,
                                   const uint32_t *__restrict__ in_col,
                                   const uint8_t *__restrict__ exists, uint64_t z, uint64_t arcs,
                                   uint32_t *__restrict__ outdeg, int *__restrict__ err) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < z;
         i += stride) {
        const uint64_t a = in_ptr[i], b = in_ptr[i + 1];
        if (b < a || b > arcs)
            atomicCAS(err, 0, 1);
        else if (exists && !exists[i] && b != a)
            atomicCAS(err, 0, 4);
    }
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < arcs;
         e += stride) {
        const uint32_t v = in_col[e];
        if (v >= z) {
            atomicCAS(err, 0, 2);
            continue;
        }
        if (exists && !exists[v]) {
            atomicCAS(err, 0, 3);
            continue;
        }
        atomicAdd(outdeg + v, 1u);
    }
}

// Sort key per original id: deleted nodes 0 (sorted last), existing nodes
// in-degree + 1, or with `bucketed` degree_bucket(in-degree) + 1 (the stable
// sort then keeps the caller's order inside a bucket). Counts sinks
// (existing, out-degree 0).
__global__ void make_keys(const uint64_t *__restrict__ in_ptr, const uint32_t *__restrict__ outdeg,
                          const uint8_t *__restrict__ exists, uint64_t z, int bucketed,
                          uint32_t *__restrict__ keys, uint32_t *__restrict__ ids,
                          unsigned long long *__restrict__ sinks) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    bool sink = false;
    if (i < z) {
        const bool ex = exists == nullptr || exists[i];
        const uint64_t d = in_ptr[i + 1] - in_ptr[i];
        const uint32_t k = bucketed ? degree_bucket(static_cast<uint32_t>(d))
                                    : static_cast<uint32_t>(d);
        keys[i] = ex ? k + 1 : 0u;
        ids[i] = static_cast<uint32_t>(i);
        sink = ex && outdeg[i] == 0;
    }
    const int c = __syncthreads_count(sink);
    if (threadIdx.x == 0 && c)
        atomicAdd(sinks, static_cast<unsigned long long>(c));
}

// Id locality of the caller's numbering: over `samples` arcs spread evenly
// across the CSR, how many join ids closer than `window` (the row of arc a
// is found by binary search in in_ptr).
__global__ void locality_sample(const uint64_t *__restrict__ in_ptr,
                                const uint32_t *__restrict__ in_col, uint64_t z, uint64_t arcs,
                                uint32_t samples, uint64_t window,
                                unsigned long long *__restrict__ close) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    bool c = false;
    if (s < samples && arcs) {
        const uint64_t a = arcs * s / samples;
        uint64_t lo = 0, hi = z;  // last row with in_ptr[row] <= a
        while (hi - lo > 1) {
            const uint64_t mid = (lo + hi) >> 1;
            if (in_ptr[mid] <= a)
                lo = mid;
            else
                hi = mid;
        }
        const uint64_t v = in_col[a];
        c = (v > lo ? v - lo : lo - v) < window;
    }
    const int cnt = __syncthreads_count(c);
    if (threadIdx.x == 0 && cnt)
        atomicAdd(close, static_cast<unsigned long long>(cnt));
}

// Ranking input: deleted ids get -inf so that they sort behind every score.
__global__ void ranking_prepare_kernel(double *__restrict__ keys, uint32_t *__restrict__ ids,
                                       const uint32_t *__restrict__ inv, uint64_t z) {
    const uint64_t o = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (o >= z)
        return;
    if (inv[o] == kNone)
        keys[o] = -1.0 / 0.0;
    ids[o] = static_cast<uint32_t>(o);
}

__global__ void build_perm(const uint32_t *__restrict__ sorted_ids, uint64_t n,
                           const uint64_t *__restrict__ in_ptr, uint32_t *__restrict__ perm,
                           uint32_t *__restrict__ inv, uint32_t *__restrict__ rowlen,
                           const uint32_t *__restrict__ outdeg, uint32_t *__restrict__ degc,
                           const double *__restrict__ wdeg, double *__restrict__ degw,
                           uint64_t *__restrict__ row_src) {
    const uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (r >= n)
        return;
    const uint32_t o = sorted_ids[r];
    perm[r] = o;
    row_src[r] = in_ptr[o];
    inv[o] = static_cast<uint32_t>(r);
    rowlen[r] = static_cast<uint32_t>(in_ptr[o + 1] - in_ptr[o]);
    degc[r] = outdeg[o];
    if (degw)
        degw[r] = wdeg[o];
}

// Copy every row into its new place, mapping column ids. Rows longer than
// kLaneRow arcs are a prefix [0, nb) of the new order (rows are sorted by
// length, or by half-octave length bucket whose edges fall on 2^k + 1). Their
// arcs are split into equal contiguous ranges, one per warp, so no warp holds
// a hub row alone; each lane walks its arcs with the row found by binary search
// once. The short rows go 32 consecutive rows per warp, one row per lane, so
// the dependent loads of 32 rows overlap. Neither part relies on the prefix
// order for correctness, only for speed.
constexpr uint32_t kLaneRow = 32;

__global__ void count_rows_over(const uint32_t *__restrict__ rowlen, uint64_t n, uint32_t thr,
                                unsigned long long *__restrict__ cnt) {
    const uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    const int a = __syncthreads_count(r < n && rowlen[r] > thr);
    if (threadIdx.x == 0 && a)
        atomicAdd(cnt, static_cast<unsigned long long>(a));
}

__global__ void relabel_rows(const uint32_t *__restrict__ perm, const uint64_t *__restrict__ in_ptr,
                             const uint32_t *__restrict__ in_col, const double *__restrict__ in_w,
                             const uint32_t *__restrict__ inv, const uint32_t *__restrict__ row_ptr,
                             uint64_t n, const unsigned long long *__restrict__ n_long_rows,
                             uint32_t *__restrict__ col, double *__restrict__ w) {
    const uint64_t warp = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const uint64_t nb = *n_long_rows;
    // Part 1: the arcs of rows [0, nb).
    const uint64_t big = row_ptr[nb];
    const uint64_t per = (big + nwarps - 1) / nwarps;
    const uint64_t a = warp * per;
    const uint64_t e = a + per < big ? a + per : big;
    uint64_t k = a + lane;
    if (k < e) {
        // the last row r with row_ptr[r] <= k: row_ptr[lo] <= k < row_ptr[hi]
        uint64_t lo = 0, hi = nb;
        while (hi - lo > 1) {
            const uint64_t mid = (lo + hi) >> 1;
            if (row_ptr[mid] <= k)
                lo = mid;
            else
                hi = mid;
        }
        uint64_t r = lo;
        uint64_t base = row_ptr[r], next = row_ptr[r + 1];
        uint64_t src = in_ptr[perm[r]];
        for (; k < e; k += 32) {
            if (next <= k) {
                do {
                    ++r;
                    base = next;
                    next = row_ptr[r + 1];
                } while (next <= k);
                src = in_ptr[perm[r]];
            }
            const uint64_t sk = src + (k - base);
            col[k] = inv[in_col[sk]];
            if (w)
                w[k] = in_w[sk];
        }
    }
    // Part 2: rows [nb, n), one per lane.
    for (uint64_t g0 = nb + warp * 32; g0 < n; g0 += nwarps * 32) {
        const uint64_t rr = g0 + lane;
        if (rr >= n)
            continue;
        const uint32_t dst = row_ptr[rr];
        const uint32_t len = row_ptr[rr + 1] - dst;
        const uint64_t sr = in_ptr[perm[rr]];
#pragma unroll 4
        for (uint32_t j = 0; j < len; ++j) {
            col[dst + j] = inv[in_col[sr + j]];
            if (w)
                w[dst + j] = in_w[sr + j];
        }
    }
}

// Rows longer than kChunk (a prefix, the rows are sorted by length) and, of
// those, rows with more than kShortChunks chunks.
__global__ void count_long(const uint32_t *__restrict__ rowlen, uint64_t n,
                           unsigned long long *__restrict__ cnt) {
    const uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    const bool lg = r < n && rowlen[r] > kChunk;
    const bool vl = r < n && rowlen[r] > kChunk * kShortChunks;
    const int a = __syncthreads_count(lg);
    const int b = __syncthreads_count(vl);
    if (threadIdx.x == 0) {
        if (a)
            atomicAdd(cnt, static_cast<unsigned long long>(a));
        if (b)
            atomicAdd(cnt + 1, static_cast<unsigned long long>(b));
    }
}

__global__ void chunk_counts(const uint32_t *__restrict__ rowlen, uint32_t n_long,
                             uint32_t *__restrict__ nch) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n_long)
        nch[r] = (rowlen[r] + kChunk - 1) / kChunk;
}

// chunk_row[k] = split row of chunk k, chunk_idx[k] = its index in that row.
__global__ void expand_chunks(const uint32_t *__restrict__ chunk_begin, uint32_t n_long,
                              uint32_t *__restrict__ chunk_row, uint32_t *__restrict__ chunk_idx) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint32_t r = warp; r < n_long; r += nwarps) {
        const uint32_t b = chunk_begin[r], e = chunk_begin[r + 1];
        for (uint32_t k = b + lane; k < e; k += 32) {
            chunk_row[k] = r;
            chunk_idx[k] = k - b;
        }
    }
}

// Virtual row v of slice s / lane: its first arc and its length.
struct VRow {
    uint32_t start;
    uint32_t len;
};

__device__ __forceinline__ VRow vrow_of(uint32_t s, int lane, uint32_t s_chunk, uint32_t n_chunks,
                                        uint32_t n_long, uint32_t n,
                                        const uint32_t *__restrict__ chunk_row,
                                        const uint32_t *__restrict__ chunk_idx,
                                        const uint32_t *__restrict__ row_ptr) {
    VRow v{0, 0};
    if (s < s_chunk) {
        const uint32_t k = s * 32 + lane;
        if (k < n_chunks) {
            const uint32_t r = chunk_row[k], c = chunk_idx[k];
            const uint32_t rs = row_ptr[r], re = row_ptr[r + 1];
            v.start = rs + c * kChunk;
            v.len = min(kChunk, re - v.start);
        }
    } else {
        const uint32_t r = n_long + (s - s_chunk) * 32 + lane;
        if (r < n) {
            v.start = row_ptr[r];
            v.len = row_ptr[r + 1] - v.start;
        }
    }
    return v;
}

// Slice length = longest of its 32 virtual rows (one warp per slice).
__global__ void slice_lengths(uint32_t slices, uint32_t s_chunk, uint32_t n_chunks,
                              uint32_t n_long, uint32_t n, const uint32_t *__restrict__ chunk_row,
                              const uint32_t *__restrict__ chunk_idx,
                              const uint32_t *__restrict__ row_ptr, uint32_t *__restrict__ slen,
                              uint64_t *__restrict__ scost) {
    const uint32_t s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= slices)
        return;
    const VRow v = vrow_of(s, lane, s_chunk, n_chunks, n_long, n, chunk_row, chunk_idx, row_ptr);
    uint32_t m = v.len;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) {
        slen[s] = m;
        scost[s] = static_cast<uint64_t>(m) + kSliceOverhead;
    }
}

// Fill the column-major slices; padding slots point at the zero entry n. The
// weight of CSR entry k is w[w_index[k]] (w[k] without an index); a null
// col_sell refreshes the weights only.
__global__ void fill_slices(uint32_t slices, uint32_t s_chunk, uint32_t n_chunks, uint32_t n_long,
                            uint32_t n, const uint32_t *__restrict__ chunk_row,
                            const uint32_t *__restrict__ chunk_idx,
                            const uint32_t *__restrict__ row_ptr, const uint32_t *__restrict__ col,
                            const double *__restrict__ w, const uint32_t *__restrict__ w_index,
                            const uint32_t *__restrict__ slice_off,
                            uint32_t *__restrict__ col_sell, double *__restrict__ w_sell,
                            uint32_t pad_col) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint32_t s = warp; s < slices; s += nwarps) {
        const VRow v =
            vrow_of(s, lane, s_chunk, n_chunks, n_long, n, chunk_row, chunk_idx, row_ptr);
        const uint32_t off = slice_off[s], len = slice_off[s + 1] - off;
        for (uint32_t j = 0; j < len; ++j) {
            const size_t slot = (static_cast<size_t>(off) + j) * 32 + lane;
            const bool real = j < v.len;
            if (col_sell)
                col_sell[slot] = real ? col[v.start + j] : pad_col;
            if (w_sell)
                w_sell[slot] = real ? w[w_index ? w_index[v.start + j] : v.start + j] : 0.0;
        }
    }
}

// Unit u covers slices [unit_start[u], unit_start[u+1]): the boundaries cut
// the inclusive cost prefix into `units` equal parts.
__global__ void unit_bounds(const uint64_t *__restrict__ cost_incl, uint32_t slices,
                            uint32_t units, uint32_t *__restrict__ unit_start) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u > units)
        return;
    if (u == units) {
        unit_start[u] = slices;
        return;
    }
    if (u == 0) {
        unit_start[0] = 0;
        return;
    }
    const uint64_t total = slices ? cost_incl[slices - 1] : 0;
    const uint64_t target = total * u / units;
    // First slice s whose exclusive prefix cost_incl[s-1] >= target, i.e.
    // one past the first index with an inclusive prefix >= target.
    uint32_t lo = 0, hi = slices;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (cost_incl[mid] < target)
            lo = mid + 1;
        else
            hi = mid;
    }
    unit_start[u] = lo + 1 < slices ? lo + 1 : slices;
}

template <typename T>
__global__ void convert_array(const double *__restrict__ in, T *__restrict__ out, uint64_t m) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < m; i += stride)
        out[i] = static_cast<T>(in[i]);
}

// ---------------------------------------------------------------------------
// Edge-list ingest (nkg_graph_create_from_edges): the in-CSR that
// Graph::addEdge builds (Graph.cpp:549-596), on the device.

// One key per arc: (row << 32) | edge index. Directed: row = dst. Undirected:
// both endpoints, a self-loop once (the second copy gets the sentinel key).
__global__ void ingest_keys(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                            uint64_t m, uint64_t z, int directed, uint64_t *__restrict__ keys,
                            int *__restrict__ err) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < m;
         e += stride) {
        const uint32_t u = src[e], v = dst[e];
        if (u >= z || v >= z) {
            atomicCAS(err, 0, 1);
            continue;
        }
        if (directed) {
            keys[e] = (static_cast<uint64_t>(v) << 32) | e;
        } else {
            keys[2 * e] = (static_cast<uint64_t>(u) << 32) | e;
            keys[2 * e + 1] = u == v ? ~0ull : (static_cast<uint64_t>(v) << 32) | e;
        }
    }
}

// Sorted keys -> in_col / in_w and the row histogram.
__global__ void ingest_fill(const uint64_t *__restrict__ keys, uint64_t arcs,
                            const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                            const double *__restrict__ w, int directed, uint32_t *__restrict__ col,
                            double *__restrict__ in_w, unsigned long long *__restrict__ counts) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < arcs;
         k += stride) {
        const uint64_t key = keys[k];
        const uint32_t row = static_cast<uint32_t>(key >> 32), e = static_cast<uint32_t>(key);
        const uint32_t u = src[e], v = dst[e];
        col[k] = directed ? u : (row == u ? v : u);
        if (w)
            in_w[k] = w[e];
        atomicAdd(counts + row, 1ull);
    }
}

__global__ void count_below(const uint64_t *__restrict__ keys, uint64_t count, uint64_t bound,
                            unsigned long long *__restrict__ cnt) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    unsigned long long c = 0;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < count;
         k += stride)
        c += keys[k] < bound;
    c = static_cast<unsigned long long>(warp_sum(static_cast<double>(c)));
    if ((threadIdx.x & 31) == 0 && c)
        atomicAdd(cnt, c);
}

// Sequential sum of vals[b..e) per segment (deterministic, in the given order).
__global__ void segment_sums(const uint64_t *__restrict__ ptr, const double *__restrict__ vals,
                             uint64_t segs, double *__restrict__ out) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= segs)
        return;
    double sum = 0.0;
    for (uint64_t k = ptr[i]; k < ptr[i + 1]; ++k)
        sum += vals[k];
    out[i] = sum;
}

// Directed weighted degrees: out-weights of every source in edge order.
__global__ void ingest_out_keys(const uint32_t *__restrict__ src, uint64_t m,
                                uint64_t *__restrict__ keys) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t e = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; e < m;
         e += stride)
        keys[e] = (static_cast<uint64_t>(src[e]) << 32) | e;
}

__global__ void ingest_out_vals(const uint64_t *__restrict__ keys, uint64_t m,
                                const double *__restrict__ w, double *__restrict__ vals,
                                unsigned long long *__restrict__ counts) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < m;
         k += stride) {
        const uint64_t key = keys[k];
        vals[k] = w[static_cast<uint32_t>(key)];
        atomicAdd(counts + (key >> 32), 1ull);
    }
}

// ---------------------------------------------------------------------------
// Per-run kernels

// PageRank.cpp:26: x = 1/n, stored in gather form.
template <typename T, bool WEIGHTED>
__global__ void init_iterate(T *__restrict__ y, const uint32_t *__restrict__ degc,
                             const T *__restrict__ degw, uint32_t n, double x0) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n)
        return;
    const T x = static_cast<T>(x0);
    const uint32_t dc = degc[r];
    if (dc == 0)
        y[r] = x;
    else
        y[r] = x / (WEIGHTED ? degw[r] : static_cast<T>(dc));
}

// Personalised teleport into the relabelled order.
template <typename T>
__global__ void permute_teleport(const double *__restrict__ t_orig, const uint32_t *__restrict__ perm,
                                 uint32_t n, T *__restrict__ t_new) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n)
        t_new[r] = static_cast<T>(t_orig[perm[r]]);
}

template <typename T, bool WEIGHTED>
__device__ __forceinline__ double final_x(const T *y, const uint32_t *degc, const T *degw,
                                          uint32_t r) {
    const T yv = y[r];
    const uint32_t dc = degc[r];
    if (dc == 0)
        return static_cast<double>(yv);
    const T d = WEIGHTED ? degw[r] : static_cast<T>(dc);
    return static_cast<double>(t_mul(yv, d));
}

constexpr int kRedThreads = 256;

// Sum of x, sum of x over sinks and max x (PageRank.cpp:76,83-87,95-102), two
// levels with a fixed order. red[0..2] receive the totals.
template <typename T, bool WEIGHTED>
__global__ void __launch_bounds__(kRedThreads)
    final_reduce(const T *__restrict__ y, const uint32_t *__restrict__ degc,
                 const T *__restrict__ degw, uint32_t n, double *__restrict__ part,
                 double *__restrict__ red, unsigned int *__restrict__ ticket) {
    __shared__ double s_red[32];
    __shared__ bool s_last;
    double s = 0.0, ss = 0.0, mx = -1.0 / 0.0;
    for (uint32_t r = blockIdx.x * kRedThreads + threadIdx.x; r < n; r += gridDim.x * kRedThreads) {
        const double x = final_x<T, WEIGHTED>(y, degc, degw, r);
        s += x;
        if (degc[r] == 0)
            ss += x;
        mx = fmax(mx, x);
    }
    s = block_sum<kRedThreads>(s, s_red);
    ss = block_sum<kRedThreads>(ss, s_red);
    mx = block_max<kRedThreads>(mx, s_red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x + 0] = s;
        part[3 * blockIdx.x + 1] = ss;
        part[3 * blockIdx.x + 2] = mx;
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    s = 0.0;
    ss = 0.0;
    mx = -1.0 / 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kRedThreads) {
        s += ((volatile double *)part)[3 * i + 0];
        ss += ((volatile double *)part)[3 * i + 1];
        mx = fmax(mx, ((volatile double *)part)[3 * i + 2]);
    }
    s = block_sum<kRedThreads>(s, s_red);
    ss = block_sum<kRedThreads>(ss, s_red);
    mx = block_max<kRedThreads>(mx, s_red);
    if (threadIdx.x == 0) {
        red[0] = s;
        red[1] = ss;
        red[2] = mx;
        *ticket = 0;
    }
}

// PageRank.cpp:75-92 scaling, written in the caller's id order; non-existent
// ids keep 1/n. red[3] receives maximum() for the normalised form.
template <typename T, bool WEIGHTED>
__global__ void final_scale(const T *__restrict__ y, const uint32_t *__restrict__ degc,
                            const T *__restrict__ degw, const uint32_t *__restrict__ inv,
                            uint64_t z, uint32_t n, double damp, int normalized,
                            double *__restrict__ red, double *__restrict__ out) {
    const uint64_t o = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (o >= z)
        return;
    const double factor =
        normalized ? (1.0 / static_cast<double>(n)) * ((1 - damp) + (damp * red[1])) : red[0];
    const uint32_t r = inv[o];
    double v;
    if (r == kNone)
        v = 1.0 / static_cast<double>(n);
    else
        v = final_x<T, WEIGHTED>(y, degc, degw, r) / factor;
    out[o] = v;
    if (o == 0)
        red[3] = normalized ? fmax(v, red[2] / factor) : 1.0;
}

// ---------------------------------------------------------------------------
// Host side

// Sort every in-row by source id (relabelled), weights alongside.
static void sort_rows(nkg_graph *g, cudaStream_t s) {
    const int items = static_cast<int>(g->arcs);
    const int segs = static_cast<int>(g->n);
    DeviceArray<uint32_t> col2(g->arcs, 4);
    size_t tb = 0;
    if (g->weighted) {
        DeviceArray<double> w2(g->arcs, 4);
        NKG_CUDA(cub::DeviceSegmentedSort::SortPairs(nullptr, tb, g->col.get(), col2.get(),
                                                     g->w64src.get(), w2.get(), items, segs,
                                                     g->row_ptr.get(), g->row_ptr.get() + 1, s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceSegmentedSort::SortPairs(tmp.get(), tb, g->col.get(), col2.get(),
                                                     g->w64src.get(), w2.get(), items, segs,
                                                     g->row_ptr.get(), g->row_ptr.get() + 1, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        g->w64src = std::move(w2);
    } else {
        NKG_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, tb, g->col.get(), col2.get(), items,
                                                    segs, g->row_ptr.get(), g->row_ptr.get() + 1,
                                                    s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceSegmentedSort::SortKeys(tmp.get(), tb, g->col.get(), col2.get(), items,
                                                    segs, g->row_ptr.get(), g->row_ptr.get() + 1,
                                                    s));
        NKG_CUDA(cudaStreamSynchronize(s));
    }
    g->col = std::move(col2);
    g->arc_sorted = true;
}

// Build the sliced layout L of a CSR whose n rows are sorted by length,
// descending (row_ptr, col, optional weights w through w_index, rowlen).
void build_sell(SellLayout &L, uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                const double *w, const uint32_t *w_index, const uint32_t *rowlen, int device,
                cudaStream_t s, uint32_t pad_col) {
    if (pad_col == kNone)
        pad_col = n;
    const unsigned sms = num_sms(device);
    DeviceArray<unsigned long long> cnt(2);
    NKG_CUDA(cudaMemsetAsync(cnt.get(), 0, 2 * sizeof(unsigned long long), s));
    count_long<<<ceil_div(n, 256), 256, 0, s>>>(rowlen, n, cnt.get());
    NKG_CUDA(cudaGetLastError());
    unsigned long long h_cnt[2];
    NKG_CUDA(cudaMemcpyAsync(h_cnt, cnt.get(), sizeof(h_cnt), cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    L.n_long = static_cast<uint32_t>(h_cnt[0]);
    L.n_vlong = static_cast<uint32_t>(h_cnt[1]);

    L.chunk_begin.alloc(static_cast<size_t>(L.n_long) + 1);
    NKG_CUDA(cudaMemsetAsync(L.chunk_begin.get(), 0, sizeof(uint32_t), s));
    DeviceArray<uint32_t> chunk_row, chunk_idx;
    if (L.n_long) {
        DeviceArray<uint32_t> nch(L.n_long);
        chunk_counts<<<ceil_div(L.n_long, 256), 256, 0, s>>>(rowlen, L.n_long, nch.get());
        size_t tb = 0;
        NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, nch.get(), L.chunk_begin.get() + 1,
                                               static_cast<int64_t>(L.n_long), s));
        DeviceArray<unsigned char> tmp(tb);
        NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb, nch.get(), L.chunk_begin.get() + 1,
                                               static_cast<int64_t>(L.n_long), s));
        L.n_chunks = read_scalar(L.chunk_begin.get() + L.n_long, s);
        chunk_row.alloc(L.n_chunks);
        chunk_idx.alloc(L.n_chunks);
        expand_chunks<<<sms * 4, 256, 0, s>>>(L.chunk_begin.get(), L.n_long, chunk_row.get(),
                                              chunk_idx.get());
        NKG_CUDA(cudaGetLastError());
    } else {
        L.n_chunks = 0;
    }
    L.s_chunk = (L.n_chunks + 31) / 32;
    const uint64_t s_rows = (static_cast<uint64_t>(n - L.n_long) + 31) / 32;
    const uint64_t slices = L.s_chunk + s_rows;
    require(slices < 0xffffffffull, "too many slices");
    L.slices = static_cast<uint32_t>(slices);

    DeviceArray<uint32_t> slen(L.slices);
    DeviceArray<uint64_t> scost(L.slices);
    L.slice_cost.alloc(L.slices);
    L.slice_off.alloc(static_cast<size_t>(L.slices) + 1);
    if (L.slices) {
        slice_lengths<<<ceil_div(static_cast<uint64_t>(L.slices) * 32, 256), 256, 0, s>>>(
            L.slices, L.s_chunk, L.n_chunks, L.n_long, n, chunk_row.get(), chunk_idx.get(),
            row_ptr, slen.get(), scost.get());
        NKG_CUDA(cudaGetLastError());
    }
    NKG_CUDA(cudaMemsetAsync(L.slice_off.get(), 0, sizeof(uint32_t), s));
    if (L.slices) {
        size_t tb = 0;
        NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, slen.get(), L.slice_off.get() + 1,
                                               static_cast<int64_t>(L.slices), s));
        size_t tb2 = 0;
        NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb2, scost.get(), L.slice_cost.get(),
                                               static_cast<int64_t>(L.slices), s));
        DeviceArray<unsigned char> tmp(std::max(tb, tb2));
        NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb, slen.get(), L.slice_off.get() + 1,
                                               static_cast<int64_t>(L.slices), s));
        NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb2, scost.get(), L.slice_cost.get(),
                                               static_cast<int64_t>(L.slices), s));
    }
    const uint32_t cols = read_scalar(L.slice_off.get() + L.slices, s);
    L.slots = static_cast<uint64_t>(cols) * 32;
    L.col_sell.alloc(L.slots, 4);
    if (w)
        L.w_sell64.alloc(L.slots, 4);
    if (L.slices) {
        fill_slices<<<sms * 16, 256, 0, s>>>(L.slices, L.s_chunk, L.n_chunks, L.n_long, n,
                                             chunk_row.get(), chunk_idx.get(), row_ptr, col, w,
                                             w_index, L.slice_off.get(), L.col_sell.get(),
                                             L.w_sell64.get(), pad_col);
        NKG_CUDA(cudaGetLastError());
    }
    NKG_CUDA(cudaStreamSynchronize(s));
}

// map[slot] = index[k] for the CSR entry k the slot holds (kNone for padding).
__global__ void fill_slot_map(uint32_t slices, uint32_t s_chunk, uint32_t n_chunks, uint32_t n_long,
                              uint32_t n, const uint32_t *__restrict__ chunk_row,
                              const uint32_t *__restrict__ chunk_idx,
                              const uint32_t *__restrict__ row_ptr,
                              const uint32_t *__restrict__ index,
                              const uint32_t *__restrict__ slice_off, uint32_t *__restrict__ map) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (uint32_t s = warp; s < slices; s += nwarps) {
        const VRow v =
            vrow_of(s, lane, s_chunk, n_chunks, n_long, n, chunk_row, chunk_idx, row_ptr);
        const uint32_t off = slice_off[s], len = slice_off[s + 1] - off;
        for (uint32_t j = 0; j < len; ++j)
            map[(static_cast<size_t>(off) + j) * 32 + lane] = j < v.len ? index[v.start + j] : kNone;
    }
}

void build_slot_map(const SellLayout &L, uint32_t n, const uint32_t *row_ptr, const uint32_t *index,
                    uint32_t *map, int device, cudaStream_t s) {
    if (!L.slices)
        return;
    const unsigned sms = num_sms(device);
    DeviceArray<uint32_t> chunk_row(std::max<uint32_t>(L.n_chunks, 1)),
        chunk_idx(std::max<uint32_t>(L.n_chunks, 1));
    if (L.n_long)
        expand_chunks<<<sms * 4, 256, 0, s>>>(L.chunk_begin.get(), L.n_long, chunk_row.get(),
                                              chunk_idx.get());
    fill_slot_map<<<sms * 16, 256, 0, s>>>(L.slices, L.s_chunk, L.n_chunks, L.n_long, n,
                                           chunk_row.get(), chunk_idx.get(), row_ptr, index,
                                           L.slice_off.get(), map);
    NKG_CUDA(cudaGetLastError());
    NKG_CUDA(cudaStreamSynchronize(s));
}

// Cut the slices of L into `units` cost-balanced ranges (unit_start, units+1).
void sell_units(const SellLayout &L, uint32_t units, uint32_t *unit_start, cudaStream_t s) {
    unit_bounds<<<ceil_div(static_cast<uint64_t>(units) + 1, 256), 256, 0, s>>>(
        L.slice_cost.get(), L.slices, units, unit_start);
    NKG_CUDA(cudaGetLastError());
}

void convert_to_float(const double *in, float *out, uint64_t m, int device, cudaStream_t s) {
    if (!m)
        return;
    convert_array<float><<<num_sms(device) * 8, 256, 0, s>>>(in, out, m);
    NKG_CUDA(cudaGetLastError());
}

static int option_device(const nkg_graph_options *opt) {
    int dev = opt && opt->device >= 0 ? opt->device : -1;
    if (dev < 0)
        NKG_CUDA(cudaGetDevice(&dev));
    return dev;
}

// A handle with its device, stream and events (dev current); no graph data yet.
static std::unique_ptr<nkg_graph> graph_shell(int dev, uint64_t z, uint64_t arcs, bool weighted,
                                              int directed) {
    require(z >= 1, "graph must have at least one node id (z >= 1)");
    require(z < 0xffffffffull, "node ids must fit in 32 bits (z < 2^32 - 1)");
    require(arcs < 0xfffffff0ull, "graphs with 2^32 or more arcs are not supported");
    std::unique_ptr<nkg_graph> g(new nkg_graph());
    g->device = dev;
    g->z = z;
    g->arcs = arcs;
    g->weighted = weighted;
    g->directed = directed != 0;
    g->stream = stream_acquire(dev);
    NKG_CUDA(cudaEventCreate(&g->ev0));
    NKG_CUDA(cudaEventCreate(&g->ev1));
    NKG_CUDA(cudaEventCreate(&g->ev2));
    return g;
}

static nkg_graph *build_graph(std::unique_ptr<nkg_graph> g, DeviceArray<uint64_t> &d_ptr,
                              DeviceArray<uint32_t> &d_col, DeviceArray<double> &d_w,
                              DeviceArray<double> &d_wdeg, DeviceArray<uint8_t> &d_ex,
                              const uint8_t *exists, const nkg_graph_options *opt);

static nkg_graph *create_graph(uint64_t z, uint64_t arcs, const uint64_t *in_ptr,
                               const uint32_t *in_col, const double *in_w, const double *wdeg,
                               const uint8_t *exists, int directed, const nkg_graph_options *opt) {
    require(in_ptr != nullptr, "in_row_ptr is NULL");
    require(arcs == 0 || in_col != nullptr, "in_col is NULL");
    require(in_w == nullptr || wdeg != nullptr, "weighted graph needs out_wdeg");
    DeviceGuard guard(option_device(opt));
    std::unique_ptr<nkg_graph> g = graph_shell(option_device(opt), z, arcs, in_w != nullptr,
                                               directed);
    require(in_ptr[0] == 0 && in_ptr[z] == arcs, "in_row_ptr must start at 0 and end at arcs");
    cudaStream_t s = g->stream;

    // Upload.
    DeviceArray<uint64_t> d_ptr(z + 1);
    DeviceArray<uint32_t> d_col(arcs);
    DeviceArray<double> d_w, d_wdeg;
    DeviceArray<uint8_t> d_ex;
    NKG_CUDA(cudaMemcpyAsync(d_ptr.get(), in_ptr, (z + 1) * sizeof(uint64_t),
                             cudaMemcpyHostToDevice, s));
    if (arcs)
        NKG_CUDA(cudaMemcpyAsync(d_col.get(), in_col, arcs * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, s));
    if (in_w) {
        d_w.alloc(arcs);
        d_wdeg.alloc(z);
        if (arcs)
            NKG_CUDA(cudaMemcpyAsync(d_w.get(), in_w, arcs * sizeof(double),
                                     cudaMemcpyHostToDevice, s));
        NKG_CUDA(cudaMemcpyAsync(d_wdeg.get(), wdeg, z * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    if (exists) {
        d_ex.alloc(z);
        NKG_CUDA(cudaMemcpyAsync(d_ex.get(), exists, z, cudaMemcpyHostToDevice, s));
    }
    NKG_CUDA(cudaEventRecord(g->ev0, s));
    return build_graph(std::move(g), d_ptr, d_col, d_w, d_wdeg, d_ex, exists, opt);
}

// The rest of the upload from the in-CSR in device memory: validation,
// relabelling, sliced layout, per-run buffers. `exists` (host, nullable) is
// the existence mask d_ex holds on the device.
static nkg_graph *build_graph(std::unique_ptr<nkg_graph> g, DeviceArray<uint64_t> &d_ptr,
                              DeviceArray<uint32_t> &d_col, DeviceArray<double> &d_w,
                              DeviceArray<double> &d_wdeg, DeviceArray<uint8_t> &d_ex,
                              const uint8_t *exists, const nkg_graph_options *opt) {
    const uint64_t z = g->z, arcs = g->arcs;
    const int dev = g->device;
    cudaStream_t s = g->stream;

    // Validate + out-degree count.
    DeviceArray<uint32_t> outdeg(z);
    DeviceArray<int> err(1);
    DeviceArray<unsigned long long> cnt(1);
    NKG_CUDA(cudaMemsetAsync(outdeg.get(), 0, z * sizeof(uint32_t), s));
    NKG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
    NKG_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(unsigned long long), s));
    const unsigned sms = num_sms(dev);
    validate_and_count<<<sms * 8, 256, 0, s>>>(d_ptr.get(), d_col.get(), d_ex.get(), z, arcs,
                                              outdeg.get(), err.get());
    NKG_CUDA(cudaGetLastError());
    const int h_err = read_scalar(err.get(), s);
    switch (h_err) {
    case 0: break;
    case 1: throw Error(NKG_ERR_INVALID_ARG, "in_row_ptr is not non-decreasing within [0, arcs]");
    case 2: throw Error(NKG_ERR_INVALID_ARG, "in_col holds a node id >= z");
    case 3: throw Error(NKG_ERR_INVALID_ARG, "in_col refers to a non-existent node");
    default: throw Error(NKG_ERR_INVALID_ARG, "a non-existent node has in-arcs");
    }

    // Relabelling order: in-degree descending (row_order 0) or half-octave
    // in-degree buckets descending (row_order 1), ties by id; -1 picks 1 when
    // the caller's ids carry locality (more than 1/4 of 65,536 sampled arcs
    // join ids closer than max(64, z/1024)).
    int row_order = opt ? opt->row_order : -1;  // no options: automatic
    require(row_order >= -1 && row_order <= 1, "row_order must be -1, 0 or 1");
    if (row_order < 0) {
        constexpr uint32_t kSamples = 65536;
        DeviceArray<unsigned long long> close(1);
        NKG_CUDA(cudaMemsetAsync(close.get(), 0, sizeof(unsigned long long), s));
        locality_sample<<<kSamples / 256, 256, 0, s>>>(d_ptr.get(), d_col.get(), z, arcs, kSamples,
                                                       std::max<uint64_t>(64, z / 1024),
                                                       close.get());
        NKG_CUDA(cudaGetLastError());
        row_order = (arcs && read_scalar(close.get(), s) * 4 > kSamples) ? 1 : 0;
    }
    g->row_order = row_order;
    DeviceArray<uint32_t> keys(z), ids(z), keys_s(z), ids_s(z);
    make_keys<<<ceil_div(z, 256), 256, 0, s>>>(d_ptr.get(), outdeg.get(), d_ex.get(), z,
                                               row_order, keys.get(), ids.get(), cnt.get());
    NKG_CUDA(cudaGetLastError());
    size_t tmp_bytes = 0;
    NKG_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_bytes, keys.get(), keys_s.get(),
                                                       ids.get(), ids_s.get(), static_cast<int64_t>(z),
                                                       0, 32, s));
    DeviceArray<unsigned char> tmp(tmp_bytes);
    NKG_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.get(), tmp_bytes, keys.get(), keys_s.get(),
                                                       ids.get(), ids_s.get(), static_cast<int64_t>(z),
                                                       0, 32, s));
    uint64_t n = z;
    if (exists) {
        n = 0;
        for (uint64_t i = 0; i < z; ++i)
            n += exists[i] != 0;
    }
    require(n >= 1, "graph has no existing node");
    g->n = n;
    g->sinks = read_scalar(cnt.get(), s);

    g->perm.alloc(n);
    g->inv.alloc(z);
    g->degc.alloc(n);
    g->row_src.alloc(n);
    g->row_ptr.alloc(n + 1, 4);
    DeviceArray<uint32_t> rowlen(n);
    if (g->weighted)
        g->degw64src.alloc(n);
    NKG_CUDA(cudaMemsetAsync(g->inv.get(), 0xff, z * sizeof(uint32_t), s));
    build_perm<<<ceil_div(n, 256), 256, 0, s>>>(ids_s.get(), n, d_ptr.get(), g->perm.get(),
                                                g->inv.get(), rowlen.get(), outdeg.get(),
                                                g->degc.get(), d_wdeg.get(), g->degw64src.get(),
                                                g->row_src.get());
    NKG_CUDA(cudaGetLastError());
    NKG_CUDA(cudaMemsetAsync(g->row_ptr.get(), 0, sizeof(uint32_t), s));
    tmp_bytes = 0;
    NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, rowlen.get(), g->row_ptr.get() + 1,
                                           static_cast<int64_t>(n), s));
    tmp.alloc(tmp_bytes);
    NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tmp_bytes, rowlen.get(), g->row_ptr.get() + 1,
                                           static_cast<int64_t>(n), s));
    g->col.alloc(arcs, 4);
    if (g->weighted)
        g->w64src.alloc(arcs, 4);
    if (arcs) {
        NKG_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(unsigned long long), s));
        count_rows_over<<<ceil_div(n, 256), 256, 0, s>>>(rowlen.get(), n, kLaneRow, cnt.get());
        relabel_rows<<<sms * 16, 256, 0, s>>>(g->perm.get(), d_ptr.get(), d_col.get(), d_w.get(),
                                              g->inv.get(), g->row_ptr.get(), n, cnt.get(),
                                              g->col.get(), g->w64src.get());
    }
    NKG_CUDA(cudaGetLastError());
    if (opt) {
        require(opt->sweep_shape >= -1 && opt->sweep_shape < kNumSweepShapes,
                "unknown sweep shape");
        require(opt->arc_order == 0 || opt->arc_order == 1, "arc_order must be 0 or 1");
        require(opt->hot_tier_kb >= -1 && opt->hot_tier_kb <= static_cast<int>(kHotMaxBytes / 1024),
                "hot_tier_kb must be in [-1, 224]");
        g->hot_tier_kb = opt->hot_tier_kb;
        if (opt->sweep_shape >= 0)
            g->sweep_shape = opt->sweep_shape;
        if (opt->arc_order == 1 && arcs > 1 && arcs < 0x7fffffffull)
            sort_rows(g.get(), s);
    }
    build_sell(g->fw, static_cast<uint32_t>(n), g->row_ptr.get(), g->col.get(), g->w64src.get(),
               nullptr, rowlen.get(), dev, s);
    NKG_CUDA(cudaEventRecord(g->ev1, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    NKG_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    g->ms_create = ms;

    // Per-run bookkeeping buffers. The partial-sum arrays are sized for the
    // largest grid any sweep launch can use (32 resident CTAs per SM), so
    // they are never reallocated under a captured graph.
    g->cta_res.alloc(static_cast<size_t>(sms) * 32);
    g->cta_sink.alloc(static_cast<size_t>(sms) * 32);
    // Fix-up grids also cover the queued sweep's unit partials (at most one
    // unit per slice, kUnitsPerFixThread per thread).
    const size_t fix = std::max<size_t>(
        static_cast<size_t>(g->fw.n_vlong) + ceil_div(g->fw.n_long, kFixThreads) + 1,
        fix_ctas_with_units(1, g->fw.slices, kFixThreads));
    g->fix_res.alloc(fix);
    g->fix_sink.alloc(fix);
    g->rp.alloc(1);
    g->st.alloc(1);
    g->trace.alloc(kTraceCapacity);
    g->red.alloc(4 + 3 * 4096);
    g->red_ticket.alloc(1);
    NKG_CUDA(cudaMemsetAsync(g->red_ticket.get(), 0, sizeof(unsigned int), s));
    g->st_host.alloc(1);
    g->scalars_host.alloc(16);
    NKG_CUDA(cudaStreamSynchronize(s));
    return g.release();
}

static void sort_keys64(DeviceArray<uint64_t> &keys, uint64_t count, int end_bit, cudaStream_t s) {
    DeviceArray<uint64_t> out(std::max<uint64_t>(count, 1));
    size_t tb = 0;
    NKG_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys.get(), out.get(),
                                            static_cast<int64_t>(count), 0, end_bit, s));
    DeviceArray<unsigned char> tmp(tb);
    NKG_CUDA(cub::DeviceRadixSort::SortKeys(tmp.get(), tb, keys.get(), out.get(),
                                            static_cast<int64_t>(count), 0, end_bit, s));
    keys = std::move(out);
}

// counts (z) -> offsets (z + 1).
static void counts_to_ptr(const unsigned long long *counts, uint64_t z, uint64_t *ptr,
                          cudaStream_t s) {
    NKG_CUDA(cudaMemsetAsync(ptr, 0, sizeof(uint64_t), s));
    size_t tb = 0;
    NKG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, counts, ptr + 1,
                                           static_cast<int64_t>(z), s));
    DeviceArray<unsigned char> tmp(tb);
    NKG_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tb, counts, ptr + 1,
                                           static_cast<int64_t>(z), s));
}

// The graph of m edges inserted in the given order (src[e], dst[e], weight
// w[e]), as nkg_graph_create would get it from Graph::forInEdgesOf.
static nkg_graph *create_from_edges(uint64_t z, uint64_t m, const uint32_t *src,
                                    const uint32_t *dst, const double *w, const uint8_t *exists,
                                    int directed, bool on_device, const nkg_graph_options *opt) {
    require(m == 0 || (src != nullptr && dst != nullptr), "src / dst is NULL");
    require(m < 0x7fffffffull, "edge lists of 2^31 or more edges are not supported");
    DeviceGuard guard(option_device(opt));
    const uint64_t max_arcs = directed ? m : 2 * m;
    std::unique_ptr<nkg_graph> g0 = graph_shell(option_device(opt), z, 0, w != nullptr, directed);
    cudaStream_t s = g0->stream;
    const unsigned sms = num_sms(g0->device);
    DeviceArray<uint32_t> d_src, d_dst;
    DeviceArray<double> d_ew;
    const uint32_t *ps = src, *pd = dst;
    const double *pw = w;
    if (!on_device && m) {
        d_src.alloc(m);
        d_dst.alloc(m);
        NKG_CUDA(cudaMemcpyAsync(d_src.get(), src, m * 4, cudaMemcpyHostToDevice, s));
        NKG_CUDA(cudaMemcpyAsync(d_dst.get(), dst, m * 4, cudaMemcpyHostToDevice, s));
        ps = d_src.get();
        pd = d_dst.get();
        if (w) {
            d_ew.alloc(m);
            NKG_CUDA(cudaMemcpyAsync(d_ew.get(), w, m * 8, cudaMemcpyHostToDevice, s));
            pw = d_ew.get();
        }
    }
    std::vector<uint8_t> ex_host;
    DeviceArray<uint8_t> d_ex;
    const uint8_t *exh = nullptr;
    if (exists) {
        d_ex.alloc(z);
        ex_host.resize(z);
        if (on_device) {
            NKG_CUDA(cudaMemcpyAsync(ex_host.data(), exists, z, cudaMemcpyDeviceToHost, s));
            NKG_CUDA(cudaMemcpyAsync(d_ex.get(), exists, z, cudaMemcpyDeviceToDevice, s));
        } else {
            std::memcpy(ex_host.data(), exists, z);
            NKG_CUDA(cudaMemcpyAsync(d_ex.get(), exists, z, cudaMemcpyHostToDevice, s));
        }
        exh = ex_host.data();
    }
    NKG_CUDA(cudaEventRecord(g0->ev0, s));

    int zbits = 1;
    while (zbits < 32 && (1ull << zbits) < z)
        ++zbits;
    DeviceArray<uint64_t> keys(std::max<uint64_t>(max_arcs, 1));
    DeviceArray<int> err(1);
    NKG_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
    if (m)
        ingest_keys<<<sms * 8, 256, 0, s>>>(ps, pd, m, z, directed, keys.get(), err.get());
    NKG_CUDA(cudaGetLastError());
    require(read_scalar(err.get(), s) == 0, "an edge endpoint is >= z");
    // Self-loop copies carry the all-ones key and sort behind every arc.
    sort_keys64(keys, max_arcs, directed ? 32 + zbits : 64, s);
    uint64_t arcs = max_arcs;
    if (!directed && m) {
        // arcs = number of keys below the sentinel: find it on the host side of a
        // small read-back (the sentinel keys form the tail).
        DeviceArray<unsigned long long> cnt(1);
        NKG_CUDA(cudaMemsetAsync(cnt.get(), 0, sizeof(unsigned long long), s));
        count_below<<<sms * 8, 256, 0, s>>>(keys.get(), max_arcs, ~0ull, cnt.get());
        NKG_CUDA(cudaGetLastError());
        arcs = read_scalar(cnt.get(), s);
    }
    require(arcs < 0xfffffff0ull, "graphs with 2^32 or more arcs are not supported");
    g0->arcs = arcs;
    DeviceArray<uint64_t> d_ptr(z + 1);
    DeviceArray<uint32_t> d_col(std::max<uint64_t>(arcs, 1));
    DeviceArray<double> d_w, d_wdeg;
    DeviceArray<unsigned long long> counts(z);
    NKG_CUDA(cudaMemsetAsync(counts.get(), 0, z * sizeof(unsigned long long), s));
    if (w) {
        d_w.alloc(std::max<uint64_t>(arcs, 1));
        d_wdeg.alloc(z);
    }
    if (arcs)
        ingest_fill<<<sms * 8, 256, 0, s>>>(keys.get(), arcs, ps, pd, pw, directed, d_col.get(),
                                            d_w.get(), counts.get());
    NKG_CUDA(cudaGetLastError());
    counts_to_ptr(counts.get(), z, d_ptr.get(), s);
    if (w) {
        if (directed) {
            // out-weights of every source in edge order
            DeviceArray<uint64_t> okeys(std::max<uint64_t>(m, 1));
            DeviceArray<double> ovals(std::max<uint64_t>(m, 1));
            DeviceArray<uint64_t> optr(z + 1);
            NKG_CUDA(cudaMemsetAsync(counts.get(), 0, z * sizeof(unsigned long long), s));
            if (m) {
                ingest_out_keys<<<sms * 8, 256, 0, s>>>(ps, m, okeys.get());
                sort_keys64(okeys, m, 32 + zbits, s);
                ingest_out_vals<<<sms * 8, 256, 0, s>>>(okeys.get(), m, pw, ovals.get(),
                                                        counts.get());
            }
            counts_to_ptr(counts.get(), z, optr.get(), s);
            segment_sums<<<ceil_div(z, 256), 256, 0, s>>>(optr.get(), ovals.get(), z,
                                                          d_wdeg.get());
        } else {
            segment_sums<<<ceil_div(z, 256), 256, 0, s>>>(d_ptr.get(), d_w.get(), z,
                                                          d_wdeg.get());
        }
        NKG_CUDA(cudaGetLastError());
    }
    keys.reset();
    d_src.reset();
    d_dst.reset();
    d_ew.reset();
    return build_graph(std::move(g0), d_ptr, d_col, d_w, d_wdeg, d_ex, exh, opt);
}

// Graph creation from an in-CSR another translation unit built on the device
// (the NetworkitBinaryGraph decoder, nkbg.cu): a shell on `device` whose
// stream the builder uses, then the regular validation, relabelling and
// layout of build_graph once z and arcs are known.
std::unique_ptr<nkg_graph> device_graph_shell(const nkg_graph_options *opt, uint64_t z,
                                              bool weighted, int directed) {
    DeviceGuard guard(option_device(opt));
    return graph_shell(option_device(opt), z, 0, weighted, directed);
}

nkg_graph *device_graph_build(std::unique_ptr<nkg_graph> g, uint64_t arcs,
                              DeviceArray<uint64_t> &d_ptr, DeviceArray<uint32_t> &d_col,
                              DeviceArray<double> &d_w, DeviceArray<double> &d_wdeg,
                              DeviceArray<uint8_t> &d_ex, const uint8_t *exists_host,
                              const nkg_graph_options *opt) {
    DeviceGuard guard(g->device);
    g->arcs = arcs;
    NKG_CUDA(cudaEventRecord(g->ev0, g->stream));
    return build_graph(std::move(g), d_ptr, d_col, d_w, d_wdeg, d_ex, exists_host, opt);
}

static void destroy_plane_graphs(nkg_graph *g) {
    for (int i = 0; i < 2; ++i) {
        if (g->p64.exec[i])
            cudaGraphExecDestroy(g->p64.exec[i]);
        if (g->p32.exec[i])
            cudaGraphExecDestroy(g->p32.exec[i]);
        g->p64.exec[i] = g->p32.exec[i] = nullptr;
    }
}

}  // namespace nkg

// Waits for the handle's stream, then releases its CUDA objects (the stream
// goes back to the per-device pool); the device arrays free themselves after.
nkg_graph::~nkg_graph() {
    if (stream)
        cudaStreamSynchronize(stream);
    nkg::destroy_plane_graphs(this);
    if (ev0)
        cudaEventDestroy(ev0);
    if (ev1)
        cudaEventDestroy(ev1);
    if (ev2)
        cudaEventDestroy(ev2);
    nkg::stream_release(device, stream);
}

namespace nkg {

template <typename T>
Plane<T> &plane(nkg_graph *g);
template <>
Plane<double> &plane<double>(nkg_graph *g) { return g->p64; }
template <>
Plane<float> &plane<float>(nkg_graph *g) { return g->p32; }

// Tier size used when the options leave it to the library (KB per SM): none,
// the measured best (the tier costs L1 that the gathers need).
constexpr int kDefaultHotTierKB = 0;

// Ids held by the shared-memory tier of the PageRank sweep: the requested KB
// in ids, at most the n + 1 entries of the iterate rounded up to 16 bytes
// (the iterate buffers carry 4 elements of zero padding past n + 1, so the
// rounded copy stays inside them and the extra ids read zero).
template <typename T>
static uint32_t hot_tier_ids(const nkg_graph *g) {
    const int kb = g->hot_tier_kb < 0 ? kDefaultHotTierKB : g->hot_tier_kb;
    if (kb <= 0)
        return 0;
    constexpr uint64_t per16 = 16 / sizeof(T);
    const uint64_t want = static_cast<uint64_t>(kb) * 1024 / sizeof(T);
    const uint64_t all = (g->n + 1 + per16 - 1) / per16 * per16;
    return static_cast<uint32_t>(std::min(want, all) / per16 * per16);
}

template <typename T, bool WEIGHTED>
static void sweep_setup(nkg_graph *g) {
    Plane<T> &P = plane<T>(g);
    if (P.y[0])
        return;
    cudaStream_t s = g->stream;
    const uint64_t n = g->n;
    const unsigned sms = num_sms(g->device);
    for (int b = 0; b < 2; ++b) {
        P.y[b].alloc(n + 1, 4);
        NKG_CUDA(cudaMemsetAsync(P.y[b].get(), 0, (n + 1 + 4) * sizeof(T), s));
    }
    P.chunk_val.alloc(static_cast<size_t>(g->fw.s_chunk) * 32 + 1);
    if (WEIGHTED && !std::is_same<T, double>::value) {
        P.w_sell.alloc(g->fw.slots, 4);
        P.degw.alloc(n);
        if (g->fw.slots)
            convert_array<T><<<sms * 8, 256, 0, s>>>(g->fw.w_sell64.get(), P.w_sell.get(), g->fw.slots);
        convert_array<T><<<sms * 8, 256, 0, s>>>(g->degw64src.get(), P.degw.get(), n);
        NKG_CUDA(cudaGetLastError());
    }
    int occ = 0, threads = 0;
    with_sweep_shape(g->sweep_shape, [&](auto S) {
        using Sh = decltype(S);
        auto kfn = sweep_kernel<T, WEIGHTED, Sh::threads, Sh::unroll, false, false, true>;
        // The kernel needs almost no shared memory: give the L1 the most room.
        NKG_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, 0));
        NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, Sh::threads, 0));
        threads = Sh::threads;
    });
    require(occ >= 1, "sweep kernel does not fit on an SM");
    P.sweep_ctas = static_cast<unsigned>(std::max<uint64_t>(
        1, std::min<uint64_t>(static_cast<uint64_t>(occ) * sms,
                              (static_cast<uint64_t>(g->fw.slices) * 32 + threads - 1) / threads)));
    const uint64_t warps = static_cast<uint64_t>(P.sweep_ctas) * (threads / 32);
    P.units = static_cast<uint32_t>(
        std::max<uint64_t>(1, std::min<uint64_t>(warps * kUnitsPerWarp, g->fw.slices)));
    P.unit_start.alloc(static_cast<size_t>(P.units) + 1);
    unit_bounds<<<ceil_div(static_cast<uint64_t>(P.units) + 1, 256), 256, 0, s>>>(
        g->fw.slice_cost.get(), g->fw.slices, P.units, P.unit_start.get());
    NKG_CUDA(cudaGetLastError());
    P.fix_ctas = fix_vlong_ctas(g->fw.n_vlong) +
                 ceil_div(std::max<uint32_t>(g->fw.n_long - g->fw.n_vlong, 1), kFixThreads);
    P.hot = hot_tier_ids<T>(g);
    if (!P.hot) {
        // The queued sweep's units (the tier kernel keeps the static ones).
        P.q_units = static_cast<uint32_t>(std::max<uint64_t>(
            1, std::min<uint64_t>(warps * kQueueUnitsPerWarp, g->fw.slices)));
        P.q_unit_start.alloc(static_cast<size_t>(P.q_units) + 1);
        P.q_part.alloc(2 * static_cast<size_t>(P.q_units));
        unit_bounds<<<ceil_div(static_cast<uint64_t>(P.q_units) + 1, 256), 256, 0, s>>>(
            g->fw.slice_cost.get(), g->fw.slices, P.q_units, P.q_unit_start.get());
        NKG_CUDA(cudaGetLastError());
        P.fix_ctas = fix_ctas_with_units(P.fix_ctas, P.q_units, kFixThreads);
        P.close_in_sweep = g->fw.n_long == 0 && P.q_units <= kCloseInSweepUnits;
    }
    if (P.hot) {
        const int bytes = static_cast<int>(P.hot * sizeof(T));
        int sm_smem = 0;
        NKG_CUDA(cudaDeviceGetAttribute(&sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                                        g->device));
        require(sm_smem > 0, "device reports no shared memory");
        // Two CTAs of 768 threads per SM where two copies of the tier fit
        // (with the static scratch and the per-CTA reserve), else one of 1024.
        const int per_cta = bytes + 2048;
        const int copies = 2 * per_cta <= sm_smem ? 2 : 1;
        P.hot_threads = copies == 2 ? kHotThreadsPair : kHotThreads;
        auto kfn = copies == 2 ? sweep_kernel<T, WEIGHTED, kHotThreadsPair, kHotUnroll, true>
                               : sweep_kernel<T, WEIGHTED, kHotThreads, kHotUnroll, true>;
        // Carve out only what the CTAs need, leaving the rest of the SM's L1
        // to the gathers.
        const int carve = std::min(100, (copies * per_cta) * 100 / sm_smem + 1);
        NKG_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        NKG_CUDA(cudaFuncSetAttribute(kfn, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
        int hocc = 0;
        NKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&hocc, kfn, P.hot_threads, bytes));
        require(hocc >= 1, "shared-memory tier does not fit on an SM");
        P.hot_ctas = static_cast<unsigned>(std::max<uint64_t>(
            1, std::min<uint64_t>(static_cast<uint64_t>(hocc) * sms,
                                  (static_cast<uint64_t>(g->fw.slices) * 32 + P.hot_threads - 1) /
                                      P.hot_threads)));
        const uint64_t hwarps = static_cast<uint64_t>(P.hot_ctas) * (P.hot_threads / 32);
        P.hot_units = static_cast<uint32_t>(
            std::max<uint64_t>(1, std::min<uint64_t>(hwarps * kUnitsPerWarp, g->fw.slices)));
        P.hot_unit_start.alloc(static_cast<size_t>(P.hot_units) + 1);
        unit_bounds<<<ceil_div(static_cast<uint64_t>(P.hot_units) + 1, 256), 256, 0, s>>>(
            g->fw.slice_cost.get(), g->fw.slices, P.hot_units, P.hot_unit_start.get());
        NKG_CUDA(cudaGetLastError());
        require(P.hot_ctas <= g->cta_res.size(), "partial-sum buffers too small");
    }
    require(P.sweep_ctas <= g->cta_res.size() && P.fix_ctas <= g->fix_res.size(),
            "partial-sum buffers too small");
    NKG_CUDA(cudaStreamSynchronize(s));
}

template <typename T, bool WEIGHTED>
static SweepArgs<T> sweep_args(nkg_graph *g, int in_buf) {
    Plane<T> &P = plane<T>(g);
    SweepArgs<T> a{};
    a.col_sell = g->fw.col_sell.get();
    if (std::is_same<T, double>::value) {
        a.w_sell = reinterpret_cast<const T *>(g->fw.w_sell64.get());
        a.degw = reinterpret_cast<const T *>(g->degw64src.get());
    } else {
        a.w_sell = P.w_sell.get();
        a.degw = P.degw.get();
    }
    a.slice_off = g->fw.slice_off.get();
    a.unit_start = P.unit_start.get();
    a.chunk_begin = g->fw.chunk_begin.get();
    a.degc = g->degc.get();
    a.tele = P.tele.get();
    a.y_in = P.y[in_buf].get();
    a.y_out = P.y[in_buf ^ 1].get();
    a.chunk_val = P.chunk_val.get();
    a.cta_res = g->cta_res.get();
    a.cta_sink = g->cta_sink.get();
    a.fix_res = g->fix_res.get();
    a.fix_sink = g->fix_sink.get();
    a.rp = g->rp.get();
    a.st = g->st.get();
    a.n = static_cast<uint32_t>(g->n);
    a.n_long = g->fw.n_long;
    a.n_vlong = g->fw.n_vlong;
    a.s_chunk = g->fw.s_chunk;
    a.units = P.hot ? P.hot_units : P.units;
    a.sweep_ctas = P.hot ? P.hot_ctas : P.sweep_ctas;
    if (P.hot)
        a.unit_start = P.hot_unit_start.get();
    if (P.q_units) {
        a.units = P.q_units;
        a.unit_start = P.q_unit_start.get();
        a.unit_res = P.q_part.get();
        a.unit_sink = P.q_part.get() + P.q_units;
        a.close_in_sweep = P.close_in_sweep ? 1 : 0;
    }
    a.hot = P.hot;
    a.trace = g->trace.get();
    a.trace_cap = kTraceCapacity;
    return a;
}

template <typename T, bool WEIGHTED>
static void launch_sweep_kernel(nkg_graph *g, const SweepArgs<T> &a, cudaStream_t s) {
    Plane<T> &P = plane<T>(g);
    if (P.hot) {
        if (P.hot_threads == kHotThreadsPair)
            sweep_kernel<T, WEIGHTED, kHotThreadsPair, kHotUnroll, true>
                <<<P.hot_ctas, kHotThreadsPair, P.hot * sizeof(T), s>>>(a);
        else
            sweep_kernel<T, WEIGHTED, kHotThreads, kHotUnroll, true>
                <<<P.hot_ctas, kHotThreads, P.hot * sizeof(T), s>>>(a);
        return;
    }
    with_sweep_shape(g->sweep_shape, [&](auto S) {
        using Sh = decltype(S);
        sweep_kernel<T, WEIGHTED, Sh::threads, Sh::unroll, false, false, true>
            <<<P.sweep_ctas, Sh::threads, 0, s>>>(a);
    });
}

template <typename T, bool WEIGHTED>
static void launch_sweep(nkg_graph *g, int in_buf, cudaStream_t s) {
    Plane<T> &P = plane<T>(g);
    const SweepArgs<T> a = sweep_args<T, WEIGHTED>(g, in_buf);
    launch_sweep_kernel<T, WEIGHTED>(g, a, s);
    if (!P.close_in_sweep)
        fixup_kernel<T, WEIGHTED><<<P.fix_ctas, kFixThreads, 0, s>>>(a);
}

// Kernel launches of one iteration: the sweep, and the fix-up unless the
// sweep closes the iteration itself.
template <typename T>
static uint64_t launches_per_sweep(nkg_graph *g) {
    return plane<T>(g).close_in_sweep ? 1 : 2;
}

// Capture kSweepsPerGraph sweeps (sweep + fix-up each) as one CUDA graph.
template <typename T, bool WEIGHTED>
static cudaGraphExec_t sweep_graph(nkg_graph *g, int personal) {
    Plane<T> &P = plane<T>(g);
    cudaGraphExec_t &exec = P.exec[personal];
    if (exec)
        return exec;
    cudaStream_t s = g->stream;
    cudaGraph_t graph = nullptr;
    NKG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < kSweepsPerGraph; ++i)
        launch_sweep<T, WEIGHTED>(g, i & 1, s);
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    NKG_CUDA(e);
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    NKG_CUDA(e);
    return exec;
}

struct RunResult {
    uint64_t iterations = 0;
    double residual = 0.0, sink_mass = 0.0, maximum = 1.0;
    double ms_total = 0.0, ms_iter = 0.0;
    uint64_t launches = 0;
    uint64_t fp64_sweeps = 0, fp32_sweeps = 0;
    // Residuals of the sweeps with a stopping test: trace_length of them, in
    // g->trace on the device (power iterations, written by the fix-up) or in
    // host_trace (the FP64 sweeps of the refinement, read by the host).
    uint64_t trace_length = 0;
    bool device_trace = false;
    std::vector<double> host_trace;
};

// PageRank.cpp:75-102 on the final iterate yfin (gather form, this plane's
// precision), written to d_out in the caller's id order; fills the timings.
template <typename T, bool WEIGHTED>
static void finalize(nkg_graph *g, const nkg_pr_params &p, const T *yfin, double *d_out,
                     RunResult &R) {
    cudaStream_t s = g->stream;
    const uint32_t n = static_cast<uint32_t>(g->n);
    const T *degw = sweep_args<T, WEIGHTED>(g, 0).degw;
    const unsigned rblocks = std::min<unsigned>(num_sms(g->device) * 2, 4096);
    final_reduce<T, WEIGHTED><<<rblocks, kRedThreads, 0, s>>>(
        yfin, g->degc.get(), degw, n, g->red.get() + 4, g->red.get(), g->red_ticket.get());
    final_scale<T, WEIGHTED><<<ceil_div(g->z, 256), 256, 0, s>>>(
        yfin, g->degc.get(), degw, g->inv.get(), g->z, n, p.damp, p.normalized ? 1 : 0,
        g->red.get(), d_out);
    NKG_CUDA(cudaGetLastError());
    R.launches += 2;
    NKG_CUDA(cudaEventRecord(g->ev2, s));
    double *hs = g->scalars_host.get();
    NKG_CUDA(cudaMemcpyAsync(hs, g->red.get(), 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    NKG_CUDA(cudaStreamSynchronize(s));
    R.maximum = hs[3];
    float ms = 0.f;
    NKG_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev2));
    R.ms_total = ms;
    NKG_CUDA(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
    R.ms_iter = ms;
}

static uint64_t bytes_per_sweep(const nkg_graph *g, int elem) {
    // Algorithmic bytes of one sweep: column ids, row offsets, gathered
    // iterate (each value once), previous iterate, new iterate, degree
    // (+ weights and a weighted degree of `elem` bytes for weighted graphs).
    uint64_t b = 4 * g->arcs + 4 * (g->n + 1) + 3ull * elem * g->n;
    if (g->weighted)
        b += static_cast<uint64_t>(elem) * g->arcs + static_cast<uint64_t>(elem) * g->n;
    else
        b += 4 * g->n;
    return b;
}

template <typename T, bool WEIGHTED>
static void upload_run_state(nkg_graph *g, const nkg_pr_params &p, int personal,
                             const double *d_tele) {
    cudaStream_t s = g->stream;
    Plane<T> &P = plane<T>(g);
    const uint32_t n = static_cast<uint32_t>(g->n);
    RunParams *rp = reinterpret_cast<RunParams *>(g->scalars_host.get());
    static_assert(sizeof(RunParams) <= 8 * sizeof(double), "RunParams fits the pinned buffer");
    std::memset(rp, 0, sizeof(RunParams));
    rp->damp = p.damp;
    rp->tele_uniform = (1.0 - p.damp) / static_cast<double>(n);
    rp->one_minus_damp = 1.0 - p.damp;
    rp->inv_n = 1.0 / static_cast<double>(n);
    rp->distribute = p.distribute_sinks ? 1 : 0;
    rp->personal = personal;
    rp->l2 = p.norm == NKG_NORM_L2 ? 1 : 0;
    rp->tol = p.tol;
    rp->max_iterations = p.max_iterations;
    NKG_CUDA(cudaMemcpyAsync(g->rp.get(), rp, sizeof(RunParams), cudaMemcpyHostToDevice, s));
    const double x0 = 1.0 / static_cast<double>(n);
    if (personal) {
        if (!P.tele)
            P.tele.alloc(n);
        permute_teleport<T><<<ceil_div(n, 256), 256, 0, s>>>(d_tele, g->perm.get(), n,
                                                             P.tele.get());
    }
    const double S0 = static_cast<double>(g->sinks) * x0;
    IterState *sh = g->st_host.get();
    std::memset(sh, 0, sizeof(IterState));
    sh->sink_coef = p.distribute_sinks ? (personal ? S0 : S0 / static_cast<double>(n)) : 0.0;
    sh->sink_mass = S0;
    NKG_CUDA(cudaMemcpyAsync(g->st.get(), sh, sizeof(IterState), cudaMemcpyHostToDevice, s));
    init_iterate<T, WEIGHTED><<<ceil_div(n, 256), 256, 0, s>>>(
        P.y[0].get(), g->degc.get(), sweep_args<T, WEIGHTED>(g, 0).degw, n, x0);
    NKG_CUDA(cudaGetLastError());
}

template <typename T, bool WEIGHTED>
static RunResult run_power(nkg_graph *g, const nkg_pr_params &p, const double *d_tele,
                           double *d_out) {
    cudaStream_t s = g->stream;
    sweep_setup<T, WEIGHTED>(g);
    Plane<T> &P = plane<T>(g);
    const int personal = d_tele ? 1 : 0;
    RunResult R;

    NKG_CUDA(cudaEventRecord(g->ev0, s));
    upload_run_state<T, WEIGHTED>(g, p, personal, d_tele);
    R.launches += 1 + personal;

    cudaGraphExec_t exec = sweep_graph<T, WEIGHTED>(g, personal);
    IterState *sh = g->st_host.get();
    // Graph launches between status read-backs: 2, 4, 8, 8, ... (16 sweeps
    // first: a host round trip costs more than the no-op sweeps it saves).
    int batch = 2;
    for (;;) {
        for (int b = 0; b < batch; ++b)
            NKG_CUDA(cudaGraphLaunch(exec, s));
        R.launches += static_cast<uint64_t>(batch) * launches_per_sweep<T>(g) * kSweepsPerGraph;
        NKG_CUDA(cudaMemcpyAsync(sh, g->st.get(), sizeof(IterState), cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        if (sh->done)
            break;
        check_cancel(g, "PageRank run cancelled");
        batch = std::min(batch * 2, 8);
    }
    NKG_CUDA(cudaEventRecord(g->ev1, s));
    R.iterations = sh->iteration;
    R.residual = sh->residual;
    R.sink_mass = sh->sink_mass;
    R.trace_length = R.iterations;
    R.device_trace = true;
    const int fin = static_cast<int>(R.iterations & 1ull);
    finalize<T, WEIGHTED>(g, p, P.y[fin].get(), d_out, R);
    return R;
}

// FP32 BiCGSTAB bulk solve + FP64 Jacobi residual / correction rounds
// (refine.cuh). The stopping test is the reference's, applied to the FP64
// sweep: the returned scores are that sweep's iterate, like PageRank.cpp:70.
template <bool WEIGHTED>
static RunResult run_refine(nkg_graph *g, const nkg_pr_params &p, const double *d_tele,
                            double *d_out) {
    cudaStream_t s = g->stream;
    sweep_setup<float, WEIGHTED>(g);
    sweep_setup<double, WEIGHTED>(g);
    Plane<float> &P32 = g->p32;
    Plane<double> &P64 = g->p64;
    const int personal = d_tele ? 1 : 0;
    const uint32_t n = static_cast<uint32_t>(g->n);
    const unsigned sms = num_sms(g->device);
    RunResult R;
    NKG_CUDA(cudaEventRecord(g->ev0, s));
    nkg_pr_params p1 = p;
    p1.max_iterations = 1;  // every FP64 launch is exactly one Jacobi sweep
    upload_run_state<double, WEIGHTED>(g, p1, personal, d_tele);
    if (personal) {
        if (!P32.tele)
            P32.tele.alloc(n);
        permute_teleport<float><<<ceil_div(n, 256), 256, 0, s>>>(d_tele, g->perm.get(),
                                                                 n, P32.tele.get());
    }
    const unsigned vec_ctas = std::max<unsigned>(1, std::min<unsigned>(sms * 4, ceil_div(n, kBiThreads)));
    RefineWork &W = g->refine_work;
    if (!W.x64) {
        for (auto *v : {&W.x, &W.r, &W.rhat, &W.p, &W.v, &W.s, &W.t})
            v->alloc(n);
        W.g.alloc(n + 1, 4);
        W.x64.alloc(n);
        W.sc.alloc(sizeof(BiScalars));
        NKG_CUDA(cudaMemsetAsync(W.g.get(), 0, (n + 1 + 4) * sizeof(float), s));
    }
    const size_t part_n = 2 * static_cast<size_t>(std::max<unsigned>(P32.sweep_ctas, vec_ctas));
    if (W.part.size() < part_n)
        W.part.alloc(part_n);
    DeviceArray<float> &bx = W.x, &br = W.r, &brhat = W.rhat, &bp = W.p, &bv = W.v, &bs = W.s,
                       &bt = W.t, &bg = W.g;
    DeviceArray<double> &x64 = W.x64, &part = W.part;
    const unsigned fix_ctas = fix_ctas_with_units(split_fix_ctas<kBiThreads>(g->fw.n_long, g->fw.n_vlong),
                                                  P32.q_units, kBiThreads);
    if (W.fix_part.size() < 2 * static_cast<size_t>(fix_ctas))
        W.fix_part.alloc(2 * static_cast<size_t>(fix_ctas));
    DeviceArray<double> &fix_part = W.fix_part;
    BiScalars *scp = reinterpret_cast<BiScalars *>(W.sc.get());
    NKG_CUDA(cudaMemsetAsync(scp, 0, sizeof(BiScalars), s));
    BiArgs a{};
    a.col_sell = g->fw.col_sell.get();
    a.w_sell = P32.w_sell.get();
    a.slice_off = g->fw.slice_off.get();
    a.unit_start = P32.unit_start.get();
    a.chunk_begin = g->fw.chunk_begin.get();
    a.degc = g->degc.get();
    a.degw = P32.degw.get();
    a.tele = P32.tele.get();
    a.chunk_val = P32.chunk_val.get();
    a.x = bx.get();
    a.r = br.get();
    a.rhat = brhat.get();
    a.p = bp.get();
    a.v = bv.get();
    a.s = bs.get();
    a.t = bt.get();
    a.g = bg.get();
    a.part = part.get();
    a.fix_part = fix_part.get();
    a.sc = scp;
    a.damp = p.damp;
    a.inv_n = 1.0 / static_cast<double>(n);
    a.n = n;
    a.n_long = g->fw.n_long;
    a.n_vlong = g->fw.n_vlong;
    a.s_chunk = g->fw.s_chunk;
    a.units = P32.units;
    a.sweep_ctas = P32.sweep_ctas;
    if (P32.q_units) {
        // The queued cut of the FP32 sweep (bi_mv QUEUED).
        if (W.unit_part.size() < 2 * static_cast<size_t>(P32.q_units))
            W.unit_part.alloc(2 * static_cast<size_t>(P32.q_units));
        a.units = P32.q_units;
        a.unit_start = P32.q_unit_start.get();
        a.unit_part = W.unit_part.get();
    }
    a.distribute = p.distribute_sinks ? 1 : 0;
    a.personal = personal;
    a.l2 = p.norm == NKG_NORM_L2;
    BiScalars *hsc = reinterpret_cast<BiScalars *>(g->scalars_host.get());
    static_assert(sizeof(BiScalars) <= 16 * sizeof(double), "BiScalars fits the pinned buffer");

    BiLaunch bl;
    bl.stream = s;
    bl.sweep_shape = g->sweep_shape;
    bl.sweep_ctas = P32.sweep_ctas;
    bl.vec_ctas = vec_ctas;
    bl.fix_ctas = fix_ctas;
    bl.d_sc = scp;
    bl.h_sc = hsc;
    bl.cancel = &g->cancel;
    // Solve (I - dM) x = r (r holds the right-hand side).
    auto solve = [&](double rel) { bi_solve<WEIGHTED, 0>(a, bl, rel, 0.25 * p.tol); };

    cudaGraphExec_t exec = sweep_graph<double, WEIGHTED>(g, personal);
    IterState *sh = g->st_host.get();
    const double *degw64 = g->degw64src.get();
    bi_rhs_teleport<<<ceil_div(n, 256), 256, 0, s>>>(a);
    solve(1e-6);
    int add = 0;
    uint64_t fp64 = 0;
    for (int round = 0;; ++round) {
        require(round < 40, "FP32 refinement did not reach the tolerance in 40 rounds");
        std::memset(sh, 0, sizeof(IterState));
        NKG_CUDA(cudaMemcpyAsync(g->st.get(), sh, sizeof(IterState), cudaMemcpyHostToDevice, s));
        bi_to_fp64<WEIGHTED><<<vec_ctas, kBiThreads, 0, s>>>(
            bx.get(), x64.get(), P64.y[0].get(), g->degc.get(), degw64, n, add, part.get(),
            g->st.get(), &scp->ticket, a.distribute, personal);
        NKG_CUDA(cudaGraphLaunch(exec, s));
        R.launches += 1 + launches_per_sweep<double>(g) * kSweepsPerGraph;
        ++fp64;
        NKG_CUDA(cudaMemcpyAsync(sh, g->st.get(), sizeof(IterState), cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        if (R.host_trace.size() < kTraceCapacity)
            R.host_trace.push_back(sh->residual);
        if (sh->residual <= p.tol)
            break;
        bi_residual_rhs<WEIGHTED><<<ceil_div(n, 256), 256, 0, s>>>(
            P64.y[1].get(), x64.get(), g->degc.get(), degw64, n, br.get());
        solve(1e-5);
        add = 1;
    }
    NKG_CUDA(cudaEventRecord(g->ev1, s));
    R.iterations = fp64 + bl.matvecs;
    R.residual = sh->residual;
    R.sink_mass = sh->sink_mass;
    R.fp64_sweeps = fp64;
    R.fp32_sweeps = bl.matvecs;
    R.trace_length = fp64;
    R.launches += bl.launches;
    finalize<double, WEIGHTED>(g, p, P64.y[1].get(), d_out, R);
    return R;
}

static void check_params(const nkg_pr_params *p) {
    require(p != nullptr, "params is NULL");
    require(p->norm == NKG_NORM_L1 || p->norm == NKG_NORM_L2, "norm must be L1 (0) or L2 (1)");
    require(p->precision >= NKG_PREC_FP64 && p->precision <= NKG_PREC_FP32,
            "unknown precision");
    require(std::isfinite(p->damp), "damp must be finite");
    require(!std::isnan(p->tol), "tol must not be NaN");
}

static RunResult run_dispatch(nkg_graph *g, const nkg_pr_params *p, const double *teleport,
                              double *d_out) {
    check_params(p);
    DeviceGuard guard(g->device);
    RunScope scope(g);
    RunResult R;
    if (p->precision == NKG_PREC_FP64) {
        R = g->weighted ? run_power<double, true>(g, *p, teleport, d_out)
                        : run_power<double, false>(g, *p, teleport, d_out);
    } else if (p->precision == NKG_PREC_FP32) {
        R = g->weighted ? run_power<float, true>(g, *p, teleport, d_out)
                        : run_power<float, false>(g, *p, teleport, d_out);
    } else {
        R = g->weighted ? run_refine<true>(g, *p, teleport, d_out)
                        : run_refine<false>(g, *p, teleport, d_out);
    }
    g->has_run = true;
    return R;
}

static void fill_stats(const nkg_graph *g, const RunResult &R, int precision, nkg_stats *st) {
    if (!st)
        return;
    clear_stats(st);
    st->trace_length = R.trace_length;
    st->iterations = R.iterations;
    st->residual = R.residual;
    st->sink_mass = R.sink_mass;
    st->ms_total = R.ms_total;
    st->ms_iterations = R.ms_iter;
    st->kernel_launches = R.launches;
    if (precision == NKG_PREC_FP64) {
        st->fp64_sweeps = R.iterations;
    } else if (precision == NKG_PREC_FP32) {
        st->fp32_sweeps = R.iterations;
    } else {
        st->fp64_sweeps = R.fp64_sweeps;
        st->fp32_sweeps = R.fp32_sweeps;
    }
    st->bytes_per_sweep_fp64 = bytes_per_sweep(g, 8);
    st->bytes_per_sweep_fp32 = bytes_per_sweep(g, 4);
}

// Time `sweeps` sweeps with events around every sweep-kernel launch; the
// stopping test is disabled (tol < 0, no iteration cap).
template <typename T, bool WEIGHTED>
static void profile_sweeps(nkg_graph *g, int sweeps, double *ms_kernel, double *ms_iter) {
    cudaStream_t s = g->stream;
    sweep_setup<T, WEIGHTED>(g);
    Plane<T> &P = plane<T>(g);
    nkg_pr_params p{};
    p.damp = 0.85;
    p.tol = -1.0;
    p.norm = NKG_NORM_L1;
    p.max_iterations = ~0ull;
    upload_run_state<T, WEIGHTED>(g, p, 0, nullptr);
    std::vector<cudaEvent_t> ev(2 * static_cast<size_t>(sweeps), nullptr);
    for (auto &e : ev)
        NKG_CUDA(cudaEventCreate(&e));
    for (int i = 0; i < sweeps; ++i) {
        const SweepArgs<T> a = sweep_args<T, WEIGHTED>(g, i & 1);
        NKG_CUDA(cudaEventRecord(ev[2 * i], s));
        launch_sweep_kernel<T, WEIGHTED>(g, a, s);
        NKG_CUDA(cudaEventRecord(ev[2 * i + 1], s));
        if (!P.close_in_sweep)
            fixup_kernel<T, WEIGHTED><<<P.fix_ctas, kFixThreads, 0, s>>>(a);
    }
    NKG_CUDA(cudaGetLastError());
    NKG_CUDA(cudaStreamSynchronize(s));
    double sum = 0.0;
    for (int i = 0; i < sweeps; ++i) {
        float ms = 0.f;
        NKG_CUDA(cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]));
        sum += ms;
    }
    float total = 0.f;
    if (sweeps > 1)
        NKG_CUDA(cudaEventElapsedTime(&total, ev[0], ev[2 * (sweeps - 1)]));
    for (auto &e : ev)
        cudaEventDestroy(e);
    *ms_kernel = sum / sweeps;
    *ms_iter = sweeps > 1 ? total / (sweeps - 1) : sum;
}

// Diagnostic: only the gathers of a sweep - the same slot stream (the sliced
// layout's columns in storage order, padding included) into the same
// iterate - summed per thread, eight gathers in flight per thread. Its time
// is the random-gather bound of the graph on this GPU.
template <typename T>
__global__ void __launch_bounds__(256) gather_bound_kernel(const uint32_t *__restrict__ col,
                                                           uint64_t slots, const T *__restrict__ y,
                                                           T *__restrict__ sink) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    uint64_t i = t;
    T acc = 0;
    for (; i + 7 * stride < slots; i += 8 * stride) {
        uint32_t c[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            c[k] = col[i + k * stride];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            acc += y[c[k]];
    }
    for (; i < slots; i += stride)
        acc += y[col[i]];
    sink[t] = acc;
}

template <typename T, bool WEIGHTED>
static double profile_gathers(nkg_graph *g, int reps) {
    cudaStream_t s = g->stream;
    sweep_setup<T, WEIGHTED>(g);
    Plane<T> &P = plane<T>(g);
    nkg_pr_params p{};
    p.damp = 0.85;
    p.tol = -1.0;
    p.norm = NKG_NORM_L1;
    p.max_iterations = ~0ull;
    upload_run_state<T, WEIGHTED>(g, p, 0, nullptr);
    const unsigned blocks = num_sms(g->device) * 8;
    DeviceArray<T> sink(static_cast<size_t>(blocks) * 256);
    const uint64_t slots = g->fw.slots;  // entries of col_sell
    cudaEvent_t e0, e1;
    NKG_CUDA(cudaEventCreate(&e0));
    NKG_CUDA(cudaEventCreate(&e1));
    gather_bound_kernel<T><<<blocks, 256, 0, s>>>(g->fw.col_sell.get(), slots, P.y[0].get(),
                                                  sink.get());  // warm-up
    NKG_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; ++r)
        gather_bound_kernel<T><<<blocks, 256, 0, s>>>(g->fw.col_sell.get(), slots,
                                                      P.y[r & 1].get(), sink.get());
    NKG_CUDA(cudaEventRecord(e1, s));
    NKG_CUDA(cudaGetLastError());
    NKG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    NKG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / reps;
}

static int run_to(nkg_graph *g, const nkg_pr_params *p, const double *teleport, bool tele_is_host,
                  double *out, bool out_is_host, uint64_t *iters, double *max_out,
                  nkg_stats *stats) {
    return guarded([&] {
        require(g != nullptr, "graph handle is NULL");
        require(out != nullptr, "scores_out is NULL");
        DeviceGuard guard(g->device);
        DeviceArray<double> d_tele_tmp;
        if (teleport && tele_is_host) {
            d_tele_tmp.alloc(g->z);
            NKG_CUDA(cudaMemcpyAsync(d_tele_tmp.get(), teleport, g->z * sizeof(double),
                                     cudaMemcpyHostToDevice, g->stream));
            teleport = d_tele_tmp.get();
        }
        double *d_out = out;
        if (out_is_host) {
            if (!g->out_buf)
                g->out_buf.alloc(g->z);
            d_out = g->out_buf.get();
        }
        RunResult R = run_dispatch(g, p, teleport, d_out);
        if (out_is_host) {
            NKG_CUDA(cudaMemcpyAsync(out, d_out, g->z * sizeof(double), cudaMemcpyDeviceToHost,
                                     g->stream));
            NKG_CUDA(cudaStreamSynchronize(g->stream));
        }
        if (stats && stats->residual_trace && stats->trace_capacity) {
            const uint64_t k = std::min<uint64_t>(
                std::min<uint64_t>(R.trace_length, stats->trace_capacity), kTraceCapacity);
            if (R.device_trace) {
                NKG_CUDA(cudaMemcpyAsync(stats->residual_trace, g->trace.get(), k * sizeof(double),
                                         cudaMemcpyDeviceToHost, g->stream));
                NKG_CUDA(cudaStreamSynchronize(g->stream));
            } else {
                std::copy(R.host_trace.begin(),
                          R.host_trace.begin() + std::min<uint64_t>(k, R.host_trace.size()),
                          stats->residual_trace);
            }
        }
        if (iters)
            *iters = R.iterations;
        if (max_out)
            *max_out = R.maximum;
        fill_stats(g, R, p->precision, stats);
    });
}

// The process's SIGINT route of nkg_sigint_cancels: the handle whose runs a
// SIGINT cancels (the reference's root SignalHandler), the handler it
// replaced, and whether a SIGINT arrived. The handler only does lock-free
// atomic loads and stores, which are async-signal-safe.
static std::mutex g_sigint_mutex;
static std::atomic<nkg_graph *> g_sigint_owner{nullptr};
static std::atomic<int> g_sigint_seen{0};
static struct sigaction g_sigint_prev;

static void on_sigint(int) {
    g_sigint_seen.store(1);
    nkg_graph *g = g_sigint_owner.load();
    if (g)
        g->cancel.store(1);
}

static void ranking_prepare(double *keys, uint32_t *ids, const uint32_t *inv, uint64_t z,
                            cudaStream_t s) {
    ranking_prepare_kernel<<<ceil_div(z, 256), 256, 0, s>>>(keys, ids, inv, z);
    NKG_CUDA(cudaGetLastError());
}

} // namespace nkg

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

const char *nkg_last_error(void) { return nkg::g_last_error.c_str(); }

int nkg_abi_version(void) { return NKG_ABI_VERSION; }

int nkg_release_cached_memory(int device) {
    return guarded([&] {
        int dev = device;
        if (dev < 0)
            NKG_CUDA(cudaGetDevice(&dev));
        require(dev >= 0 && dev < kMaxDevices, "device ordinal out of range");
        DeviceGuard guard(dev);
        NKG_CUDA(cudaDeviceSynchronize());
        {
            std::lock_guard<std::mutex> lock(g_cache_mutex);
            release_blocks(g_cache[dev]);
        }
        std::lock_guard<std::mutex> lock(g_pinned_mutex);
        for (auto &kv : g_pinned_free)
            cudaFreeHost(kv.second);
        g_pinned_free.clear();
    });
}

int nkg_graph_create_ex(nkg_graph **out, uint64_t z, uint64_t arcs, const uint64_t *in_row_ptr,
                        const uint32_t *in_col, const double *in_w, const double *out_wdeg,
                        const uint8_t *exists, int directed, const nkg_graph_options *opts) {
    return guarded([&] {
        require(out != nullptr, "out is NULL");
        *out = nullptr;
        *out = create_graph(z, arcs, in_row_ptr, in_col, in_w, out_wdeg, exists, directed, opts);
    });
}

int nkg_graph_create_from_edges(nkg_graph **out, uint64_t z, uint64_t m, const uint32_t *src,
                                const uint32_t *dst, const double *w, const uint8_t *exists,
                                int directed, int flags, const nkg_graph_options *opts) {
    return guarded([&] {
        require(out != nullptr, "out is NULL");
        require((flags & ~NKG_DEVICE_PTRS) == 0, "unknown flags");
        *out = nullptr;
        *out = create_from_edges(z, m, src, dst, w, exists, directed,
                                 (flags & NKG_DEVICE_PTRS) != 0, opts);
    });
}

int nkg_graph_create(nkg_graph **out, uint64_t z, uint64_t arcs, const uint64_t *in_row_ptr,
                     const uint32_t *in_col, const double *in_w, const double *out_wdeg,
                     const uint8_t *exists, int directed) {
    return nkg_graph_create_ex(out, z, arcs, in_row_ptr, in_col, in_w, out_wdeg, exists, directed,
                               nullptr);
}

void nkg_graph_destroy(nkg_graph *g) {
    if (!g)
        return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    delete g;
    if (prev >= 0)
        cudaSetDevice(prev);
}

int nkg_graph_get_info(const nkg_graph *g, nkg_graph_info *info) {
    return guarded([&] {
        require(g != nullptr && info != nullptr, "NULL argument");
        std::memset(info, 0, sizeof(*info));
        info->z = g->z;
        info->n = g->n;
        info->arcs = g->arcs;
        info->sinks = g->sinks;
        info->slots = g->fw.slots;
        info->split_rows = g->fw.n_long;
        info->weighted = g->weighted;
        info->directed = g->directed;
        info->device = g->device;
        info->ms_create = g->ms_create;
        info->row_order = g->row_order;
    });
}

int nkg_pagerank_run(nkg_graph *g, const nkg_pr_params *p, double *scores_out,
                     uint64_t *iterations_out, double *max_out, nkg_stats *stats) {
    return run_to(g, p, nullptr, true, scores_out, true, iterations_out, max_out, stats);
}

int nkg_pagerank_run_device(nkg_graph *g, const nkg_pr_params *p, double *d_scores_out,
                            uint64_t *iterations_out, double *max_out, nkg_stats *stats) {
    return run_to(g, p, nullptr, true, d_scores_out, false, iterations_out, max_out, stats);
}

int nkg_pagerank_run_teleport(nkg_graph *g, const nkg_pr_params *p, const double *teleport,
                              double *scores_out, uint64_t *iterations_out, double *max_out,
                              nkg_stats *stats) {
    if (!teleport) {
        nkg::set_last_error("teleport is NULL");
        return NKG_ERR_INVALID_ARG;
    }
    return run_to(g, p, teleport, true, scores_out, true, iterations_out, max_out, stats);
}

int nkg_pagerank_run_ex(nkg_graph *g, const nkg_pr_params *p, const double *teleport,
                        double *scores_out, int flags, uint64_t *iterations_out, double *max_out,
                        nkg_stats *stats) {
    if (flags & ~NKG_DEVICE_PTRS) {
        nkg::set_last_error("unknown flags");
        return NKG_ERR_INVALID_ARG;
    }
    const bool host = (flags & NKG_DEVICE_PTRS) == 0;
    return run_to(g, p, teleport, host, scores_out, host, iterations_out, max_out, stats);
}

int nkg_ranking(nkg_graph *g, const double *scores, uint64_t *ids_out, double *vals_out) {
    return guarded([&] {
        require(g != nullptr && scores != nullptr, "NULL argument");
        DeviceGuard guard(g->device);
        cudaStream_t s = g->stream;
        const uint64_t z = g->z;
        DeviceArray<double> keys(z), keys_s(z);
        DeviceArray<uint32_t> ids(z), ids_s(z);
        NKG_CUDA(cudaMemcpyAsync(keys.get(), scores, z * sizeof(double), cudaMemcpyHostToDevice, s));
        ranking_prepare(keys.get(), ids.get(), g->inv.get(), z, s);
        size_t tmp_bytes = 0;
        NKG_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_bytes, keys.get(),
                                                           keys_s.get(), ids.get(), ids_s.get(),
                                                           static_cast<int64_t>(z), 0, 64, s));
        DeviceArray<unsigned char> tmp(tmp_bytes);
        NKG_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.get(), tmp_bytes, keys.get(),
                                                           keys_s.get(), ids.get(), ids_s.get(),
                                                           static_cast<int64_t>(z), 0, 64, s));
        const uint64_t n = g->n;
        std::vector<uint32_t> hid(n);
        if (vals_out)
            NKG_CUDA(cudaMemcpyAsync(vals_out, keys_s.get(), n * sizeof(double),
                                     cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaMemcpyAsync(hid.data(), ids_s.get(), n * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, s));
        NKG_CUDA(cudaStreamSynchronize(s));
        if (ids_out)
            for (uint64_t i = 0; i < n; ++i)
                ids_out[i] = hid[i];
    });
}

void nkg_cancel(nkg_graph *g) {
    if (g)
        g->cancel.store(1);
}

int nkg_sigint_cancels(nkg_graph *g, int enable, int *got_sigint_out) {
    return guarded([&] {
        require(g != nullptr, "graph handle is NULL");
        std::lock_guard<std::mutex> lock(nkg::g_sigint_mutex);
        if (enable) {
            nkg_graph *owner = nkg::g_sigint_owner.load();
            require(owner == nullptr || owner == g,
                    "SIGINT is already routed to another graph handle");
            if (owner == g)
                return;
            nkg::g_sigint_seen.store(0);
            nkg::g_sigint_owner.store(g);
            struct sigaction sa {};
            sa.sa_handler = nkg::on_sigint;
            sigemptyset(&sa.sa_mask);
            if (sigaction(SIGINT, &sa, &nkg::g_sigint_prev) != 0) {
                nkg::g_sigint_owner.store(nullptr);
                throw nkg::Error(NKG_ERR_INVALID_ARG, "sigaction(SIGINT) failed");
            }
        } else {
            if (nkg::g_sigint_owner.load() == g) {
                sigaction(SIGINT, &nkg::g_sigint_prev, nullptr);
                nkg::g_sigint_owner.store(nullptr);
            }
            if (got_sigint_out)
                *got_sigint_out = nkg::g_sigint_seen.load();
        }
    });
}

int nkg_profile_sweeps(nkg_graph *g, int precision, int sweeps, double *ms_sweep_kernel,
                       double *ms_iteration) {
    return guarded([&] {
        require(g != nullptr && ms_sweep_kernel != nullptr && ms_iteration != nullptr,
                "NULL argument");
        require(sweeps >= 1 && sweeps <= 100000, "sweeps must be in [1, 100000]");
        require(precision == NKG_PREC_FP64 || precision == NKG_PREC_FP32,
                "precision must be FP64 or FP32");
        DeviceGuard guard(g->device);
        if (precision == NKG_PREC_FP64) {
            if (g->weighted)
                profile_sweeps<double, true>(g, sweeps, ms_sweep_kernel, ms_iteration);
            else
                profile_sweeps<double, false>(g, sweeps, ms_sweep_kernel, ms_iteration);
        } else {
            if (g->weighted)
                profile_sweeps<float, true>(g, sweeps, ms_sweep_kernel, ms_iteration);
            else
                profile_sweeps<float, false>(g, sweeps, ms_sweep_kernel, ms_iteration);
        }
    });
}

int nkg_profile_gathers(nkg_graph *g, int precision, int reps, double *ms_gather_kernel) {
    return guarded([&] {
        require(g != nullptr && ms_gather_kernel != nullptr, "NULL argument");
        require(reps >= 1 && reps <= 100000, "reps must be in [1, 100000]");
        require(precision == NKG_PREC_FP64 || precision == NKG_PREC_FP32,
                "precision must be FP64 or FP32");
        DeviceGuard guard(g->device);
        if (precision == NKG_PREC_FP64)
            *ms_gather_kernel = g->weighted ? profile_gathers<double, true>(g, reps)
                                            : profile_gathers<double, false>(g, reps);
        else
            *ms_gather_kernel = g->weighted ? profile_gathers<float, true>(g, reps)
                                            : profile_gathers<float, false>(g, reps);
    });
}

} // extern "C"
