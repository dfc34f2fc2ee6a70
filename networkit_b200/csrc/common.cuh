// Shared host/device helpers of libnkgpu: error plumbing, RAII device
// buffers, warp/block reductions with a fixed combination order.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>

#include "nkgpu.h"

namespace nkg {

// Internal failure carrying an NKG_ERR_* code; the C-ABI wrappers turn it into
// a return code plus the thread-local message.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string &m);

inline void cuda_check(cudaError_t e, const char *what, const char *file, int line) {
    if (e == cudaSuccess)
        return;
    const int code = (e == cudaErrorMemoryAllocation) ? NKG_ERR_OOM
                     : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
                         ? NKG_ERR_NO_DEVICE
                         : NKG_ERR_CUDA;
    char buf[512];
    snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    throw Error(code, buf);
}

#define NKG_CUDA(call) ::nkg::cuda_check((call), #call, __FILE__, __LINE__)

inline void require(bool ok, const std::string &msg) {
    if (!ok)
        throw Error(NKG_ERR_INVALID_ARG, msg);
}

// Zero the statistics a call reports, keeping the caller's residual-trace
// array and its capacity (inputs of the struct).
inline void clear_stats(nkg_stats *st) {
    double *trace = st->residual_trace;
    const uint64_t cap = st->trace_capacity;
    *st = nkg_stats{};
    st->residual_trace = trace;
    st->trace_capacity = cap;
}

// Device memory of the library: cudaMalloc'ed blocks that are kept, once
// freed, in a per-device cache keyed by size, so that graph create / destroy
// cycles do not map and unmap gigabytes each time. device_free first waits
// for the device, as cudaFree does, then files the block in the cache.
// nkg_release_cached_memory hands the cached blocks back.
void *device_alloc(size_t bytes, int &device);
void device_free(void *p, int device);

// Page-locked host memory of the library: cudaHostAlloc'ed blocks kept, once
// freed, in a process-wide cache keyed by size (allocating and freeing
// page-locked memory costs milliseconds, more than a small graph's whole
// build). pinned_free files the block; the caller has waited for every copy
// that uses it. nkg_release_cached_memory hands the cached blocks back.
void *pinned_alloc(size_t bytes);
void pinned_free(void *p, size_t bytes);

// Streams of the library's handles: kept per device once a handle is
// destroyed (creating and destroying a stream costs about 0.1 ms). The
// stream returned is non-blocking and idle.
cudaStream_t stream_acquire(int device);
void stream_release(int device, cudaStream_t s);

// Owning device allocation (device_alloc/device_free). Sizes are in elements;
// the allocation is padded by `pad` elements so that vectorised or bulk copies
// that round an end offset up stay inside it.
template <typename T>
class DeviceArray {
  public:
    DeviceArray() = default;
    explicit DeviceArray(size_t n, size_t pad = 0) { alloc(n, pad); }
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    DeviceArray(DeviceArray &&o) noexcept : p_(o.p_), n_(o.n_), dev_(o.dev_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DeviceArray &operator=(DeviceArray &&o) noexcept {
        if (this != &o) {
            reset();
            p_ = o.p_;
            n_ = o.n_;
            dev_ = o.dev_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    ~DeviceArray() { reset(); }

    void alloc(size_t n, size_t pad = 0) {
        reset();
        const size_t bytes = (n + pad) * sizeof(T);
        if (bytes)
            p_ = static_cast<T *>(device_alloc(bytes, dev_));
        n_ = n;
    }
    void reset() {
        if (p_)
            device_free(p_, dev_);
        p_ = nullptr;
        n_ = 0;
    }
    T *get() const { return p_; }
    size_t size() const { return n_; }
    explicit operator bool() const { return p_ != nullptr; }

  private:
    T *p_ = nullptr;
    size_t n_ = 0;
    int dev_ = 0;
};

// Pinned host buffer (cudaHostAlloc) for status read-back.
template <typename T>
class PinnedHost {
  public:
    PinnedHost() = default;
    explicit PinnedHost(size_t n) { alloc(n); }
    void alloc(size_t n) {
        reset();
        p_ = static_cast<T *>(pinned_alloc(n * sizeof(T)));
        bytes_ = n * sizeof(T);
    }
    void reset() {
        if (p_)
            pinned_free(p_, bytes_);
        p_ = nullptr;
        bytes_ = 0;
    }
    PinnedHost(const PinnedHost &) = delete;
    PinnedHost &operator=(const PinnedHost &) = delete;
    ~PinnedHost() { reset(); }
    T *get() const { return p_; }

  private:
    T *p_ = nullptr;
    size_t bytes_ = 0;
};

constexpr uint32_t kNone = 0xffffffffu;

// Relabelling bucket of an in-degree d: half-octaves of d - 1 (0 for d <= 1).
// d > T for a power of two T is exactly bucket >= 2 log2(T) + 1, so rows
// longer than any power-of-two threshold stay a prefix of a bucket order.
__host__ __device__ inline uint32_t degree_bucket(uint32_t d) {
    if (d <= 1)
        return 0;
    const uint32_t x = d - 1;
    uint32_t e = 0;
    while ((x >> e) > 1)
        ++e;
    const uint32_t half = static_cast<uint64_t>(x) * x >= (1ull << (2 * e + 1)) ? 1u : 0u;
    return 2 * e + half + 1;
}

inline unsigned ceil_div(uint64_t a, uint64_t b) { return static_cast<unsigned>((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// Device helpers

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum with a fixed tree (deterministic for a fixed block size).
// Result valid in thread 0. `scratch` holds >= 32 doubles. Ends with a barrier
// so the scratch can be reused right away.
template <int THREADS>
__device__ __forceinline__ double block_sum(double v, double *scratch) {
    static_assert(THREADS % 32 == 0 && THREADS <= 1024, "block size");
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0)
        scratch[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = lane < THREADS / 32 ? scratch[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

template <int THREADS>
__device__ __forceinline__ double block_max(double v, double *scratch) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_max(v);
    if (lane == 0)
        scratch[wid] = v;
    __syncthreads();
    double r = -1.0 / 0.0;
    if (wid == 0) {
        r = lane < THREADS / 32 ? scratch[lane] : -1.0 / 0.0;
        r = warp_max(r);
    }
    __syncthreads();
    return r;
}

// Streaming read-only loads for data touched once per sweep: no L1
// allocation and an evict-first L2 policy, so both caches keep the gathered
// scores.
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;"
        : "=r"(v)
        : "l"(p), "l"(l2_evict_first_policy()));
    return v;
}
__device__ __forceinline__ float ld_stream(const float *p) {
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
        : "=f"(v)
        : "l"(p), "l"(l2_evict_first_policy()));
    return v;
}
__device__ __forceinline__ double ld_stream(const double *p) {
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;"
        : "=d"(v)
        : "l"(p), "l"(l2_evict_first_policy()));
    return v;
}

} // namespace nkg
